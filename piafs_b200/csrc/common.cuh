// Shared device-side definitions for the PIAFS GPU path.
//
// Device layout (structure of arrays): variable v of point p lives at
// u[v * ps + p], where p = (i + g) + W0 * (j + g) is the reference's point
// index (include/arrayfunctions.h:43-50) and ps is the plane stride (the
// ghosted point count rounded up to 32 doubles so every plane starts on a
// 256-byte boundary).  Interface arrays use the same scheme with the
// reference's interface index (bounds_inter, HyperbolicFunction.c:64-66):
// q = i + (N0+1) * j along x, q = i + N0 * j along y.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace piafs {

enum Model { EULER1D = 0, NS2D = 1 };
enum Scheme { WENO5 = 0, CRWENO5 = 1, UPW5 = 2 };   // UPW5: fifth-order upwind (hyp_space_scheme upw5)
enum Upwind { UPW_ROE = 0, UPW_RF = 1, UPW_LLF = 2, UPW_RUSANOV = 3 };
enum WenoType { W_JS = 0, W_MAPPED = 1, W_BORGES = 2, W_YC = 3 };
enum BcType {
  BC_PERIODIC = 0, BC_EXTRAPOLATE = 1, BC_SLIPWALL = 2, BC_DIRICHLET = 3, BC_REFLECT = 4,
  // flow boundaries of the Euler / Navier-Stokes models (2D in the reference)
  BC_NOSLIP = 5, BC_SUB_INFLOW = 6, BC_SUB_OUTFLOW = 7, BC_SUB_AMBIVALENT = 8, BC_SUP_INFLOW = 9,
  BC_SUP_OUTFLOW = 10
};

constexpr int MAX_ZONES = 16;
constexpr int MAX_STAGES = 4;

// Everything a kernel needs to know about one simulation; passed by value.
struct DevParams {
  int ndims, nvars, ghosts;
  int N0, N1;            // interior sizes (N1 = 1 in 1D)
  int W0, W1;            // ghosted sizes (W1 = 1 in 1D)
  int g1;                // ghosts along dim 1 (0 in 1D)
  long long npg;         // ghosted points
  long long ps;          // plane stride (points)
  long long nint[2];     // interfaces per direction
  long long pis;         // interface plane stride
  int model, scheme, upwind, weno_type, no_limiting;
  double eps;
  double gamma, bc_gamma, Re, Pr, Tref, T0, TS, TA, TB;
  int viscous;
  // photochemistry (normalised, ChemistryInitialize.c:267-353)
  int chem, nflow, nz, zstride;
  double k[11], q[11];
  double chem_gamma, I0, ch_c, ch_h, ch_nu, n_O2, t_start_norm, t_pulse_norm, sO3, dz;
  double dt;
  int mixed;             // 1: FP32 inner arithmetic on FP64 state (mixed precision)
  int char_interp;       // 1: WENO5 / upw5 on characteristic variables (hyp_interp_type characteristic)
  int par4;              // 1: fourth-order central first derivatives in the viscous terms (par_space_scheme 4)
  // rows [jg0, jg0 + N1) of a grid of N1g rows (a row slab of a decomposed
  // grid); 0 and N1 for a whole grid
  int jg0, N1g;
  // 1: the CRWENO5 line solve stores the passive variables' interface values
  // packed for their scalar upwinding -- uL - uR in the uL array, fL + fR in
  // the fL array -- and the upwind kernels read them so (2D Navier-Stokes,
  // upwinding other than RF)
  int pack_sp;
};

__host__ __device__ inline long long pidx(const DevParams& P, int i, int j) {
  return (long long)(i + P.ghosts) + (long long)P.W0 * (long long)(j + P.g1);
}

// ------------------------------------------------------------ flow variables
// _NavierStokes2DGetFlowVar_ (navierstokes2d.h:70-80)
template <typename T>
__device__ __forceinline__ void ns_flowvar(T rho_in, T ru, T rv, T e_in, T gamma, T& rho, T& vx,
                                           T& vy, T& e, T& P) {
  rho = rho_in;
  vx = (rho == T(0)) ? T(0) : ru / rho;
  vy = (rho == T(0)) ? T(0) : rv / rho;
  e = e_in;
  T vsq = (vx * vx) + (vy * vy);
  P = (e - T(0.5) * rho * vsq) * (gamma - T(1));
}
// _Euler1DGetFlowVar_ (euler1d.h:61-69)
template <typename T>
__device__ __forceinline__ void eu_flowvar(T rho_in, T ru, T e_in, T gamma, T& rho, T& v, T& e, T& P) {
  rho = rho_in;
  v = ru / rho;
  e = e_in;
  P = (e - T(0.5) * rho * v * v) * (gamma - T(1));
}

// Reciprocal 1/x of a finite, nonzero, normal x whose reciprocal is normal.
// From the hardware estimate y of PTX rcp.approx.ftz.f64, with relative
// error d (y = (1 - d)/x, so e = 1 - x y = d), one step of the third-order
// iteration y <- y + y (e + e^2) gives (1 - d)(1 + d + d^2)/x = (1 - d^3)/x:
// the estimate's error cubed, far below a unit in the last place, and the
// two rounded multiply-adds leave the result within a unit or two in the
// last place.  The step is the series 1/x = y / (1 - e) = y (1 + e + e^2 +
// ...) cut after e^2, a third-order relative of the Newton-Raphson
// refinement y <- y + y e (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34
// (1990) 111-119).  x = 0 gives NaN, which callers detect separately.
#ifdef __CUDACC__
// a product rounded on its own (never contracted into a following add), and
// a fused multiply-add, for sums whose terms are formed in different kernels
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}
// FP32 reciprocal of the mixed-precision inner arithmetic: the hardware
// approximation of PTX rcp.approx.ftz.f32 (within about 1 ulp of FP32).
__device__ __forceinline__ float rcp_nr(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
#endif

// --------------------------------------------------------------- WENO weights
// Nonlinear weights of the fifth-order WENO family for one stencil
// (m3,m2,m1,p1,p2) and optimal weights (c1,c2,c3).  Jiang-Shu, mapped
// (Henrick-Aslam-Powers), Borges (WENO-Z) and Yamaleev-Carpenter variants as
// selected in weno.inp (interpolation.h:255-545); WT_NONE (no_limiting) gives
// the optimal weights.  weno_alpha_t returns them unnormalised, a_k, with
// their normalising factor inv = 1 / sum a_k: a weight is w_k = a_k inv, and a
// reconstruction sum_k w_k f_k is formed as (sum_k a_k f_k) inv.  The
// Jiang-Shu a_k = c_k prod_{m!=k} q_m with q_m = (beta_m + eps)^2 (equal to
// c_k/q_k up to a common factor).  The smoothness indicators are kept at 4x
// their value with eps at 4x (and the Yamaleev-Carpenter tau at 4x), which
// scales all a_k of a stencil alike.  Quotients use rcp_nr (Newton-Raphson
// reciprocal), so weights agree with the reference's divisions to rounding.
constexpr int WT_NONE = 4;
// the linear fifth-order upwind scheme in place of WENO5 (upw5)
constexpr int WT_UPW5 = 5;

// the unnormalised weights from the stencil's three (4x) smoothness
// indicators and, for Z / YC, the reference indicator tau (4x)
template <int WT, typename T>
__device__ __forceinline__ void weno_alpha_b(T c1, T c2, T c3, T b1, T b2, T b3, T tau, T eps, T& a1, T& a2,
                                             T& a3, T& inv) {
  if (WT == WT_NONE) { a1 = c1; a2 = c2; a3 = c3; inv = T(1); return; }
  const T e4 = T(4) * eps;
  if (WT == W_JS || WT == W_MAPPED) {
    T s1 = b1 + e4, s2 = b2 + e4, s3 = b3 + e4;
    T q1 = s1 * s1, q2 = s2 * s2, q3 = s3 * s3;
    a1 = c1 * q2 * q3; a2 = c2 * q1 * q3; a3 = c3 * q1 * q2;
    inv = rcp_nr(a1 + a2 + a3);
    if (WT == W_MAPPED) {
      T x1 = a1 * inv, x2 = a2 * inv, x3 = a3 * inv;
      T n1 = x1 * (c1 + c1 * c1 - T(3) * c1 * x1 + x1 * x1), d1m = (c1 * c1 + x1 * (T(1) - T(2) * c1));
      T n2 = x2 * (c2 + c2 * c2 - T(3) * c2 * x2 + x2 * x2), d2m = (c2 * c2 + x2 * (T(1) - T(2) * c2));
      T n3 = x3 * (c3 + c3 * c3 - T(3) * c3 * x3 + x3 * x3), d3m = (c3 * c3 + x3 * (T(1) - T(2) * c3));
      a1 = n1 * rcp_nr(d1m); a2 = n2 * rcp_nr(d2m); a3 = n3 * rcp_nr(d3m);
      inv = rcp_nr(a1 + a2 + a3);
    }
    return;
  }
  if (WT == W_BORGES) tau = (b3 - b1) < T(0) ? (b1 - b3) : (b3 - b1);
  T r1 = tau * rcp_nr(b1 + e4), r2 = tau * rcp_nr(b2 + e4), r3 = tau * rcp_nr(b3 + e4);
  a1 = c1 * (T(1) + r1 * r1); a2 = c2 * (T(1) + r2 * r2); a3 = c3 * (T(1) + r3 * r3);
  inv = rcp_nr(a1 + a2 + a3);
}

template <int WT, typename T>
__device__ __forceinline__ void weno_alpha_t(T c1, T c2, T c3, T m3, T m2, T m1, T p1, T p2, T eps, T& a1, T& a2,
                                             T& a3, T& inv) {
  if (WT == WT_NONE) { a1 = c1; a2 = c2; a3 = c3; inv = T(1); return; }
  const T t1343 = T(13.0 / 3.0);
  T d1 = m3 - T(2) * m2 + m1, e1 = m3 - T(4) * m2 + T(3) * m1;
  T d2 = m2 - T(2) * m1 + p1, e2 = m2 - p1;
  T d3 = m1 - T(2) * p1 + p2, e3 = T(3) * m1 - T(4) * p1 + p2;
  T b1 = t1343 * d1 * d1 + e1 * e1;
  T b2 = t1343 * d2 * d2 + e2 * e2;
  T b3 = t1343 * d3 * d3 + e3 * e3;
  T tau = T(0);
  if (WT == W_YC) { T t = m3 - T(4) * m2 + T(6) * m1 - T(4) * p1 + p2; tau = T(4) * t * t; }
  weno_alpha_b<WT>(c1, c2, c3, b1, b2, b3, tau, eps, a1, a2, a3, inv);
}

// the normalised weights
template <int WT, typename T>
__device__ __forceinline__ void weno_weights_t(T c1, T c2, T c3, T m3, T m2, T m1, T p1, T p2, T eps, T& w1, T& w2,
                                               T& w3) {
  T a1, a2, a3, inv;
  weno_alpha_t<WT>(c1, c2, c3, m3, m2, m1, p1, p2, eps, a1, a2, a3, inv);
  w1 = a1 * inv; w2 = a2 * inv; w3 = a3 * inv;
}

template <typename T>
__device__ __forceinline__ void weno_weights(int type, T c1, T c2, T c3, T m3, T m2, T m1, T p1, T p2, T eps, T& w1,
                                             T& w2, T& w3) {
  switch (type) {
    case W_MAPPED: weno_weights_t<W_MAPPED>(c1, c2, c3, m3, m2, m1, p1, p2, eps, w1, w2, w3); break;
    case W_BORGES: weno_weights_t<W_BORGES>(c1, c2, c3, m3, m2, m1, p1, p2, eps, w1, w2, w3); break;
    case W_YC: weno_weights_t<W_YC>(c1, c2, c3, m3, m2, m1, p1, p2, eps, w1, w2, w3); break;
    default: weno_weights_t<W_JS>(c1, c2, c3, m3, m2, m1, p1, p2, eps, w1, w2, w3); break;
  }
}

// The fifth-order upwind value at an interface from the cells m3 .. p2 of its
// bias (Interp1PrimFifthOrderUpwind.c:118-126, the same five products in the
// same order)
template <typename T>
__device__ __forceinline__ T upw5_value(T m3, T m2, T m1, T p1, T p2) {
  return T(1.0 / 30.0) * m3 - T(13.0 / 60.0) * m2 + T(47.0 / 60.0) * m1 + T(27.0 / 60.0) * p1 - T(1.0 / 20.0) * p2;
}

// 3-point candidate values of explicit WENO5 (Interp1PrimFifthOrderWENO.c:144-146)
template <typename T>
__device__ __forceinline__ T weno5_value(T w1, T w2, T w3, T m3, T m2, T m1, T p1, T p2) {
  const T s = T(1.0 / 6.0);
  T f1 = (T(2) * s) * m3 + (T(-7) * s) * m2 + (T(11) * s) * m1;
  T f2 = (-s) * m2 + (T(5) * s) * m1 + (T(2) * s) * p1;
  T f3 = (T(2) * s) * m1 + (T(5) * s) * p1 + (-s) * p2;
  return w1 * f1 + w2 * f2 + w3 * f3;
}

// The four WENO5 interface values at one interface (Interp1PrimFifthOrderWENO.c
// for upw = +1 / -1 on u and f) with the weights of type WT (each value formed
// from the unnormalised weights, then scaled by their normalisation): a[0..5] and
// b[0..5] are u and f at cells i-3 .. i+2 around interface i; left-biased
// stencils use cells i-3..i+1, right-biased ones cells i+2..i-2.
// Both biases of one field at interface i from the cells c[0..5] = i-3 .. i+2:
// the left-biased stencil uses the windows (c0 c1 c2), (c1 c2 c3), (c2 c3 c4),
// the right-biased one (c3 c4 c5), (c2 c3 c4), (c1 c2 c3) read backwards, so
// the four windows' curvature terms (13/3 d^2) are computed once for both.
template <int WT, typename T>
__device__ __forceinline__ void weno5_pair_t(const T* c, T eps, T& vL, T& vR) {
  const T c1 = T(0.1), c2 = T(0.6), c3 = T(0.3);
  T a1, a2, a3, inv;
  if (WT == WT_UPW5) {
    vL = upw5_value(c[0], c[1], c[2], c[3], c[4]);
    vR = upw5_value(c[5], c[4], c[3], c[2], c[1]);
    return;
  }
  if (WT == WT_NONE) {
    vL = weno5_value(c1, c2, c3, c[0], c[1], c[2], c[3], c[4]);
    vR = weno5_value(c1, c2, c3, c[5], c[4], c[3], c[2], c[1]);
    return;
  }
  const T t1343 = T(13.0 / 3.0);
  T dd[4];
#pragma unroll
  for (int w = 0; w < 4; w++) {
    const T d = c[w] - T(2) * c[w + 1] + c[w + 2];
    dd[w] = t1343 * d * d;
  }
  // e-forms: x0 - 4 x1 + 3 x2, x0 - x2, 3 x0 - 4 x1 + x2 of window (x0 x1 x2)
  const T eA0 = c[0] - T(4) * c[1] + T(3) * c[2];
  const T eB1 = c[1] - c[3], eA1 = c[1] - T(4) * c[2] + T(3) * c[3];
  const T eC2 = T(3) * c[2] - T(4) * c[3] + c[4], eB2 = c[2] - c[4];
  const T eC3 = T(3) * c[3] - T(4) * c[4] + c[5];
  T tauL = T(0), tauR = T(0);
  if (WT == W_YC) {
    const T tl = c[0] - T(4) * c[1] + T(6) * c[2] - T(4) * c[3] + c[4];
    const T tr = c[5] - T(4) * c[4] + T(6) * c[3] - T(4) * c[2] + c[1];
    tauL = T(4) * tl * tl; tauR = T(4) * tr * tr;
  }
  weno_alpha_b<WT>(c1, c2, c3, dd[0] + eA0 * eA0, dd[1] + eB1 * eB1, dd[2] + eC2 * eC2, tauL, eps, a1, a2, a3,
                   inv);
  vL = weno5_value(a1, a2, a3, c[0], c[1], c[2], c[3], c[4]) * inv;
  weno_alpha_b<WT>(c1, c2, c3, dd[3] + eC3 * eC3, dd[2] + eB2 * eB2, dd[1] + eA1 * eA1, tauR, eps, a1, a2, a3,
                   inv);
  vR = weno5_value(a1, a2, a3, c[5], c[4], c[3], c[2], c[1]) * inv;
}

template <int WT, typename T>
__device__ __forceinline__ void weno5_iface_t(const T* a, const T* b, T eps, T& uL, T& uR, T& fL, T& fR) {
  weno5_pair_t<WT>(a, eps, uL, uR);
  weno5_pair_t<WT>(b, eps, fL, fR);
}

// the reconstruction of the explicit schemes: upw5, WENO5 with the optimal
// weights (no_limiting), or WENO5 with the deck's weights
__host__ __device__ inline int weno_kind(const DevParams& P) {
  return P.scheme == UPW5 ? WT_UPW5 : P.no_limiting ? WT_NONE : P.weno_type;
}

// weno5_iface_t for N independent interfaces with one branch on the weight
// type (the straight-line code of the N interfaces can be interleaved);
// o[n][0..3] = uL, uR, fL, fR of interface n.
template <int N, typename T>
__device__ __forceinline__ void weno5_iface_n(const DevParams& P, const T (*a)[6], const T (*b)[6], T (*o)[4]) {
  const T eps = (T)P.eps;
#define PIAFS_WENO_N(WT) \
  _Pragma("unroll") for (int n = 0; n < N; n++) weno5_iface_t<WT>(a[n], b[n], eps, o[n][0], o[n][1], o[n][2], o[n][3])
  switch (weno_kind(P)) {
    case WT_UPW5: PIAFS_WENO_N(WT_UPW5); break;
    case WT_NONE: PIAFS_WENO_N(WT_NONE); break;
    case W_MAPPED: PIAFS_WENO_N(W_MAPPED); break;
    case W_BORGES: PIAFS_WENO_N(W_BORGES); break;
    case W_YC: PIAFS_WENO_N(W_YC); break;
    default: PIAFS_WENO_N(W_JS); break;
  }
#undef PIAFS_WENO_N
}

// weno5_pair_t with the deck's weights
template <typename T>
__device__ __forceinline__ void weno5_pair(const DevParams& P, const T* c, T& vL, T& vR) {
  const T eps = (T)P.eps;
  switch (weno_kind(P)) {
    case WT_UPW5: weno5_pair_t<WT_UPW5>(c, eps, vL, vR); break;
    case WT_NONE: weno5_pair_t<WT_NONE>(c, eps, vL, vR); break;
    case W_MAPPED: weno5_pair_t<W_MAPPED>(c, eps, vL, vR); break;
    case W_BORGES: weno5_pair_t<W_BORGES>(c, eps, vL, vR); break;
    case W_YC: weno5_pair_t<W_YC>(c, eps, vL, vR); break;
    default: weno5_pair_t<W_JS>(c, eps, vL, vR); break;
  }
}

// the four WENO5 values at one interface with the deck's weights
template <typename T>
__device__ __forceinline__ void weno5_iface(const DevParams& P, const T* a, const T* b, T& uL, T& uR, T& fL,
                                            T& fR) {
  T o[1][4];
  weno5_iface_n<1, T>(P, (const T(*)[6])a, (const T(*)[6])b, o);
  uL = o[0][0]; uR = o[0][1]; fL = o[0][2]; fR = o[0][3];
}

}  // namespace piafs
