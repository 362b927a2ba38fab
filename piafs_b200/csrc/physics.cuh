// Device-side physics of the two models on the hot path: Roe averages,
// eigenvalues and the flow-block eigenvectors of 1D Euler and 2D
// Navier-Stokes, and the four interface upwinding schemes.
//
// The eigenvector matrices of both models are block diagonal: a 3x3 (Euler1D)
// or 4x4 (NS2D) flow block and the identity on the passively advected species
// (navierstokes2d.h:243-247, 307-311; euler1d.h:170-199).  Only the flow block
// is formed; species are handled with their scalar eigenvalue (the normal
// velocity), which is exactly what the reference's full nvars x nvars products
// reduce to.
#pragma once
#include "common.cuh"

namespace piafs {

template <int MODEL> struct Flow;

// ----------------------------------------------------------- 2D Navier-Stokes
template <> struct Flow<NS2D> {
  static constexpr int NF = 4;
  // _NavierStokes2DRoeAverage_ (navierstokes2d.h:115-159), flow variables
  template <typename T>
  __device__ static void roe_avg(const T* uL, const T* uR, T g, T* ua) {
    T rhoL = uL[0], vxL = uL[1] / rhoL, vyL = uL[2] / rhoL, eL = uL[3];
    T vsqL = vxL * vxL + vyL * vyL, PL = (eL - T(0.5) * rhoL * vsqL) * (g - T(1));
    T cLsq = g * PL / rhoL, HL = T(0.5) * (vxL * vxL + vyL * vyL) + cLsq / (g - T(1));
    T rhoR = uR[0], vxR = uR[1] / rhoR, vyR = uR[2] / rhoR, eR = uR[3];
    T vsqR = vxR * vxR + vyR * vyR, PR = (eR - T(0.5) * rhoR * vsqR) * (g - T(1));
    T cRsq = g * PR / rhoR, HR = T(0.5) * (vxR * vxR + vyR * vyR) + cRsq / (g - T(1));
    T tL = sqrt(rhoL), tR = sqrt(rhoR);
    T rho = tL * tR, inv = T(1) / (tL + tR);
    T vx = (tL * vxL + tR * vxR) * inv, vy = (tL * vyL + tR * vyR) * inv;
    T H = (tL * HL + tR * HR) * inv;
    T vsq = vx * vx + vy * vy;
    T csq = (g - T(1)) * (H - T(0.5) * vsq);
    T P = csq * rho / g;
    ua[0] = rho; ua[1] = rho * vx; ua[2] = rho * vy;
    ua[3] = P / (g - T(1)) + T(0.5) * rho * vsq;
  }
  // _NavierStokes2DEigenvalues_ (navierstokes2d.h:161-190); returns vn
  template <typename T>
  __device__ static T eigvals(const T* u, T g, int dir, T* D) {
    T rho, vx, vy, e, P;
    ns_flowvar(u[0], u[1], u[2], u[3], g, rho, vx, vy, e, P);
    T c = sqrt(g * P / rho);
    T vn = dir == 0 ? vx : vy;
    D[0] = vn - c;
    if (dir == 0) { D[1] = vn + c; D[2] = vn; } else { D[1] = vn; D[2] = vn + c; }
    D[3] = vn;
    return vn;
  }
  // _NavierStokes2DLeftEigenvectors_ / _RightEigenvectors_ (navierstokes2d.h:194-313)
  template <typename T>
  __device__ static void eigvec(const T* u, T ga, int dir, T L[4][4], T R[4][4]) {
    T gm1 = ga - T(1), rho, vx, vy, e, P;
    ns_flowvar(u[0], u[1], u[2], u[3], ga, rho, vx, vy, e, P);
    T ek = T(0.5) * (vx * vx + vy * vy);
    T a = sqrt(ga * P / rho);
    T a2 = a * a, i2a2 = T(1) / (T(2) * a2), ia2 = T(1) / a2;
    T h0 = a2 / gm1 + ek;
    if (dir == 0) {
      T un = vx;
      L[0][0] = (gm1 * ek + a * un) * i2a2; L[0][1] = ((-gm1) * vx - a) * i2a2;
      L[0][2] = ((-gm1) * vy) * i2a2;       L[0][3] = gm1 * i2a2;
      L[3][0] = (a2 - gm1 * ek) * ia2;      L[3][1] = (gm1 * vx) * ia2;
      L[3][2] = (gm1 * vy) * ia2;           L[3][3] = (-gm1) * ia2;
      L[1][0] = (gm1 * ek - a * un) * i2a2; L[1][1] = ((-gm1) * vx + a) * i2a2;
      L[1][2] = ((-gm1) * vy) * i2a2;       L[1][3] = gm1 * i2a2;
      L[2][0] = vy; L[2][1] = T(0); L[2][2] = T(-1); L[2][3] = T(0);
      R[0][0] = T(1); R[1][0] = vx - a; R[2][0] = vy; R[3][0] = h0 - a * un;
      R[0][3] = T(1); R[1][3] = vx;     R[2][3] = vy; R[3][3] = ek;
      R[0][1] = T(1); R[1][1] = vx + a; R[2][1] = vy; R[3][1] = h0 + a * un;
      R[0][2] = T(0); R[1][2] = T(0);   R[2][2] = T(-1); R[3][2] = -vy;
    } else {
      T un = vy;
      L[0][0] = (gm1 * ek + a * un) * i2a2; L[0][1] = ((T(1) - ga) * vx) * i2a2;
      L[0][2] = ((T(1) - ga) * vy - a) * i2a2; L[0][3] = gm1 * i2a2;
      L[3][0] = (a2 - gm1 * ek) * ia2;      L[3][1] = gm1 * vx * ia2;
      L[3][2] = gm1 * vy * ia2;             L[3][3] = (T(1) - ga) * ia2;
      L[2][0] = (gm1 * ek - a * un) * i2a2; L[2][1] = ((T(1) - ga) * vx) * i2a2;
      L[2][2] = ((T(1) - ga) * vy + a) * i2a2; L[2][3] = gm1 * i2a2;
      L[1][0] = -vx; L[1][1] = T(1); L[1][2] = T(0); L[1][3] = T(0);
      R[0][0] = T(1); R[1][0] = vx; R[2][0] = vy - a; R[3][0] = h0 - a * un;
      R[0][3] = T(1); R[1][3] = vx; R[2][3] = vy;     R[3][3] = ek;
      R[0][2] = T(1); R[1][2] = vx; R[2][2] = vy + a; R[3][2] = h0 + a * un;
      R[0][1] = T(0); R[1][1] = T(1); R[2][1] = T(0); R[3][1] = vx;
    }
  }
  template <typename T>
  __device__ static void sound_and_vn(const T* u, T g, int dir, T& c, T& vn) {
    T rho, vx, vy, e, P;
    ns_flowvar(u[0], u[1], u[2], u[3], g, rho, vx, vy, e, P);
    c = sqrt(g * P / rho);
    vn = dir == 0 ? vx : vy;
  }
};

// ------------------------------------------------------------------ 1D Euler
template <> struct Flow<EULER1D> {
  static constexpr int NF = 3;
  // _Euler1DRoeAverage_ (euler1d.h:93-125)
  template <typename T>
  __device__ static void roe_avg(const T* uL, const T* uR, T g, T* ua) {
    T rhoL = uL[0], vL = uL[1] / rhoL, eL = uL[2];
    T PL = (eL - T(0.5) * rhoL * vL * vL) * (g - T(1));
    T cLsq = g * PL / rhoL, HL = T(0.5) * vL * vL + cLsq / (g - T(1));
    T rhoR = uR[0], vR = uR[1] / rhoR, eR = uR[2];
    T PR = (eR - T(0.5) * rhoR * vR * vR) * (g - T(1));
    T cRsq = g * PR / rhoR, HR = T(0.5) * vR * vR + cRsq / (g - T(1));
    T tL = sqrt(rhoL), tR = sqrt(rhoR);
    T rho = tL * tR, inv = T(1) / (tL + tR);
    T v = (tL * vL + tR * vR) * inv, H = (tL * HL + tR * HR) * inv;
    T csq = (g - T(1)) * (H - T(0.5) * v * v);
    T P = csq * rho / g;
    ua[0] = rho; ua[1] = rho * v; ua[2] = P / (g - T(1)) + T(0.5) * rho * v * v;
  }
  // _Euler1DEigenvalues_ (euler1d.h:131-147)
  template <typename T>
  __device__ static T eigvals(const T* u, T g, int, T* D) {
    T rho, v, e, P;
    eu_flowvar(u[0], u[1], u[2], g, rho, v, e, P);
    T c = sqrt(g * P / rho);
    D[0] = v; D[1] = v - c; D[2] = v + c;
    return v;
  }
  // _Euler1DLeftEigenvectors_ / _RightEigenvectors_ (euler1d.h:153-200)
  template <typename T>
  __device__ static void eigvec(const T* u, T gamma, int, T L[4][4], T R[4][4]) {
    T rho, v, e, P;
    eu_flowvar(u[0], u[1], u[2], gamma, rho, v, e, P);
    T c = sqrt(gamma * P / rho);
    T gm1 = gamma - T(1), f = gm1 / (rho * c), ic = T(1) / c, i2c = T(1) / (T(2) * c);
    L[1][0] = f * (-(v * v) / T(2) - c * v / gm1);
    L[1][1] = f * (v + c / gm1);
    L[1][2] = -f;
    L[0][0] = f * (rho * (-(v * v) / T(2) + c * c / gm1) * ic);
    L[0][1] = f * (rho * v * ic);
    L[0][2] = f * (-rho * ic);
    L[2][0] = f * ((v * v) / T(2) - c * v / gm1);
    L[2][1] = f * (-v + c / gm1);
    L[2][2] = f;
    R[0][1] = -rho * i2c; R[1][1] = -rho * (v - c) * i2c;
    R[2][1] = -rho * ((v * v) / T(2) + (c * c) / gm1 - c * v) * i2c;
    R[0][0] = T(1); R[1][0] = v; R[2][0] = v * v / T(2);
    R[0][2] = rho * i2c; R[1][2] = rho * (v + c) * i2c;
    R[2][2] = rho * ((v * v) / T(2) + (c * c) / gm1 + c * v) * i2c;
  }
};

// Cell-centred fluxes of the flow variables along dir (NavierStokes2DFlux.c:
// 24-52, Euler1DFlux.c) and the normal velocity that scales the passive
// variables (F_m = vn u_m).  Products and sums are rounded operations that the
// compiler never contracts into a neighbouring FMA, so a flux has the same
// bits whether it is stored and reloaded (the single-simulation kernels) or
// consumed in registers (the batched stage kernel).
__device__ __forceinline__ void ns2d_flux(double u0, double u1, double u2, double u3, double gamma, int dir,
                                          double* f, double& vn) {
  double rho, vx, vy, e, pr;
  ns_flowvar(u0, u1, u2, u3, gamma, rho, vx, vy, e, pr);
  vn = dir == 0 ? vx : vy;
  f[0] = __dmul_rn(rho, vn);
  if (dir == 0) {
    f[1] = __fma_rn(__dmul_rn(rho, vx), vx, pr);
    f[2] = __dmul_rn(__dmul_rn(rho, vx), vy);
  } else {
    f[1] = __dmul_rn(__dmul_rn(rho, vy), vx);
    f[2] = __fma_rn(__dmul_rn(rho, vy), vy, pr);
  }
  f[3] = __dmul_rn(__dadd_rn(e, pr), vn);
}
__device__ __forceinline__ void euler1d_flux(double u0, double u1, double u2, double gamma, double* f, double& vn) {
  double rho, v, e, pr;
  eu_flowvar(u0, u1, u2, gamma, rho, v, e, pr);
  vn = v;
  f[0] = __dmul_rn(rho, v);
  f[1] = __fma_rn(__dmul_rn(rho, v), v, pr);
  f[2] = __dmul_rn(__dadd_rn(e, pr), v);
}

// Reciprocal in the working precision: rcp_nr (common.cuh) for both types.
template <typename T> __device__ __forceinline__ T rcpw(T x) { return rcp_nr(x); }

// The characteristic-upwinding set-up of 2D Navier-Stokes at one interface
// (NavierStokes2DUpwind.c:190-260 / 271-332): the Roe average of the two
// interface states (_NavierStokes2DRoeAverage_, navierstokes2d.h:115-159),
// its left / right eigenvectors (_NavierStokes2DLeftEigenvectors_ /
// _RightEigenvectors_, :194-313) and the eigenvalues at the left, right and
// averaged states (_NavierStokes2DEigenvalues_, :161-190).  The same
// formulas as Flow<NS2D>::roe_avg / eigvec / eigvals, evaluated once per
// state: each state's velocity, pressure and sound speed are formed once
// and shared by the average and the eigenvalues, quotients by a density or by
// a^2 are products with one reciprocal (rcp_nr), and the averaged state's
// velocity, sound speed and enthalpy are used as computed rather than
// re-derived from its conserved variables -- 4 reciprocals and 5 square
// roots per interface where the per-macro form takes 25 divisions and 7
// roots.  The results agree with the macro form to rounding.
template <typename T>
__device__ __forceinline__ void ns2d_char_setup(const T* uL, const T* uR, T g, int dir, T L[4][4], T R[4][4],
                                                T* eL, T* eR, T* eC, T& vnL, T& vnR, T& vnC) {
  const T gm1 = g - T(1), igm1 = rcpw(gm1);
  // one side: rho, velocity, pressure (_NavierStokes2DGetFlowVar_,
  // navierstokes2d.h:70-80), c^2 = gamma P / rho, enthalpy
  auto side = [&](const T* u, T& rho, T& vx, T& vy, T& csq, T& H) {
    rho = u[0];
    const T ir = rho == T(0) ? T(0) : rcpw(rho);
    vx = u[1] * ir;
    vy = u[2] * ir;
    const T vsq = vx * vx + vy * vy;
    const T P = (u[3] - T(0.5) * rho * vsq) * gm1;
    csq = g * P * ir;
    H = T(0.5) * vsq + csq * igm1;
  };
  T rhoL, vxL, vyL, cLsq, HL, rhoR, vxR, vyR, cRsq, HR;
  side(uL, rhoL, vxL, vyL, cLsq, HL);
  side(uR, rhoR, vxR, vyR, cRsq, HR);
  const T cL = sqrt(cLsq), cR = sqrt(cRsq);
  // Roe average
  const T tL = sqrt(rhoL), tR = sqrt(rhoR);
  const T inv = rcpw(tL + tR);
  const T vx = (tL * vxL + tR * vxR) * inv, vy = (tL * vyL + tR * vyR) * inv;
  const T H = (tL * HL + tR * HR) * inv;
  const T ek = T(0.5) * (vx * vx + vy * vy);
  const T a = sqrt(gm1 * (H - ek));
  // eigenvalues (x: u-c, u+c, u, u; y: v-c, v, v+c, v)
  vnL = dir == 0 ? vxL : vyL;
  vnR = dir == 0 ? vxR : vyR;
  vnC = dir == 0 ? vx : vy;
  auto eig = [&](T vn, T c, T* D) {
    D[0] = vn - c;
    if (dir == 0) { D[1] = vn + c; D[2] = vn; } else { D[1] = vn; D[2] = vn + c; }
    D[3] = vn;
  };
  eig(vnL, cL, eL);
  eig(vnR, cR, eR);
  eig(vnC, a, eC);
  // eigenvectors of the averaged state
  const T a2 = a * a, ia2 = rcpw(a2), i2a2 = T(0.5) * ia2;
  const T h0 = a2 * igm1 + ek;
  if (dir == 0) {
    const T un = vx;
    L[0][0] = (gm1 * ek + a * un) * i2a2; L[0][1] = ((-gm1) * vx - a) * i2a2;
    L[0][2] = ((-gm1) * vy) * i2a2;       L[0][3] = gm1 * i2a2;
    L[3][0] = (a2 - gm1 * ek) * ia2;      L[3][1] = (gm1 * vx) * ia2;
    L[3][2] = (gm1 * vy) * ia2;           L[3][3] = (-gm1) * ia2;
    L[1][0] = (gm1 * ek - a * un) * i2a2; L[1][1] = ((-gm1) * vx + a) * i2a2;
    L[1][2] = ((-gm1) * vy) * i2a2;       L[1][3] = gm1 * i2a2;
    L[2][0] = vy; L[2][1] = T(0); L[2][2] = T(-1); L[2][3] = T(0);
    R[0][0] = T(1); R[1][0] = vx - a; R[2][0] = vy; R[3][0] = h0 - a * un;
    R[0][3] = T(1); R[1][3] = vx;     R[2][3] = vy; R[3][3] = ek;
    R[0][1] = T(1); R[1][1] = vx + a; R[2][1] = vy; R[3][1] = h0 + a * un;
    R[0][2] = T(0); R[1][2] = T(0);   R[2][2] = T(-1); R[3][2] = -vy;
  } else {
    const T un = vy;
    L[0][0] = (gm1 * ek + a * un) * i2a2; L[0][1] = ((T(1) - g) * vx) * i2a2;
    L[0][2] = ((T(1) - g) * vy - a) * i2a2; L[0][3] = gm1 * i2a2;
    L[3][0] = (a2 - gm1 * ek) * ia2;      L[3][1] = gm1 * vx * ia2;
    L[3][2] = gm1 * vy * ia2;             L[3][3] = (T(1) - g) * ia2;
    L[2][0] = (gm1 * ek - a * un) * i2a2; L[2][1] = ((T(1) - g) * vx) * i2a2;
    L[2][2] = ((T(1) - g) * vy + a) * i2a2; L[2][3] = gm1 * i2a2;
    L[1][0] = -vx; L[1][1] = T(1); L[1][2] = T(0); L[1][3] = T(0);
    R[0][0] = T(1); R[1][0] = vx; R[2][0] = vy - a; R[3][0] = h0 - a * un;
    R[0][3] = T(1); R[1][3] = vx; R[2][3] = vy;     R[3][3] = ek;
    R[0][2] = T(1); R[1][2] = vx; R[2][2] = vy + a; R[3][2] = h0 + a * un;
    R[0][1] = T(0); R[1][1] = T(1); R[2][1] = T(0); R[3][1] = vx;
  }
}

template <typename T> __device__ __forceinline__ T absv(T a) { return a < T(0) ? -a : a; }
template <typename T> __device__ __forceinline__ T maxv(T a, T b) { return a > b ? a : b; }
template <typename T> __device__ __forceinline__ T max3v(T a, T b, T c) { return maxv(maxv(a, b), maxv(b, c)); }

// Upwind flux of the flow block at one interface.  Inputs hold NF flow
// values; uCL/uCR are the cell-centred states left and right of the interface.
// Returns the species dissipation speed (scalar eigenvalue treatment) in
// *sp_alpha and the species scheme selector in *sp_mode:
//   mode 0: fI = 0.5(fL+fR) - alpha*0.5(uR-uL)     (Roe, Rusanov)
//   mode 1: fI = 0.5(fL+fR + alpha(uL-uR))         (LLF, RF mixed)
//   mode 2: fI = fL ; mode 3: fI = fR               (RF pure upwind)
// Reference: NavierStokes2DUpwind.c:26-332, Euler1DUpwind.c:27-330.
template <int MODEL, int UPW, typename T>
__device__ void upwind_flow(const T* uL, const T* uR, const T* fL, const T* fR, const T* uCL,
                            const T* uCR, T g, int dir, T* fI, T* sp_alpha, int* sp_mode) {
  typedef Flow<MODEL> F;
  constexpr int NF = F::NF;
  T ua[4], D[4];
  if (UPW == UPW_ROE) {
    T L[4][4], R[4][4];
    F::roe_avg(uCL, uCR, g, ua);
    T vn = F::eigvals(ua, g, dir, D);
    F::eigvec(ua, g, dir, L, R);
    T Ds[4], dsp;
    if (MODEL == NS2D) {
      // entropy fix, delta = 1e-6 (NavierStokes2DUpwind.c:75-78)
      const T delta = T(0.000001), delta2 = delta * delta, i2d = T(1) / (T(2) * delta);
#pragma unroll
      for (int a = 0; a < NF; a++) Ds[a] = absv(D[a]) < delta ? (D[a] * D[a] + delta2) * i2d : absv(D[a]);
      dsp = absv(vn) < delta ? (vn * vn + delta2) * i2d : absv(vn);
    } else {
#pragma unroll
      for (int a = 0; a < NF; a++) Ds[a] = absv(D[a]);
      dsp = absv(vn);
    }
    T ud[4], w[4];
#pragma unroll
    for (int a = 0; a < NF; a++) ud[a] = T(0.5) * (uR[a] - uL[a]);
#pragma unroll
    for (int a = 0; a < NF; a++) {
      T s = T(0);
#pragma unroll
      for (int b = 0; b < NF; b++) s += L[a][b] * ud[b];
      w[a] = Ds[a] * s;
    }
#pragma unroll
    for (int a = 0; a < NF; a++) {
      T s = T(0);
#pragma unroll
      for (int b = 0; b < NF; b++) s += R[a][b] * w[b];
      fI[a] = T(0.5) * (fL[a] + fR[a]) - s;
    }
    *sp_alpha = dsp; *sp_mode = 0;
  } else if (UPW == UPW_RUSANOV) {
    F::roe_avg(uCL, uCR, g, ua);
    T cL, cR, cA, vL, vR, vA;
    if (MODEL == NS2D) {
      Flow<NS2D>::sound_and_vn(uCL, g, dir, cL, vL);
      Flow<NS2D>::sound_and_vn(uCR, g, dir, cR, vR);
      Flow<NS2D>::sound_and_vn(ua, g, dir, cA, vA);
    } else {
      // the 1D Rusanov speed uses gamma*P/rho without the square root
      // (Euler1DUpwind.c, Euler1DUpwindRusanov)
      T rho, v, e, P;
      eu_flowvar(uCL[0], uCL[1], uCL[2], g, rho, v, e, P); cL = g * P / rho; vL = v;
      eu_flowvar(uCR[0], uCR[1], uCR[2], g, rho, v, e, P); cR = g * P / rho; vR = v;
      eu_flowvar(ua[0], ua[1], ua[2], g, rho, v, e, P); cA = g * P / rho; vA = v;
    }
    T alpha = max3v(cL + absv(vL), cR + absv(vR), cA + absv(vA));
#pragma unroll
    for (int a = 0; a < NF; a++) fI[a] = T(0.5) * (fL[a] + fR[a]) - alpha * (T(0.5) * (uR[a] - uL[a]));
    *sp_alpha = alpha; *sp_mode = 0;
  } else {
    // characteristic LLF / RF
    T L[4][4], R[4][4], eL[4], eR[4], eC[4], vnL, vnR, vnC;
    if (MODEL == NS2D) {
      ns2d_char_setup<T>(uL, uR, g, dir, L, R, eL, eR, eC, vnL, vnR, vnC);
    } else {
      // Euler1D averages and evaluates the eigenvalues at the cell centres
      F::roe_avg(uCL, uCR, g, ua);
      F::eigvec(ua, g, dir, L, R);
      vnL = F::eigvals(uCL, g, dir, eL);
      vnR = F::eigvals(uCR, g, dir, eR);
      vnC = F::eigvals(ua, g, dir, eC);
    }
    T fc[4];
#pragma unroll
    for (int a = 0; a < NF; a++) {
      T ucL = T(0), ucR = T(0), fcL = T(0), fcR = T(0);
#pragma unroll
      for (int b = 0; b < NF; b++) {
        ucL += L[a][b] * uL[b]; ucR += L[a][b] * uR[b];
        fcL += L[a][b] * fL[b]; fcR += L[a][b] * fR[b];
      }
      if (UPW == UPW_RF && eL[a] > T(0) && eC[a] > T(0) && eR[a] > T(0)) fc[a] = fcL;
      else if (UPW == UPW_RF && eL[a] < T(0) && eC[a] < T(0) && eR[a] < T(0)) fc[a] = fcR;
      else {
        T alpha = max3v(absv(eL[a]), absv(eC[a]), absv(eR[a]));
        fc[a] = T(0.5) * (fcL + fcR + alpha * (ucL - ucR));
      }
    }
#pragma unroll
    for (int a = 0; a < NF; a++) {
      T s = T(0);
#pragma unroll
      for (int b = 0; b < NF; b++) s += R[a][b] * fc[b];
      fI[a] = s;
    }
    if (UPW == UPW_RF && vnL > T(0) && vnC > T(0) && vnR > T(0)) *sp_mode = 2;
    else if (UPW == UPW_RF && vnL < T(0) && vnC < T(0) && vnR < T(0)) *sp_mode = 3;
    else *sp_mode = 1;
    *sp_alpha = max3v(absv(vnL), absv(vnC), absv(vnR));
  }
}

// Deviation form of upwind_flow for the mixed-precision path.  uL, uR, fL,
// fR are taken relative to constants shared by both sides of the interface
// (the reference values of the interface's grid line); uAL / uAR are the
// absolute interface states (the NS2D characteristic schemes take the Roe
// average and the eigenvalues from them) and uCL / uCR the absolute
// cell-centred states.  The flux comes back relative to the same constant as
// fL and fR.  With fbar = (fL + fR) / 2, every scheme is fI = fbar + R s (or
// fbar - R |D| L (uR - uL) / 2 for Roe), with s formed from differences of
// the inputs only, so no O(1) background goes through FP32 rounding before
// the divergence differences the interface fluxes.  Mathematically equal to
// upwind_flow on the absolute values.
template <int MODEL, int UPW, typename T>
__device__ void upwind_flow_dev(const T* uL, const T* uR, const T* fL, const T* fR, const T* uAL, const T* uAR,
                                const T* uCL, const T* uCR, T g, int dir, T* fI, T* sp_alpha, int* sp_mode) {
  typedef Flow<MODEL> F;
  constexpr int NF = F::NF;
  if (UPW == UPW_ROE || UPW == UPW_RUSANOV) {   // these are in deviation form already
    upwind_flow<MODEL, UPW, T>(uL, uR, fL, fR, uCL, uCR, g, dir, fI, sp_alpha, sp_mode);
    return;
  }
  T ua[4], L[4][4], R[4][4], eL[4], eR[4], eC[4], vnL, vnR, vnC;
  if (MODEL == NS2D) {
    ns2d_char_setup<T>(uAL, uAR, g, dir, L, R, eL, eR, eC, vnL, vnR, vnC);
  } else {
    F::roe_avg(uCL, uCR, g, ua);
    F::eigvec(ua, g, dir, L, R);
    vnL = F::eigvals(uCL, g, dir, eL);
    vnR = F::eigvals(uCR, g, dir, eR);
    vnC = F::eigvals(ua, g, dir, eC);
  }
  T sc[4];
#pragma unroll
  for (int a = 0; a < NF; a++) {
    T df = T(0), du = T(0);
#pragma unroll
    for (int b = 0; b < NF; b++) { df += L[a][b] * (fL[b] - fR[b]); du += L[a][b] * (uL[b] - uR[b]); }
    if (UPW == UPW_RF && eL[a] > T(0) && eC[a] > T(0) && eR[a] > T(0)) sc[a] = T(0.5) * df;
    else if (UPW == UPW_RF && eL[a] < T(0) && eC[a] < T(0) && eR[a] < T(0)) sc[a] = T(-0.5) * df;
    else sc[a] = T(0.5) * max3v(absv(eL[a]), absv(eC[a]), absv(eR[a])) * du;
  }
#pragma unroll
  for (int a = 0; a < NF; a++) {
    T s = T(0);
#pragma unroll
    for (int b = 0; b < NF; b++) s += R[a][b] * sc[b];
    fI[a] = T(0.5) * (fL[a] + fR[a]) + s;
  }
  if (UPW == UPW_RF && vnL > T(0) && vnC > T(0) && vnR > T(0)) *sp_mode = 2;
  else if (UPW == UPW_RF && vnL < T(0) && vnC < T(0) && vnR < T(0)) *sp_mode = 3;
  else *sp_mode = 1;
  *sp_alpha = max3v(absv(vnL), absv(vnC), absv(vnR));
}

template <typename T>
__device__ __forceinline__ T upwind_species(int mode, T alpha, T uL, T uR, T fL, T fR) {
  if (mode == 0) return T(0.5) * (fL + fR) - alpha * (T(0.5) * (uR - uL));
  if (mode == 1) return T(0.5) * (fL + fR + alpha * (uL - uR));
  return mode == 2 ? fL : fR;
}
// the same for modes 0 and 1 from the packed values du = uL - uR and
// sf = fL + fR (uR - uL = -du exactly, so the values are the same)
template <typename T>
__device__ __forceinline__ T upwind_species_packed(int mode, T alpha, T du, T sf) {
  if (mode == 0) return T(0.5) * sf - alpha * (T(0.5) * (-du));
  return T(0.5) * (sf + alpha * du);
}

}  // namespace piafs
