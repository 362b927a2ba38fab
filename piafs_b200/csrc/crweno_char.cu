// CRWENO5 on characteristic variables with its block-tridiagonal line solves
// (Interp1PrimFifthOrderCRWENOChar.c:96-266 with blocktridiagLU.c:146-300,
// serial path), for the models whose blocks the reference can invert: 1D
// Euler (3x3 blocks) and 2D Navier-Stokes without chemistry (4x4).
//
// The reference builds, at interface i of a line and for each characteristic
// field v, the block rows
//   A_i[v][:] = a_v L_i[v][:],  B_i[v][:] = b_v L_i[v][:],  C_i[v][:] = c_v L_i[v][:]
// (L_i: left eigenvectors of the Roe average of the two cells beside the
// interface; a, b, c from the field's WENO weights on its projected stencil),
// right-hand side F_i[v] = w1 f1 + w2 f2 + w3 f3 of the projected compact
// candidates, and solves sum A_i x_{i-1} + B_i x_i + C_i x_{i+1} = F_i for the
// conserved interface values x.  Rows 0 and N are the WENO5 rows (B = L,
// A = C = 0) as in the component scheme.
//
// Two kernels per direction:
//   k_crwchar_rows   one thread per interface: average, eigenvectors, the
//                    projected six-cell stencils of u and f, the weights of
//                    both biases, the four systems' (uL, uR, fL, fR) block rows
//                    into a scratch array, line index fastest;
//   k_crwchar_solve  one thread per (line, system): the block elimination of
//                    blocktridiagLU (pivot-free block inverses, the reference's
//                    elimination and back-substitution order), writing the
//                    solution in the standard interface layout that the
//                    upwind kernels read.
// These lines are few and short next to the component CRWENO5 workload (the
// option is off the benchmark configurations); the solve is sequential along
// a line, parallel over lines and systems.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "physics.cuh"

namespace piafs {

namespace {

// Inverse of an NV x NV block by Gaussian elimination without pivoting, the
// steps of _MatrixInvert_ (matops.h:91-125): forward sweep on a copy that also
// builds the inverse of the unit lower factor, then the backward sweep with
// the upper factor; a zero pivot raises *err (the reference prints an error
// and carries on with the non-finite result).
template <int NV>
__device__ __forceinline__ void block_inverse(const double (&A)[NV][NV], double (&Bi)[NV][NV], int* err) {
  double Ac[NV][NV];
#pragma unroll
  for (int r = 0; r < NV; r++)
#pragma unroll
    for (int c = 0; c < NV; c++) { Ac[r][c] = A[r][c]; Bi[r][c] = r == c ? 1.0 : 0.0; }
#pragma unroll
  for (int i = 0; i < NV - 1; i++) {
    if (Ac[i][i] == 0.0) *err = 1;
#pragma unroll
    for (int j = i + 1; j < NV; j++) {
      const double f = Ac[j][i] / Ac[i][i];
#pragma unroll
      for (int k = i + 1; k < NV; k++) Ac[j][k] -= f * Ac[i][k];
#pragma unroll
      for (int k = 0; k < j; k++) Bi[j][k] -= f * Bi[i][k];
    }
  }
  if (Ac[NV - 1][NV - 1] == 0.0) *err = 1;
#pragma unroll
  for (int i = NV - 1; i >= 0; i--) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double s = 0.0;
#pragma unroll
      for (int j = i + 1; j < NV; j++) s += Ac[i][j] * Bi[j][k];
      Bi[i][k] = (Bi[i][k] - s) / Ac[i][i];
    }
  }
}

// elements per system and interface in the row scratch: A, B, C, F
template <int NV> __host__ __device__ constexpr int row_elems() { return 3 * NV * NV + NV; }

template <int MODEL, int DIR>
__global__ void k_crwchar_rows(DevParams P, const double* __restrict__ U, const double* __restrict__ F,
                               double* __restrict__ S, int nl, int N) {
  constexpr int NV = Flow<MODEL>::NF;
  constexpr int K = row_elems<NV>();
  const long long nrows = (long long)nl * (N + 1);
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  const int l = (int)(q % nl), i = (int)(q / nl);
  const long long st = DIR == 0 ? 1 : P.W0;
  const long long c0 = DIR == 0 ? pidx(P, i, l) : pidx(P, l, i);   // cell i, right of the interface
  const long long ps = P.ps;
  double cl[4], cr[4], ua[4], L[4][4], R[4][4];
#pragma unroll
  for (int m = 0; m < NV; m++) { cl[m] = U[m * ps + c0 - st]; cr[m] = U[m * ps + c0]; }
  Flow<MODEL>::roe_avg(cl, cr, P.gamma, ua);
  Flow<MODEL>::eigvec(ua, P.gamma, DIR, L, R);
  const bool bnd = (i == 0 || i == N);
  // optimal weights (WENOFifthOrderCalculateWeights.c:861-878)
  const double c1 = bnd ? 0.1 : 0.2, c2 = bnd ? 0.6 : 0.5, c3 = 0.3;
  const double one_third = 1.0 / 3.0, one_sixth = 1.0 / 6.0;
#pragma unroll
  for (int fld = 0; fld < 2; fld++) {
    const double* src = fld ? F : U;
    double w[NV][6];   // projected values, cells i-3 .. i+2
#pragma unroll
    for (int r = 0; r < 6; r++) {
      double cv[NV];
#pragma unroll
      for (int m = 0; m < NV; m++) cv[m] = src[m * ps + c0 + (r - 3) * st];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < NV; k++) acc += L[v][k] * cv[k];
        w[v][r] = acc;
      }
    }
#pragma unroll
    for (int bias = 0; bias < 2; bias++) {        // 0: upw > 0, 1: upw < 0
      const int sys = 2 * fld + bias;             // uL, uR, fL, fR
      double* o = S + (long long)sys * K * nrows + q;
#pragma unroll
      for (int v = 0; v < NV; v++) {
        // stencil of the bias (Interp1PrimFifthOrderCRWENOChar.c:157-171)
        const double m3 = bias ? w[v][5] : w[v][0], m2 = bias ? w[v][4] : w[v][1];
        const double m1 = bias ? w[v][3] : w[v][2], p1 = bias ? w[v][2] : w[v][3];
        const double p2 = bias ? w[v][1] : w[v][4];
        double w1, w2, w3;
        if (P.no_limiting) { w1 = c1; w2 = c2; w3 = c3; }
        else weno_weights(P.weno_type, c1, c2, c3, m3, m2, m1, p1, p2, P.eps, w1, w2, w3);
        double f1, f2, f3, a, b, c;
        if (bnd) {     // WENO5 row (:190-201)
          f1 = (2 * one_sixth) * m3 - (7.0 * one_sixth) * m2 + (11.0 * one_sixth) * m1;
          f2 = (-one_sixth) * m2 + (5.0 * one_sixth) * m1 + (2 * one_sixth) * p1;
          f3 = (2 * one_sixth) * m1 + (5 * one_sixth) * p1 - (one_sixth) * p2;
          a = 0.0; b = 1.0; c = 0.0;
        } else {       // compact row (:202-206, :218-236)
          f1 = (one_sixth) * (m2 + 5 * m1);
          f2 = (one_sixth) * (5 * m1 + p1);
          f3 = (one_sixth) * (m1 + 5 * p1);
          const double lo = (2 * one_third) * w1 + (one_third) * w2, hi = (one_third) * w3;
          b = (one_third) * w1 + (2 * one_third) * (w2 + w3);
          a = bias ? hi : lo;
          c = bias ? lo : hi;
        }
#pragma unroll
        for (int k = 0; k < NV; k++) {
          o[(long long)(v * NV + k) * nrows] = bnd ? 0.0 : a * L[v][k];
          o[(long long)(NV * NV + v * NV + k) * nrows] = bnd ? L[v][k] : b * L[v][k];
          o[(long long)(2 * NV * NV + v * NV + k) * nrows] = bnd ? 0.0 : c * L[v][k];
        }
        o[(long long)(3 * NV * NV + v) * nrows] = w1 * f1 + w2 * f2 + w3 * f3;
      }
    }
  }
}

template <int NV>
__device__ __forceinline__ void load_block(const double* p, long long stride, double (&M)[NV][NV]) {
#pragma unroll
  for (int r = 0; r < NV; r++)
#pragma unroll
    for (int c = 0; c < NV; c++) M[r][c] = p[(long long)(r * NV + c) * stride];
}
template <int NV>
__device__ __forceinline__ void store_block(double* p, long long stride, const double (&M)[NV][NV]) {
#pragma unroll
  for (int r = 0; r < NV; r++)
#pragma unroll
    for (int c = 0; c < NV; c++) p[(long long)(r * NV + c) * stride] = M[r][c];
}

// blocktridiagLU (blocktridiagLU.c:146-163 elimination, :282-300
// back-substitution; one rank).  In the elimination the sub-diagonal blocks
// stay zero (row 0 has none), so their updates and the x_0 terms of the
// back-substitution are zero and are left out.  The inverse of each
// eliminated diagonal block is kept in place of the block (the reference
// inverts it again for the back-substitution; the result is the same).
template <int NV>
__global__ void k_crwchar_solve(DevParams P, double* __restrict__ S, int nl, int N, int dir, double* __restrict__ o0,
                                double* __restrict__ o1, double* __restrict__ o2, double* __restrict__ o3,
                                int* __restrict__ err) {
  constexpr int K = row_elems<NV>();
  const long long nrows = (long long)nl * (N + 1);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * nl) return;
  const int l = t % nl, sys = t / nl;
  double* base = S + (long long)sys * K * nrows + l;
  double* out = sys == 0 ? o0 : sys == 1 ? o1 : sys == 2 ? o2 : o3;
  auto A_at = [&](int i) { return base + (long long)i * nl; };
  auto B_at = [&](int i) { return base + (long long)i * nl + (long long)(NV * NV) * nrows; };
  auto C_at = [&](int i) { return base + (long long)i * nl + (long long)(2 * NV * NV) * nrows; };
  auto F_at = [&](int i) { return base + (long long)i * nl + (long long)(3 * NV * NV) * nrows; };
  int bad = 0;
  double Bi[NV][NV], Cp[NV][NV], xp[NV];
  {
    double B0[NV][NV];
    load_block<NV>(B_at(0), nrows, B0);
    block_inverse<NV>(B0, Bi, &bad);
    store_block<NV>(B_at(0), nrows, Bi);
    load_block<NV>(C_at(0), nrows, Cp);
#pragma unroll
    for (int v = 0; v < NV; v++) xp[v] = F_at(0)[(long long)v * nrows];
  }
  for (int i = 1; i <= N; i++) {
    double A[NV][NV], B[NV][NV], fac[NV][NV], x[NV];
    load_block<NV>(A_at(i), nrows, A);
    load_block<NV>(B_at(i), nrows, B);
#pragma unroll
    for (int v = 0; v < NV; v++) x[v] = F_at(i)[(long long)v * nrows];
    // factor = A_i inv(B_{i-1}); B_i -= factor C_{i-1}; x_i -= factor x_{i-1}
#pragma unroll
    for (int r = 0; r < NV; r++)
#pragma unroll
      for (int c = 0; c < NV; c++) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NV; k++) s += A[r][k] * Bi[k][c];
        fac[r][c] = s;
      }
#pragma unroll
    for (int r = 0; r < NV; r++)
#pragma unroll
      for (int c = 0; c < NV; c++)
#pragma unroll
        for (int k = 0; k < NV; k++) B[r][c] -= fac[r][k] * Cp[k][c];
#pragma unroll
    for (int r = 0; r < NV; r++)
#pragma unroll
      for (int k = 0; k < NV; k++) x[r] -= fac[r][k] * xp[k];
    block_inverse<NV>(B, Bi, &bad);
    store_block<NV>(B_at(i), nrows, Bi);
#pragma unroll
    for (int v = 0; v < NV; v++) F_at(i)[(long long)v * nrows] = x[v];
    load_block<NV>(C_at(i), nrows, Cp);
#pragma unroll
    for (int v = 0; v < NV; v++) xp[v] = x[v];
  }
  // back-substitution: x_N = inv(B_N) x_N; x_i = inv(B_i) (x_i - C_i x_{i+1})
  auto put = [&](int i, const double* x) {
    const long long qs = dir == 0 ? (long long)i + (long long)(P.N0 + 1) * l : (long long)l + (long long)P.N0 * i;
#pragma unroll
    for (int v = 0; v < NV; v++) out[(long long)v * P.pis + qs] = x[v];
  };
  double xn[NV];
#pragma unroll
  for (int r = 0; r < NV; r++) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < NV; k++) s += Bi[r][k] * xp[k];
    xn[r] = s;
  }
  put(N, xn);
  for (int i = N - 1; i >= 0; i--) {
    double C[NV][NV], Binv[NV][NV], x[NV], xt[NV];
    load_block<NV>(C_at(i), nrows, C);
    load_block<NV>(B_at(i), nrows, Binv);
#pragma unroll
    for (int v = 0; v < NV; v++) x[v] = F_at(i)[(long long)v * nrows];
#pragma unroll
    for (int r = 0; r < NV; r++)
#pragma unroll
      for (int k = 0; k < NV; k++) x[r] -= C[r][k] * xn[k];
#pragma unroll
    for (int r = 0; r < NV; r++) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NV; k++) s += Binv[r][k] * x[k];
      xt[r] = s;
    }
#pragma unroll
    for (int v = 0; v < NV; v++) xn[v] = xt[v];
    put(i, xn);
  }
  if (bad) *err = 1;
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

template <int MODEL>
void crwchar_dir(const DevParams& P, const double* U, const double* F, double* uL, double* uR, double* fL, double* fR,
                 int dir, double* S, int* err, cudaStream_t s) {
  constexpr int NV = Flow<MODEL>::NF;
  const int N = dir == 0 ? P.N0 : P.N1;
  const int nl = P.ndims == 1 ? 1 : (dir == 0 ? P.N1 : P.N0);
  const long long nrows = (long long)nl * (N + 1);
  if (dir == 0) k_crwchar_rows<MODEL, 0><<<nblk(nrows, 128), 128, 0, s>>>(P, U, F, S, nl, N);
  else k_crwchar_rows<MODEL, 1><<<nblk(nrows, 128), 128, 0, s>>>(P, U, F, S, nl, N);
  k_crwchar_solve<NV><<<nblk(4LL * nl, 64), 64, 0, s>>>(P, S, nl, N, dir, uL, uR, fL, fR, err);
}

}  // namespace

long long crweno_char_scratch(const DevParams& P) {
  const int NV = P.model == NS2D ? 4 : 3;
  const long long nmax = P.nint[0] > P.nint[1] ? P.nint[0] : P.nint[1];
  return 4LL * (3 * NV * NV + NV) * nmax;
}

void launch_crweno_char(const DevParams& P, const double* U, const double* F, double* uL, double* uR, double* fL,
                        double* fR, int dir, double* scratch, int* err, cudaStream_t s) {
  if (P.model == NS2D) crwchar_dir<NS2D>(P, U, F, uL, uR, fL, fR, dir, scratch, err, s);
  else crwchar_dir<EULER1D>(P, U, F, uL, uR, fL, fR, dir, scratch, err, s);
}

}  // namespace piafs
