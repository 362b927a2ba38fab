// The CRWENO5 line solve of one (line, component, field) as a device
// function of a whole CTA (crweno_line.cu); the method is
// described in crweno_line.cu.
#pragma once
#include <type_traits>

#include "crweno_common.cuh"

namespace piafs {

// staged cell slot: one pad slot per 8 cells
__host__ __device__ __forceinline__ int cpad(int j) { return j + (j >> 3); }
// staged output slot: one pad slot per 16 rows
__host__ __device__ __forceinline__ int opad(int i) { return i + (i >> 4); }

__host__ __device__ constexpr int line_threads_max() { return 512; }

// threads of a line of N interfaces at M rows per thread (a multiple of 32)
template <int M>
__host__ __device__ constexpr int line_threads_m(int N) {
  return ((N - 1 + M - 1) / M + 31) / 32 * 32;
}

// Rows s .. s+M-1 of both biases from the staged cells, reduced to the
// chunk's separator: on return x_{s+r} = rh[q][r] - al[q][r] X_s -
// cg[q][r] X_{s+M} for r = 1 .. M-1, and (As, Bs, Cs, Rs) is the separator
// row s.  FULL: every row lies in [2, N-2] (no boundary folding, no identity
// rows).  R: the arithmetic of the nonlinear weights (double, or float in
// mixed precision); the rows' right-hand sides, the rows themselves and their
// elimination are FP64 in both, and in mixed precision each weight product
// is converted once and serves both biases' rows.
template <int M, int WT, bool FULL, typename R>
__device__ __forceinline__ void crw_chunk(const double* __restrict__ cs, int k, int s, int N, const double* x0,
                                          const double* xN, R eps, double (&As)[2], double (&Bs)[2],
                                          double (&Cs)[2], double (&Rs)[2], double (&al)[2][M],
                                          double (&cg)[2][M], double (&rh)[2][M], int& bad) {
  // cells s-3 .. s+M+1 (staged index = cell + 3), and the same in the
  // weights' arithmetic
  double c[M + 5];
  R cw[M + 5];
#pragma unroll
  for (int r = 0; r < M + 5; r++) { c[r] = cs[cpad(k * M + 1 + r)]; cw[r] = (R)c[r]; }
  // Per window t (cells s-3+t .. s-1+t): the smoothness indicators at 4x
  // (b1: 13/3 d^2 + (a-4b+3c)^2, b2: .. (a-c)^2, b3: .. (3a-4b+c)^2) and,
  // for Jiang-Shu, q = (beta + eps)^2.  Two-cell averages of the compact
  // right-hand side at 3x for cells (s-3+j, s-2+j): pp = 5/2 left + 1/2
  // right, qq = 1/2 left + 5/2 right.  Everything is produced in the row
  // loop as the rows need it (row r reads windows up to r+3), which keeps
  // the live range of each value short.
  R b1[M + 3], b2[M + 3], b3[M + 3], q1[M + 3], q2[M + 3], q3[M + 3];
  double pp[M + 3], qq[M + 3];
  auto window = [&](int t) {
    if (WT != WT_NOLIM) {
      const R a = cw[t], b = cw[t + 1], cc = cw[t + 2];
      const R d = (a + cc) - R(2) * b;
      const R e1 = a - R(4) * b + R(3) * cc, e2 = a - cc, e3 = R(3) * a - R(4) * b + cc;
      const R dd = R(13.0 / 3.0) * d * d;
      b1[t] = dd + e1 * e1;
      b2[t] = dd + e2 * e2;
      b3[t] = dd + e3 * e3;
      if (WT == W_JS) {
        const R s1 = b1[t] + eps, s2 = b2[t] + eps, s3 = b3[t] + eps;
        q1[t] = s1 * s1; q2[t] = s2 * s2; q3[t] = s3 * s3;
      }
    }
    if (t >= 1) {
      pp[t] = 2.5 * c[t] + 0.5 * c[t + 1];
      qq[t] = 0.5 * c[t] + 2.5 * c[t + 1];
    }
  };
  // Jiang-Shu products of left-row index j: P23 = q2[j+1] q3[j+2],
  // P13 = q1[j] q3[j+2] (kept at 5x), P12 = q1[j] q2[j+1]; the left row j
  // has the weights (0.2 P23, 0.5 P13, 0.3 P12), the right row j-1 (0.2 P12,
  // 0.5 P13, 0.3 P23)
  double P23[M + 1], P13x5[M + 1], P12[M + 1];
  auto products = [&](int j) {
    P23[j] = (double)(q2[j + 1] * q3[j + 2]);
    P13x5[j] = (double)((R(5) * q1[j]) * q3[j + 2]);
    P12[j] = (double)(q1[j] * q2[j + 1]);
  };
  window(0); window(1); window(2);
  if (WT == W_JS) products(0);

#pragma unroll
  for (int r = 0; r < M; r++) {
    const int i = s + r;
    window(r + 3);
    if (WT == W_JS) products(r + 1);
#pragma unroll
    for (int q = 0; q < 2; q++) {
      double Ar, Br, Cr, Rr;
      if (WT == W_JS) {
        // rows at 30x: weights (W1, W2, W3) = 10 (w1, w2, w3), the 3x rows
        // and right-hand side of the general branch times 10
        const double W1 = q == 0 ? 2.0 * P23[r] : 2.0 * P12[r + 1];
        const double W2 = q == 0 ? P13x5[r] : P13x5[r + 1];
        const double W3 = q == 0 ? 3.0 * P12[r] : 3.0 * P23[r + 1];
        const double lo = 2.0 * W1 + W2;
        Br = W1 + 2.0 * (W2 + W3);
        Ar = q == 0 ? lo : W3;
        Cr = q == 0 ? W3 : lo;
        Rr = q == 0 ? W1 * qq[r + 1] + W2 * pp[r + 2] + W3 * qq[r + 2]
                    : W1 * pp[r + 3] + W2 * qq[r + 2] + W3 * pp[r + 2];
      } else {
        R v1, v2, v3, tau = R(0);
        if (q == 0) {
          if (WT == W_BORGES) tau = fabs(b3[r + 2] - b1[r]);
          if (WT == W_YC) { const R t4 = cw[r] - R(4) * cw[r + 1] + R(6) * cw[r + 2] - R(4) * cw[r + 3] + cw[r + 4]; tau = R(4) * t4 * t4; }
          crw_weights<WT, R>(b1[r], b2[r + 1], b3[r + 2], tau, eps, v1, v2, v3);
        } else {
          if (WT == W_BORGES) tau = fabs(b1[r + 1] - b3[r + 3]);
          if (WT == W_YC) { const R t4 = cw[r + 5] - R(4) * cw[r + 4] + R(6) * cw[r + 3] - R(4) * cw[r + 2] + cw[r + 1]; tau = R(4) * t4 * t4; }
          crw_weights<WT, R>(b3[r + 3], b2[r + 2], b1[r + 1], tau, eps, v1, v2, v3);
        }
        const double w1 = v1, w2 = v2, w3 = v3;
        // rows at 3x: (2 w1 + w2, w1 + 2 w2 + 2 w3, w3) and 3x the
        // right-hand side (pp, qq above)
        const double lo = 2.0 * w1 + w2, hi = w3;
        Br = w1 + 2.0 * (w2 + w3);
        Ar = q == 0 ? lo : hi;
        Cr = q == 0 ? hi : lo;
        Rr = q == 0 ? w1 * qq[r + 1] + w2 * pp[r + 2] + w3 * qq[r + 2]
                    : w1 * pp[r + 3] + w2 * qq[r + 2] + w3 * pp[r + 2];
      }
      if (!FULL) {
        if (i > N - 1) { Ar = 0.0; Br = 1.0; Cr = 0.0; Rr = 0.0; }
        if (i == 1) { Rr -= Ar * x0[q]; Ar = 0.0; }
        if (i == N - 1) { Rr -= Cr * xN[q]; Cr = 0.0; }
      }
      const double A = Ar, B = Br, C = Cr, Rv = Rr;
      if (r == 0) { As[q] = A; Bs[q] = B; Cs[q] = C; Rs[q] = Rv; continue; }
      // rows scaled to a unit diagonal: x_r + cg_r x_{r+1} = rh_r - al_r X_s
      const double be = r == 1 ? B : B - A * cg[q][r - 1];
      bad |= (be == 0.0);
      const double rb = rcp_nr(be);
      if (r == 1) { al[q][1] = A * rb; rh[q][1] = Rv * rb; }
      else { al[q][r] = -(A * al[q][r - 1]) * rb; rh[q][r] = (Rv - A * rh[q][r - 1]) * rb; }
      cg[q][r] = C * rb;
    }
  }
  // upward elimination: x_{s+r} = rh_r - al_r X_s - cg_r X_{s+M}
#pragma unroll
  for (int q = 0; q < 2; q++) {
#pragma unroll
    for (int r = M - 2; r >= 1; r--) {
      const double g = cg[q][r];
      al[q][r] -= g * al[q][r + 1];
      rh[q][r] -= g * rh[q][r + 1];
      cg[q][r] = -(g * cg[q][r + 1]);
    }
  }
}

// One (line, component, field) of the CRWENO5 reconstruction: both biases'
// tridiagonal systems built from the cells src[-3 .. N+2] (stride st, taken
// relative to `ref`), solved, and their N + 1 interface values staged in
// shared memory: so[q * ostride + opad(i)] for bias q (0 left, 1 right) and
// interface i.  Called by every thread of the CTA (Pt = blockDim.x threads,
// M rows each); returns after a barrier, with the staged values visible to
// the whole CTA.  Shared memory: pcA [2][3][Pt], tp [3][Pt], sy [Pt]
// (double2), the cells cs (cpad layout, Pt M + 6 doubles) and the staging
// so, which may alias cs.  Sets bad on a zero pivot.
template <int M, int WT, typename R, typename O>
__device__ __forceinline__ void line_pair_solve(const DevParams& P, const double* __restrict__ src, long long st,
                                                double ref, int N, double* cs, double2* pcA, double2* tp,
                                                double2* sy, O* so, int& bad) {
  constexpr bool MX = std::is_same<R, float>::value;
  const int Pt = blockDim.x, k = threadIdx.x, lane = k & 31;
  const int s = 1 + k * M;          // separator row (interface) of this thread
  const int kN = (N - 2) / M;       // thread owning row N-1
  const R eps = R(4) * (R)P.eps;    // with the smoothness indicators at 4x
  // cells -3 .. N+2 of the line (coalesced for x lines), zero past the last
  // cell any thread reads: all of a thread's loads are issued before the
  // first store (at most M + 1 of them: Pt M + 6 cells over Pt threads)
  {
    const int ncell = Pt * M + 6;
    double cv[M + 1];
#pragma unroll
    for (int it = 0; it <= M; it++) {
      const int j = k + it * Pt;
      cv[it] = j < N + 6 ? src[(j - 3) * st] - ref : 0.0;
    }
#pragma unroll
    for (int it = 0; it <= M; it++) {
      const int j = k + it * Pt;
      if (j < ncell) cs[cpad(j)] = cv[it];
    }
  }
  double x0[2] = {0.0, 0.0}, xN[2] = {0.0, 0.0};
  if (MX) {
    if (k == 0) { x0[0] = crw_edge_f(P, src, st, 0, 1, ref); x0[1] = crw_edge_f(P, src, st, 0, -1, ref); }
    if (k == kN) { xN[0] = crw_edge_f(P, src, st, N, 1, ref); xN[1] = crw_edge_f(P, src, st, N, -1, ref); }
  } else {
    if (k == 0) { x0[0] = crw_edge(P, src, st, 0, 1); x0[1] = crw_edge(P, src, st, 0, -1); }
    if (k == kN) { xN[0] = crw_edge(P, src, st, N, 1); xN[1] = crw_edge(P, src, st, N, -1); }
  }
  __syncthreads();

  double As[2], Bs[2], Cs[2], Rs[2];
  double al[2][M], cg[2][M], rh[2][M];
  // warp-uniform: every chunk of this warp inside rows [2, N-2]
  const int w0 = k - lane;
  if (w0 >= 1 && (w0 + 32) * M <= N - 2)
    crw_chunk<M, WT, true, R>(cs, k, s, N, x0, xN, eps, As, Bs, Cs, Rs, al, cg, rh, bad);
  else
    crw_chunk<M, WT, false, R>(cs, k, s, N, x0, xN, eps, As, Bs, Cs, Rs, al, cg, rh, bad);
  tp[k] = make_double2(al[0][M - 1], al[1][M - 1]);
  tp[Pt + k] = make_double2(cg[0][M - 1], cg[1][M - 1]);
  tp[2 * Pt + k] = make_double2(rh[0][M - 1], rh[1][M - 1]);
  __syncthreads();

  // separator equations As x_{s-1} + Bs X_k + Cs x_{s+1} = Rs, with x_{s-1}
  // from the previous chunk's last row and x_{s+1} from row 1, scaled to a
  // unit diagonal: a X_{k-1} + X_k + c X_{k+1} = d
  double a[2], cq[2], d[2];
  {
    double2 alp = make_double2(0.0, 0.0), gap = alp, rhp = alp;
    if (k > 0) { alp = tp[k - 1]; gap = tp[Pt + k - 1]; rhp = tp[2 * Pt + k - 1]; }
    const double alq[2] = {alp.x, alp.y}, gaq[2] = {gap.x, gap.y}, rhq[2] = {rhp.x, rhp.y};
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const double b = Bs[q] - As[q] * gaq[q] - Cs[q] * al[q][1];
      bad |= (b == 0.0);
      const double rb = rcp_nr(b);
      a[q] = -(As[q] * alq[q]) * rb;
      cq[q] = -(Cs[q] * cg[q][1]) * rb;
      d[q] = (Rs[q] - As[q] * rhq[q] - Cs[q] * rh[q][1]) * rb;
    }
  }
  pcA[k] = make_double2(a[0], a[1]);
  pcA[Pt + k] = make_double2(cq[0], cq[1]);
  pcA[2 * Pt + k] = make_double2(d[0], d[1]);
  __syncthreads();

  // parallel cyclic reduction on the unit-diagonal separator rows.  Row k
  // has a = 0 when k < dl (no row k - dl) and c = 0 when k + dl >= Pt: the
  // first separator row has no left coupling, the last no right coupling
  // (its rows lie past N-1), and each step keeps these zeros exactly
  // (0 x finite = 0).  So the neighbour index is clamped into the line and
  // the clamped row's finite values are multiplied by those zeros: no
  // predicated loads, no zero fill.
  int buf = 0;
  for (int dl = 1; dl < Pt; dl <<= 1) {
    const double2* cur = pcA + buf * 3 * Pt;
    double2* nxt = pcA + (buf ^ 1) * 3 * Pt;
    const int km = k >= dl ? k - dl : k, kp = k + dl < Pt ? k + dl : k;
    const double2 am = cur[km], cm = cur[Pt + km], dm = cur[2 * Pt + km];
    const double2 ap = cur[kp], cp = cur[Pt + kp], dp = cur[2 * Pt + kp];
    const double amq[2] = {am.x, am.y}, cmq[2] = {cm.x, cm.y}, dmq[2] = {dm.x, dm.y};
    const double apq[2] = {ap.x, ap.y}, cpq[2] = {cp.x, cp.y}, dpq[2] = {dp.x, dp.y};
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const double bn = 1.0 - a[q] * cmq[q] - cq[q] * apq[q];
      const double rb = rcp_nr(bn);
      const double an = -(a[q] * amq[q]) * rb, cn = -(cq[q] * cpq[q]) * rb;
      d[q] = (d[q] - a[q] * dmq[q] - cq[q] * dpq[q]) * rb;
      a[q] = an; cq[q] = cn;
    }
    nxt[k] = make_double2(a[0], a[1]);
    nxt[Pt + k] = make_double2(cq[0], cq[1]);
    nxt[2 * Pt + k] = make_double2(d[0], d[1]);
    buf ^= 1;
    __syncthreads();
  }
  sy[k] = make_double2(d[0], d[1]);
  __syncthreads();

  // recover every row into the output staging (the cells are dead by now);
  // the last row's coefficients come back from tp, which frees their
  // registers across the reduction
  const double2 xn = k + 1 < Pt ? sy[k + 1] : make_double2(0.0, 0.0);
  {
    const double2 l0 = tp[k], l1 = tp[Pt + k], l2 = tp[2 * Pt + k];
    al[0][M - 1] = l0.x; al[1][M - 1] = l0.y;
    cg[0][M - 1] = l1.x; cg[1][M - 1] = l1.y;
    rh[0][M - 1] = l2.x; rh[1][M - 1] = l2.y;
  }
  const int ostride = opad(N) + 1;
  const bool whole = s + M - 1 <= N - 1;   // every row of the chunk lies in the line
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const double Xk = d[q], Xn = q == 0 ? xn.x : xn.y;
    O* o = so + q * ostride;
    if (whole) {
      o[opad(s)] = (O)Xk;
#pragma unroll
      for (int r = 1; r < M; r++) o[opad(s + r)] = (O)(rh[q][r] - al[q][r] * Xk - cg[q][r] * Xn);
    } else {
      if (s <= N - 1) o[opad(s)] = (O)Xk;
#pragma unroll
      for (int r = 1; r < M; r++) {
        const int i = s + r;
        if (i <= N - 1) o[opad(i)] = (O)(rh[q][r] - al[q][r] * Xk - cg[q][r] * Xn);
      }
    }
    if (k == 0) o[0] = (O)x0[q];
    if (k == kN) o[opad(N)] = (O)xN[q];
  }
  __syncthreads();
}

}  // namespace piafs
