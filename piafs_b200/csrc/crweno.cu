// CRWENO5 interface reconstruction with its tridiagonal line solves (sm_100a).
//
// Interp1PrimFifthOrderCRWENO (Interp1PrimFifthOrderCRWENO.c:81-240) builds,
// for every grid line and solution component, one tridiagonal system per
// upwind bias and per reconstructed array (u and the flux f), and solves them
// with tridiagLU (tridiagLU.c:86-277).  Here one CTA owns one (line, component,
// array) and solves the left- and the right-biased systems of that array
// together, one thread per M consecutive rows:
//
//   * the M + 5 cells a thread needs are loaded once for both systems; the
//     smoothness indicators of every 3-cell window and the two-cell averages
//     of the compact right-hand side are computed once per window and shared,
//     since the right-biased stencil is the mirror image of the left-biased
//     one (the left system at interface i uses windows centred at i-2, i-1,
//     i; the right one the mirrored windows centred at i+1, i, i-1);
//   * the chunk of M rows is reduced in registers (the first row is the
//     chunk's separator; the others are eliminated down and up, so that each
//     reads x = rho - alpha X_k - gamma X_{k+1} in the separators X);
//   * the separator system, one unknown per thread and per bias, is solved by
//     parallel cyclic reduction on rows scaled to a unit diagonal (three
//     values per row), both biases in the same steps and barriers;
//   * every row is recovered from its two separators and the results are
//     staged in shared memory so that the x-direction stores are coalesced.
//
// The lines of a grid run through k_crw_line and k_crw_seg (crweno_line.cu):
// this kernel serves the lines those do not (fewer than three interfaces).
//
// Rows 0 and N are the WENO5 rows with the WENO5 optimal weights (physical
// boundaries, also on periodic domains, Interp1PrimFifthOrderCRWENO.c:164-175);
// they are computed directly and folded into rows 1 and N-1.  Rows past N-1
// are identity rows.  Divisions are reciprocals by Newton-Raphson refinement
// (rcp_nr), so results agree with the reference to rounding, not bit for bit.
#include <type_traits>

#include "crweno_common.cuh"
#include "kernels.h"

namespace piafs {

namespace {

// padded index into the output staging buffer (conflict-free for the strided
// writes of the recovery and the unit-stride reads of the store)
__device__ __forceinline__ int stg(int i) { return i + (i >> 4); }

}  // namespace

// MX (mixed precision): the cells are taken relative to the line's first
// interior value (FP64 subtraction, then FP32), the weights and the rows are
// built in FP32, the elimination and the separator solve run in FP64, and the
// interface values are stored in FP32 relative to that same reference.  The
// reconstruction reproduces constants, so the shift is exact in exact
// arithmetic; it keeps O(1) backgrounds out of the FP32 rounding, and the
// upwind/divergence kernel that reads these values only differences them
// along the line or adds the reference back.
// CTA sizes: up to 512 threads at 8 rows per thread (128 registers), up to 256
// otherwise
__host__ __device__ constexpr int crweno_max_threads(int M) { return M == 8 ? 512 : 256; }

template <int M, int DIR, int WT, bool MX>
__global__ void __launch_bounds__(crweno_max_threads(M), (M <= 4 ? 2 : 1))
    k_crweno_pair(DevParams P, const double* __restrict__ U, const double* __restrict__ F, void* __restrict__ uL,
                  void* __restrict__ uR, void* __restrict__ fL, void* __restrict__ fR, int* __restrict__ err) {
  static_assert(M >= 2, "a chunk needs a separator and at least one interior row");
  typedef typename std::conditional<MX, float, double>::type R;   // row arithmetic
  typedef typename std::conditional<MX, float, double>::type O;   // interface storage
  extern __shared__ double sm[];
  const int Pt = blockDim.x, k = threadIdx.x;
  double* pc = sm;               // PCR rows, [2 buffers][2 biases][a, c, d][Pt]
  double* tp = sm + 12 * Pt;     // last-row coefficients per chunk, [2][3][Pt]
  double* sy = sm + 18 * Pt;     // separator values, [2][Pt]
  double* so = sm + 20 * Pt;     // output staging, [2][stg(rows of the segment) + 1]
  const int K = k, Ptot = Pt;
  auto sync = [&]() { __syncthreads(); };
  auto at = [&](double* arr, int j) -> double { return arr[j]; };
  const int line = (int)blockIdx.x, v = blockIdx.y;
  const bool isF = blockIdx.z != 0;
  const int N = DIR == 0 ? P.N0 : P.N1;
  const long long st = DIR == 0 ? 1 : P.W0;
  const long long ist = DIR == 0 ? 1 : P.N0;
  const long long base = DIR == 0 ? pidx(P, 0, line) : pidx(P, line, 0);
  const long long ibase = DIR == 0 ? (long long)(P.N0 + 1) * line : line;
  const double* src = (isF ? F : U) + (long long)v * P.ps + base;
  O* oL = (O*)(isF ? fL : uL) + (long long)v * P.pis + ibase;
  O* oR = (O*)(isF ? fR : uR) + (long long)v * P.pis + ibase;
  const int s = 1 + K * M;          // separator row (interface) of this thread
  const int kN = (N - 2) / M;       // separator index owning row N-1
  const R eps = R(4) * (R)P.eps;   // with the smoothness indicators at 4x (below)
  const double ref = MX ? src[0] : 0.0;

  // cells s-3 .. s+M+1
  R c[M + 5];
#pragma unroll
  for (int r = 0; r < M + 5; r++) {
    const int cell = s - 3 + r;
    c[r] = cell <= N + 2 ? (R)(src[cell * st] - ref) : R(0);
  }
  R x0[2] = {R(0), R(0)}, xN[2] = {R(0), R(0)};
  if (MX) {
    if (K == 0) { x0[0] = crw_edge_f(P, src, st, 0, 1, ref); x0[1] = crw_edge_f(P, src, st, 0, -1, ref); }
    if (K == kN) { xN[0] = crw_edge_f(P, src, st, N, 1, ref); xN[1] = crw_edge_f(P, src, st, N, -1, ref); }
  } else {
    if (K == 0) { x0[0] = crw_edge(P, src, st, 0, 1); x0[1] = crw_edge(P, src, st, 0, -1); }
    if (K == kN) { xN[0] = crw_edge(P, src, st, N, 1); xN[1] = crw_edge(P, src, st, N, -1); }
  }

  // smoothness indicators of the windows centred at cells s-2+t (t = 0..M+2),
  // kept at 4x their value with eps at 4x, which scales every weight of a
  // stencil by the same factor: b1: 13/3 d^2 + (a-4b+3c)^2, b2: .. (a-c)^2,
  // b3: .. (3a-4b+c)^2
  R b1[M + 3], b2[M + 3], b3[M + 3];
  if (WT != WT_NOLIM) {
#pragma unroll
    for (int t = 0; t < M + 3; t++) {
      const R a = c[t], b = c[t + 1], cc = c[t + 2];
      const R d = a - R(2) * b + cc;
      const R e1 = a - R(4) * b + R(3) * cc, e2 = a - cc, e3 = R(3) * a - R(4) * b + cc;
      const R dd = R(13.0 / 3.0) * d * d;
      b1[t] = dd + e1 * e1;
      b2[t] = dd + e2 * e2;
      b3[t] = dd + e3 * e3;
    }
  }
  // two-cell averages of the compact right-hand side at 3x (the rows are built
  // at 3x, below), cells (s-3+j, s-2+j): pp = 5/2 left + 1/2 right,
  // qq = 1/2 left + 5/2 right
  constexpr R s6 = R(0.5), s56 = R(2.5);
  R pp[M + 3], qq[M + 3];
#pragma unroll
  for (int j = 1; j < M + 3; j++) {
    pp[j] = s56 * c[j] + s6 * c[j + 1];
    qq[j] = s6 * c[j] + s56 * c[j + 1];
  }

  // ---- rows and the downward elimination, both biases (q = 0 left, 1 right)
  double As[2], Bs[2], Cs[2], Rs[2];
  double al[2][M], cg[2][M], rh[2][M];
  int bad = 0;
#pragma unroll
  for (int r = 0; r < M; r++) {
    const int i = s + r;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      R Ar = R(0), Br = R(1), Cr = R(0), Rr = R(0);
      if (i <= N - 1) {
        R w1, w2, w3, f1, f2, f3, tau = R(0);
        if (q == 0) {
          if (WT == W_BORGES) tau = fabs(b3[r + 2] - b1[r]);
          if (WT == W_YC) { const R t4 = c[r] - R(4) * c[r + 1] + R(6) * c[r + 2] - R(4) * c[r + 3] + c[r + 4]; tau = R(4) * t4 * t4; }
          crw_weights<WT, R>(b1[r], b2[r + 1], b3[r + 2], tau, eps, w1, w2, w3);
          f1 = qq[r + 1]; f2 = pp[r + 2]; f3 = qq[r + 2];
        } else {
          if (WT == W_BORGES) tau = fabs(b1[r + 1] - b3[r + 3]);
          if (WT == W_YC) { const R t4 = c[r + 5] - R(4) * c[r + 4] + R(6) * c[r + 3] - R(4) * c[r + 2] + c[r + 1]; tau = R(4) * t4 * t4; }
          crw_weights<WT, R>(b3[r + 3], b2[r + 2], b1[r + 1], tau, eps, w1, w2, w3);
          f1 = pp[r + 3]; f2 = qq[r + 2]; f3 = pp[r + 2];
        }
        // the compact row at 3x: (2 w1 + w2, w1 + 2 w2 + 2 w3, w3) and 3x the
        // right-hand side (pp, qq above)
        const R lo = R(2) * w1 + w2, hi = w3;
        Br = w1 + R(2) * (w2 + w3);
        Ar = q == 0 ? lo : hi;
        Cr = q == 0 ? hi : lo;
        Rr = w1 * f1 + w2 * f2 + w3 * f3;
        if (i == 1) { Rr -= Ar * x0[q]; Ar = R(0); }
        if (i == N - 1) { Rr -= Cr * xN[q]; Cr = R(0); }
      }
      const double A = Ar, B = Br, C = Cr, Rv = Rr;
      if (r == 0) { As[q] = A; Bs[q] = B; Cs[q] = C; Rs[q] = Rv; continue; }
      // rows scaled to a unit diagonal: x_r + cg_r x_{r+1} = rh_r - al_r X_k
      const double be = r == 1 ? B : B - A * cg[q][r - 1];
      bad |= (be == 0.0);
      const double rb = rcp_nr(be);
      if (r == 1) { al[q][1] = A * rb; rh[q][1] = Rv * rb; }
      else { al[q][r] = -(A * al[q][r - 1]) * rb; rh[q][r] = (Rv - A * rh[q][r - 1]) * rb; }
      cg[q][r] = C * rb;
    }
  }
  // ---- upward elimination: x_{s+r} = rh_r - al_r X_k - cg_r X_{k+1}
#pragma unroll
  for (int q = 0; q < 2; q++) {
#pragma unroll
    for (int r = M - 2; r >= 1; r--) {
      const double g = cg[q][r];
      al[q][r] -= g * al[q][r + 1];
      rh[q][r] -= g * rh[q][r + 1];
      cg[q][r] = -(g * cg[q][r + 1]);
    }
    tp[(q * 3 + 0) * Pt + k] = al[q][M - 1];
    tp[(q * 3 + 1) * Pt + k] = cg[q][M - 1];
    tp[(q * 3 + 2) * Pt + k] = rh[q][M - 1];
  }
  sync();

  // ---- separator equations As x_{s-1} + Bs X_k + Cs x_{s+1} = Rs, with
  //      x_{s-1} from the previous chunk's last row and x_{s+1} from row 1
  double a[2], cq[2], d[2];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    double alp = 0.0, gap = 0.0, rhp = 0.0;
    if (K > 0) {
      alp = at(tp + (q * 3 + 0) * Pt, K - 1); gap = at(tp + (q * 3 + 1) * Pt, K - 1);
      rhp = at(tp + (q * 3 + 2) * Pt, K - 1);
    }
    const double b = Bs[q] - As[q] * gap - Cs[q] * al[q][1];
    bad |= (b == 0.0);
    const double rb = rcp_nr(b);
    a[q] = -(As[q] * alp) * rb;
    cq[q] = -(Cs[q] * cg[q][1]) * rb;
    d[q] = (Rs[q] - As[q] * rhp - Cs[q] * rh[q][1]) * rb;
    pc[(q * 3 + 0) * Pt + k] = a[q];
    pc[(q * 3 + 1) * Pt + k] = cq[q];
    pc[(q * 3 + 2) * Pt + k] = d[q];
  }
  if (bad) atomicOr(err, 1);
  sync();
  // ---- parallel cyclic reduction on unit-diagonal rows a x_{k-dl} + x_k + c x_{k+dl} = d
  int buf = 0;
  for (int dl = 1; dl < Ptot; dl <<= 1) {
    double* cur = pc + buf * 6 * Pt;
    double* nxt = pc + (buf ^ 1) * 6 * Pt;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      double am = 0.0, cm = 0.0, dm = 0.0, ap = 0.0, cp = 0.0, dp = 0.0;
      if (K - dl >= 0) {
        am = at(cur + (q * 3 + 0) * Pt, K - dl); cm = at(cur + (q * 3 + 1) * Pt, K - dl);
        dm = at(cur + (q * 3 + 2) * Pt, K - dl);
      }
      if (K + dl < Ptot) {
        ap = at(cur + (q * 3 + 0) * Pt, K + dl); cp = at(cur + (q * 3 + 1) * Pt, K + dl);
        dp = at(cur + (q * 3 + 2) * Pt, K + dl);
      }
      const double bn = 1.0 - a[q] * cm - cq[q] * ap;
      const double rb = rcp_nr(bn);
      const double an = -(a[q] * am) * rb, cn = -(cq[q] * cp) * rb;
      d[q] = (d[q] - a[q] * dm - cq[q] * dp) * rb;
      a[q] = an; cq[q] = cn;
      nxt[(q * 3 + 0) * Pt + k] = a[q];
      nxt[(q * 3 + 1) * Pt + k] = cq[q];
      nxt[(q * 3 + 2) * Pt + k] = d[q];
    }
    buf ^= 1;
    sync();
  }
  sy[k] = d[0];
  sy[Pt + k] = d[1];
  sync();

  // ---- recover every row
  {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const double Xk = d[q];
      const double Xn = k + 1 < Pt ? sy[q * Pt + k + 1] : 0.0;
      double* o = so + q * (stg(N) + 1);
      if (s <= N - 1) o[stg(s)] = Xk;
#pragma unroll
      for (int r = 1; r < M; r++) {
        const int i = s + r;
        if (i <= N - 1) o[stg(i)] = rh[q][r] - al[q][r] * Xk - cg[q][r] * Xn;
      }
      if (k == 0) o[0] = x0[q];
      if (k == kN) o[stg(N)] = xN[q];
    }
    __syncthreads();
    for (int i = k; i <= N; i += Pt) {
      oL[i * ist] = (O)so[stg(i)];
      oR[i * ist] = (O)so[stg(N) + 1 + stg(i)];
    }
  }
}

// rows per thread: the smallest M that keeps a line within one CTA (256
// threads, 512 at M = 8: lines of up to 4097 interfaces).  M = 8 with up to
// 512 threads rather than M = 16 with 256: the 16-row chunks need about twice
// the registers and would leave half the warps per SM.
int crweno_rows_per_thread(int N) {
  const int rows = N - 1;
  const int cand[4] = {2, 4, 8, 16};
  for (int c = 0; c < 4; c++)
    if ((rows + cand[c] - 1) / cand[c] <= crweno_max_threads(cand[c])) return cand[c];
  return -1;
}

// CTAs per line: 1 while one CTA serves the line, else the cluster size at
// M = 8 and 512 threads per CTA (at most 8, the portable cluster size: lines
// of up to 32769 interfaces); -1 beyond
int crweno_cluster_size(int N) {
  if (crweno_rows_per_thread(N) > 0) return 1;
  constexpr int per_cta = 8 * crweno_max_threads(8);
  const int n = (N - 1 + per_cta - 1) / per_cta;
  return n <= 8 ? n : -1;
}

namespace {

template <int M, int DIR, int WT, bool MX>
void crweno_launch(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                   int* err, cudaStream_t s) {
  const int N = DIR == 0 ? P.N0 : P.N1;
  const int nlines = DIR == 0 ? P.N1 : P.N0;
  int Pt = (N - 1 + M - 1) / M;
  Pt = ((Pt + 31) / 32) * 32;
  const size_t smem = (size_t)(20 * Pt + 2 * (N + (N >> 4) + 1)) * sizeof(double);
  // the largest line this M serves: T M + 1 interfaces with T threads
  constexpr int T = crweno_max_threads(M);
  raise_smem_limit<k_crweno_pair<M, DIR, WT, MX>>((20 * T + 2 * (T * M + 2 + ((T * M + 2) >> 4) + 1)) *
                                              (int)sizeof(double));
  dim3 grid(nlines, P.nvars, 2);
  k_crweno_pair<M, DIR, WT, MX><<<grid, Pt, smem, s>>>(P, U, F, uL, uR, fL, fR, err);
}

template <int M, int DIR, bool MX>
void crweno_launch_wt(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                      int* err, cudaStream_t s) {
  if (P.no_limiting) return crweno_launch<M, DIR, WT_NOLIM, MX>(P, U, F, uL, uR, fL, fR, err, s);
  switch (P.weno_type) {
    case W_MAPPED: return crweno_launch<M, DIR, W_MAPPED, MX>(P, U, F, uL, uR, fL, fR, err, s);
    case W_BORGES: return crweno_launch<M, DIR, W_BORGES, MX>(P, U, F, uL, uR, fL, fR, err, s);
    case W_YC: return crweno_launch<M, DIR, W_YC, MX>(P, U, F, uL, uR, fL, fR, err, s);
    default: return crweno_launch<M, DIR, W_JS, MX>(P, U, F, uL, uR, fL, fR, err, s);
  }
}

// the mixed-precision path runs x-direction lines only (its y pass always
// works on the transposed copy)
template <int M>
void crweno_launch_m(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                     int dir, int* err, cudaStream_t s) {
  if (P.mixed) crweno_launch_wt<M, 0, true>(P, U, F, uL, uR, fL, fR, err, s);
  else if (dir == 0) crweno_launch_wt<M, 0, false>(P, U, F, uL, uR, fL, fR, err, s);
  else crweno_launch_wt<M, 1, false>(P, U, F, uL, uR, fL, fR, err, s);
}

}  // namespace

int launch_crweno(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                  int dir, int* err, cudaStream_t s) {
  const int N = dir == 0 ? P.N0 : P.N1;
  if (P.mixed && dir != 0) return -1;
  if (crweno_line_fits(N)) return launch_crweno_line(P, U, F, uL, uR, fL, fR, dir, err, s);
  if (crweno_cluster_size(N) > 1) return launch_crweno_seg(P, U, F, uL, uR, fL, fR, dir, err, s);
  switch (crweno_rows_per_thread(N)) {
    case 2: crweno_launch_m<2>(P, U, F, uL, uR, fL, fR, dir, err, s); break;
    case 4: crweno_launch_m<4>(P, U, F, uL, uR, fL, fR, dir, err, s); break;
    case 8: crweno_launch_m<8>(P, U, F, uL, uR, fL, fR, dir, err, s); break;
    case 16: crweno_launch_m<16>(P, U, F, uL, uR, fL, fR, dir, err, s); break;
    default: return -1;
  }
  return 0;
}

}  // namespace piafs
