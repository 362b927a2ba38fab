// CRWENO5 interface reconstruction, one CTA per line, component and field,
// lines of up to 4097 interfaces (sm_100a): x lines (unit stride, also the y
// lines of a transposed state) and strided y lines; longer lines by clusters
// of CTAs (k_crw_seg, below).
//
// The method is that of k_crweno_pair (crweno.cu, which keeps the general
// form for lines of fewer than three interfaces): Interp1PrimFifthOrderCRWENO
// (Interp1PrimFifthOrderCRWENO.c:81-240) builds one tridiagonal system per
// upwind bias, and the two systems of a (line, component, field) are solved
// together by substructuring -- each thread reduces its chunk of M rows to
// its separator, the separator system is solved by parallel cyclic reduction
// (PCR) in shared memory, and every row is recovered from its two
// separators.  This kernel is the lean form of it for unit-stride lines:
//
//   * the line's cells are loaded once (coalesced on x lines) into shared memory (one
//     pad slot per 8 cells, so that the 13-cell windows that threads read at
//     a stride of 8 cells fall in distinct banks), and past the line's end
//     the staging is zero, so no thread needs a bounds check on its cells;
//   * for the Jiang-Shu weights the rows are built from three products of
//     the squared smoothness terms that the left-biased row at interface j
//     and the right-biased row at interface j-1 share (their unnormalised
//     weights are the same three products with the first and third roles
//     swapped), so a row pair costs three products instead of six;
//   * chunks inside the line (every warp but the first and the last) take a
//     path without any per-row test; only the chunks holding row 1, row N-1
//     or rows past the line run the general rows;
//   * the PCR rows of both biases are packed as double2, one 16-byte access
//     per coefficient and neighbour.
//
// Rows 0 and N are the WENO5 rows with the WENO5 optimal weights (physical
// boundaries, also on periodic domains, Interp1PrimFifthOrderCRWENO.c:164-175),
// computed directly and folded into rows 1 and N-1; rows past N-1 are
// identity rows.  Every row may be scaled by a positive constant without
// changing the solution (the elimination normalises each row), which the Jiang-Shu
// rows use: they are formed at 30x (3x for the compact scheme's thirds, 10x
// for the optimal weights 0.2, 0.5, 0.3) from unnormalised weights, and the
// smoothness indicators at 4x with eps at 4x.  Quotients use rcp_nr.
#include <cooperative_groups.h>
#include <type_traits>

#include "crweno_solve.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace piafs {

namespace {

// DIR 0: x lines (unit stride); DIR 1: y lines (stride W0, interface index
// q = i + N0 j), FP64 only
template <int M, int DIR, int WT, bool MX>
__global__ void __launch_bounds__(line_threads_max(), 1)
    k_crw_line(DevParams P, const double* __restrict__ U, const double* __restrict__ F, void* __restrict__ uL,
               void* __restrict__ uR, void* __restrict__ fL, void* __restrict__ fR, int* __restrict__ err) {
  typedef typename std::conditional<MX, float, double>::type R;   // weights' arithmetic
  typedef typename std::conditional<MX, float, double>::type O;   // interface storage
  extern __shared__ double2 sm2[];
  const int Pt = blockDim.x, k = threadIdx.x;
  double2* pcA = sm2;              // PCR rows (a, c, d), both biases: [2 buffers][3][Pt]
  double2* tp = sm2 + 6 * Pt;      // last-row coefficients (al, cg, rh) of each chunk: [3][Pt]
  double2* sy = sm2 + 9 * Pt;      // separator values [Pt]
  double* cs = (double*)(sm2 + 10 * Pt);   // staged cells; later the output staging
  O* so = (O*)(sm2 + 10 * Pt);

  const int line = blockIdx.x, v = blockIdx.y;
  const bool isF = blockIdx.z != 0;
  const int N = DIR == 0 ? P.N0 : P.N1;
  const long long st = DIR == 0 ? 1 : P.W0;            // cell stride along the line
  const long long ist = DIR == 0 ? 1 : P.N0;           // interface stride along the line
  const long long base = DIR == 0 ? pidx(P, 0, line) : pidx(P, line, 0);
  const double* src = (isF ? F : U) + (long long)v * P.ps + base;
  const long long ibase = DIR == 0 ? (long long)(P.N0 + 1) * line : line;
  O* oL = (O*)(isF ? fL : uL) + (long long)v * P.pis + ibase;
  O* oR = (O*)(isF ? fR : uR) + (long long)v * P.pis + ibase;
  const double ref = MX ? src[0] : 0.0;
  int bad = 0;
  line_pair_solve<M, WT, R, O>(P, src, st, ref, N, cs, pcA, tp, sy, so, bad);
  if (bad) atomicOr(err, 1);
  const int ostride = opad(N) + 1;
  // N + 1 interfaces over Pt threads: at most M + 1 each; the passive
  // variables packed for their upwinding when P.pack_sp (uL - uR, fL + fR)
  if (P.pack_sp && v >= P.nflow) {
#pragma unroll
    for (int it = 0; it <= M; it++) {
      const int i = k + it * Pt;
      if (i <= N) {
        const O l = so[opad(i)], r = so[ostride + opad(i)];
        oL[i * ist] = isF ? l + r : l - r;
      }
    }
    return;
  }
#pragma unroll
  for (int it = 0; it <= M; it++) {
    const int i = k + it * Pt;
    if (i <= N) {
      oL[i * ist] = so[opad(i)];
      oR[i * ist] = so[ostride + opad(i)];
    }
  }
}


// Lines longer than one CTA serves (more than 4097 interfaces): a cluster
// of ncta CTAs per line, CTA r owning the separators [r Pt, (r+1) Pt) and
// their chunks of M rows.  Each CTA builds and reduces its chunks as above,
// then solves its own part of the separator system by PCR with the two
// unknowns outside it -- the previous CTA's last separator L and the next
// CTA's first separator R -- carried as two extra columns (e, f) of every
// row, so that after the local PCR every separator reads
// X_k = d_k - e_k L - f_k R.  The first and last separators of every CTA
// then form a system of 2 ncta unknowns, gathered from the cluster's shared
// memory and solved by one thread of each CTA; L and R give every X_k.  Two
// cluster barriers (the neighbour's last chunk row for the first separator
// equation; the boundary rows) and a third before exit, instead of one per
// PCR level across the cluster.
template <int M, int DIR, int WT, bool MX>
__global__ void __launch_bounds__(line_threads_max(), 1)
    k_crw_seg(DevParams P, const double* __restrict__ U, const double* __restrict__ F, void* __restrict__ uL,
              void* __restrict__ uR, void* __restrict__ fL, void* __restrict__ fR, int* __restrict__ err) {
  typedef typename std::conditional<MX, float, double>::type R;   // weights' arithmetic
  typedef typename std::conditional<MX, float, double>::type O;   // interface storage
  extern __shared__ double2 sm2[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), ncta = (int)cl.num_blocks();
  const int Pt = blockDim.x, k = threadIdx.x, lane = k & 31;
  double2* pcA = sm2;              // PCR rows (a, c, d, e, f), both biases: [2 buffers][5][Pt]
  double2* tp = sm2 + 10 * Pt;     // last-row coefficients (al, cg, rh) of each chunk: [3][Pt]
  double2* sy = sm2 + 13 * Pt;     // separator values [Pt]
  double2* bnd = sm2 + 14 * Pt;    // (d, e, f) of the first and the last separator; L, R
  double* cs = (double*)(sm2 + 14 * Pt + 8);   // staged cells; later the output staging
  O* so = (O*)cs;

  const int line = (int)blockIdx.x / ncta, v = blockIdx.y;
  const bool isF = blockIdx.z != 0;
  const int N = DIR == 0 ? P.N0 : P.N1;
  const long long st = DIR == 0 ? 1 : P.W0;
  const long long ist = DIR == 0 ? 1 : P.N0;
  const long long base = DIR == 0 ? pidx(P, 0, line) : pidx(P, line, 0);
  const double* src = (isF ? F : U) + (long long)v * P.ps + base;
  const long long ibase = DIR == 0 ? (long long)(P.N0 + 1) * line : line;
  O* oL = (O*)(isF ? fL : uL) + (long long)v * P.pis + ibase;
  O* oR = (O*)(isF ? fR : uR) + (long long)v * P.pis + ibase;
  const double ref = MX ? src[0] : 0.0;
  const int K = rank * Pt + k;               // separator of this thread in the line
  const int rb = rank * Pt * M;              // rows before the segment
  const int s = 1 + K * M;
  const int kN = (N - 2) / M;                // separator owning row N-1
  const R eps = R(4) * (R)P.eps;
  int bad = 0;
  // cells rb-3 .. rb+Pt M+2 at staged index j = cell - rb + 3, zero past N+2
  {
    const int ncell = Pt * M + 6;
    double cv[M + 1];
#pragma unroll
    for (int it = 0; it <= M; it++) {
      const int j = k + it * Pt;
      cv[it] = (j < ncell && rb + j < N + 6) ? src[(rb + j - 3) * st] - ref : 0.0;
    }
#pragma unroll
    for (int it = 0; it <= M; it++) {
      const int j = k + it * Pt;
      if (j < ncell) cs[cpad(j)] = cv[it];
    }
  }
  double x0[2] = {0.0, 0.0}, xN[2] = {0.0, 0.0};
  if (MX) {
    if (K == 0) { x0[0] = crw_edge_f(P, src, st, 0, 1, ref); x0[1] = crw_edge_f(P, src, st, 0, -1, ref); }
    if (K == kN) { xN[0] = crw_edge_f(P, src, st, N, 1, ref); xN[1] = crw_edge_f(P, src, st, N, -1, ref); }
  } else {
    if (K == 0) { x0[0] = crw_edge(P, src, st, 0, 1); x0[1] = crw_edge(P, src, st, 0, -1); }
    if (K == kN) { xN[0] = crw_edge(P, src, st, N, 1); xN[1] = crw_edge(P, src, st, N, -1); }
  }
  __syncthreads();

  double As[2], Bs[2], Cs[2], Rs[2];
  double al[2][M], cg_[2][M], rh[2][M];
  const int Kw = K - lane;                   // first separator of this warp
  if (Kw >= 1 && (Kw + 32) * M <= N - 2)
    crw_chunk<M, WT, true, R>(cs, k, s, N, x0, xN, eps, As, Bs, Cs, Rs, al, cg_, rh, bad);
  else
    crw_chunk<M, WT, false, R>(cs, k, s, N, x0, xN, eps, As, Bs, Cs, Rs, al, cg_, rh, bad);
  tp[k] = make_double2(al[0][M - 1], al[1][M - 1]);
  tp[Pt + k] = make_double2(cg_[0][M - 1], cg_[1][M - 1]);
  tp[2 * Pt + k] = make_double2(rh[0][M - 1], rh[1][M - 1]);
  cl.sync();   // the previous CTA's last chunk row is read below

  // separator equations, scaled to a unit diagonal; the first separator of
  // CTA r > 0 couples to the previous CTA's last one (L, column e) and the
  // last of CTA r < ncta-1 to the next CTA's first (R, column f)
  double a[2], cq[2], d[2], e[2], f[2];
  {
    double2 alp = make_double2(0.0, 0.0), gap = alp, rhp = alp;
    if (k > 0) {
      alp = tp[k - 1]; gap = tp[Pt + k - 1]; rhp = tp[2 * Pt + k - 1];
    } else if (rank > 0) {
      const double2* rt = cl.map_shared_rank(tp, rank - 1);
      alp = rt[Pt - 1]; gap = rt[2 * Pt - 1]; rhp = rt[3 * Pt - 1];
    }
    const double alq[2] = {alp.x, alp.y}, gaq[2] = {gap.x, gap.y}, rhq[2] = {rhp.x, rhp.y};
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const double b = Bs[q] - As[q] * gaq[q] - Cs[q] * al[q][1];
      bad |= (b == 0.0);
      const double rbq = rcp_nr(b);
      a[q] = -(As[q] * alq[q]) * rbq;
      cq[q] = -(Cs[q] * cg_[q][1]) * rbq;
      d[q] = (Rs[q] - As[q] * rhq[q] - Cs[q] * rh[q][1]) * rbq;
      e[q] = 0.0;
      f[q] = 0.0;
      if (k == 0) { e[q] = a[q]; a[q] = 0.0; }
      if (k == Pt - 1) { f[q] = cq[q]; cq[q] = 0.0; }
    }
  }
  auto put = [&](double2* row) {
    row[k] = make_double2(a[0], a[1]);
    row[Pt + k] = make_double2(cq[0], cq[1]);
    row[2 * Pt + k] = make_double2(d[0], d[1]);
    row[3 * Pt + k] = make_double2(e[0], e[1]);
    row[4 * Pt + k] = make_double2(f[0], f[1]);
  };
  put(pcA);
  __syncthreads();
  // PCR within the CTA (rows outside it: zero couplings, clamped as in
  // line_pair_solve), the external unknowns' columns updated alongside
  int buf = 0;
  for (int dl = 1; dl < Pt; dl <<= 1) {
    const double2* cur = pcA + buf * 5 * Pt;
    const int km = k >= dl ? k - dl : k, kp = k + dl < Pt ? k + dl : k;
    const double2 am = cur[km], cm = cur[Pt + km], dm = cur[2 * Pt + km], em = cur[3 * Pt + km],
                  fm = cur[4 * Pt + km];
    const double2 ap = cur[kp], cp = cur[Pt + kp], dp = cur[2 * Pt + kp], ep = cur[3 * Pt + kp],
                  fp = cur[4 * Pt + kp];
    const double amq[2] = {am.x, am.y}, cmq[2] = {cm.x, cm.y}, dmq[2] = {dm.x, dm.y}, emq[2] = {em.x, em.y},
                 fmq[2] = {fm.x, fm.y};
    const double apq[2] = {ap.x, ap.y}, cpq[2] = {cp.x, cp.y}, dpq[2] = {dp.x, dp.y}, epq[2] = {ep.x, ep.y},
                 fpq[2] = {fp.x, fp.y};
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const double bn = 1.0 - a[q] * cmq[q] - cq[q] * apq[q];
      const double rbq = rcp_nr(bn);
      const double an = -(a[q] * amq[q]) * rbq, cn = -(cq[q] * cpq[q]) * rbq;
      d[q] = (d[q] - a[q] * dmq[q] - cq[q] * dpq[q]) * rbq;
      e[q] = (e[q] - a[q] * emq[q] - cq[q] * epq[q]) * rbq;
      f[q] = (f[q] - a[q] * fmq[q] - cq[q] * fpq[q]) * rbq;
      a[q] = an; cq[q] = cn;
    }
    put(pcA + (buf ^ 1) * 5 * Pt);
    buf ^= 1;
    __syncthreads();
  }
  // X_k = d_k - e_k L - f_k R; the first and last rows to the cluster
  if (k == 0) { bnd[0] = make_double2(d[0], d[1]); bnd[1] = make_double2(e[0], e[1]); bnd[2] = make_double2(f[0], f[1]); }
  if (k == Pt - 1) { bnd[3] = make_double2(d[0], d[1]); bnd[4] = make_double2(e[0], e[1]); bnd[5] = make_double2(f[0], f[1]); }
  cl.sync();
  // the cluster's boundary rows gathered by 6 ncta threads at once (one
  // round trip of distributed shared memory) into this CTA's cell staging,
  // free between the chunk phase and the recovery
  double2* gath = (double2*)cs;
  if (k < 6 * ncta) gath[k] = cl.map_shared_rank(bnd, k / 6)[k % 6];
  __syncthreads();
  if (k < 2) {
    // bias q = k.  Unknowns F_c (first separator of CTA c) and G_c (last):
    //   F_c = d0_c - e0_c G_{c-1} - f0_c F_{c+1},  G_c = dl_c - el_c G_{c-1} - fl_c F_{c+1}
    // (no G_{-1}, no F_{ncta}).  Forward: G_c = al_c + be_c F_{c+1} and
    // F_c = ga_c + de_c F_{c+1}; backward from F_{ncta} = 0.  This CTA needs
    // L = G_{rank-1} and R = F_{rank+1}.
    constexpr int MAXC = 8;
    const int q = k;
    double al[MAXC], be[MAXC], ga[MAXC], de[MAXC];
    double alp = 0.0, bep = 0.0;
    for (int c = 0; c < ncta; c++) {
      const double* g6 = (const double*)(gath + 6 * c);   // (d0, e0, f0, dl, el, fl), two biases each
      const double d0 = g6[0 + q], e0 = g6[2 + q], f0 = g6[4 + q];
      const double dl = g6[6 + q], el = g6[8 + q], fl = g6[10 + q];
      const double den = 1.0 + e0 * bep;
      bad |= (den == 0.0);
      const double rd = rcp_nr(den);
      ga[c] = (d0 - e0 * alp) * rd;
      de[c] = -f0 * rd;
      al[c] = dl - el * (alp + bep * ga[c]);
      be[c] = -(el * bep * de[c] + fl);
      alp = al[c];
      bep = be[c];
    }
    double Fn = 0.0, Lv = 0.0, Rv = 0.0;   // Fn: F_{c+1}
    for (int c = ncta - 1; c >= 0; c--) {
      if (c == rank + 1) Rv = ga[c] + de[c] * Fn;
      if (c == rank - 1) Lv = al[c] + be[c] * Fn;
      Fn = ga[c] + de[c] * Fn;
    }
    ((double*)(bnd + 6))[q] = Lv;
    ((double*)(bnd + 7))[q] = Rv;
  }
  cl.sync();   // every CTA's reads of the others' shared memory are done
  const double2 Lv = bnd[6], Rv = bnd[7];
  const double Lq[2] = {Lv.x, Lv.y}, Rq[2] = {Rv.x, Rv.y};
#pragma unroll
  for (int q = 0; q < 2; q++) d[q] = d[q] - e[q] * Lq[q] - f[q] * Rq[q];
  sy[k] = make_double2(d[0], d[1]);
  __syncthreads();

  // recover the segment's rows into the output staging (index row - rb)
  const double2 xn = k + 1 < Pt ? sy[k + 1] : Rv;
  {
    const double2 l0 = tp[k], l1 = tp[Pt + k], l2 = tp[2 * Pt + k];
    al[0][M - 1] = l0.x; al[1][M - 1] = l0.y;
    cg_[0][M - 1] = l1.x; cg_[1][M - 1] = l1.y;
    rh[0][M - 1] = l2.x; rh[1][M - 1] = l2.y;
  }
  const int ostride = opad(Pt * M + 1) + 1;
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const double Xk = d[q], Xn = q == 0 ? xn.x : xn.y;
    O* o = so + q * ostride;
    if (s <= N - 1) o[opad(s - rb)] = (O)Xk;
#pragma unroll
    for (int r = 1; r < M; r++) {
      const int i = s + r;
      if (i <= N - 1) o[opad(i - rb)] = (O)(rh[q][r] - al[q][r] * Xk - cg_[q][r] * Xn);
    }
    if (K == 0) o[0] = (O)x0[q];
    if (K == kN) o[opad(N - rb)] = (O)xN[q];
  }
  if (bad) atomicOr(err, 1);
  __syncthreads();
  const int lo = rank == 0 ? 0 : rb + 1;
  const int hi = kN / Pt == rank ? N : min(N - 1, rb + Pt * M);
  for (int i = lo + k; i <= hi; i += Pt) {
    oL[i * ist] = so[opad(i - rb)];
    oR[i * ist] = so[ostride + opad(i - rb)];
  }
}

// shared memory of a launch: PCR rows, last-row coefficients, separators,
// and the larger of the staged cells and the output staging
template <int M, bool MX>
size_t line_smem(int N, int Pt) {
  const size_t osz = MX ? sizeof(float) : sizeof(double);
  const size_t cells = (size_t)(Pt * M + 6 + (Pt * M + 6) / 8 + 1) * sizeof(double);
  const size_t outs = (size_t)2 * (N + N / 16 + 1) * osz;
  return (size_t)10 * Pt * sizeof(double2) + (cells > outs ? cells : outs);
}

template <bool MX>
size_t seg_smem(int Pt) {
  const size_t osz = MX ? sizeof(float) : sizeof(double);
  const int M = 8;
  const size_t cells = (size_t)(Pt * M + 6 + (Pt * M + 6) / 8 + 1) * sizeof(double);
  const size_t outs = (size_t)2 * (opad(Pt * M + 1) + 1) * osz;
  return (size_t)(14 * Pt + 8) * sizeof(double2) + (cells > outs ? cells : outs);
}

template <int DIR, int WT, bool MX>
void seg_launch(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                int* err, int ncta, cudaStream_t s) {
  constexpr int M = 8;
  const int N = DIR == 0 ? P.N0 : P.N1;
  const int nlines = DIR == 0 ? P.N1 : P.N0;
  const int chunks = (N - 1 + M - 1) / M;
  const int Pt = ((chunks + ncta - 1) / ncta + 31) / 32 * 32;
  raise_smem_limit<k_crw_seg<M, DIR, WT, MX>>((int)seg_smem<MX>(line_threads_max()));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nlines * ncta), (unsigned)P.nvars, 2);
  cfg.blockDim = dim3((unsigned)Pt, 1, 1);
  cfg.dynamicSmemBytes = seg_smem<MX>(Pt);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)ncta;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_crw_seg<M, DIR, WT, MX>, P, U, F, uL, uR, fL, fR, err);
}

template <int DIR, bool MX>
void seg_launch_wt(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                   int* err, int ncta, cudaStream_t s) {
  if (P.no_limiting) return seg_launch<DIR, WT_NOLIM, MX>(P, U, F, uL, uR, fL, fR, err, ncta, s);
  switch (P.weno_type) {
    case W_MAPPED: return seg_launch<DIR, W_MAPPED, MX>(P, U, F, uL, uR, fL, fR, err, ncta, s);
    case W_BORGES: return seg_launch<DIR, W_BORGES, MX>(P, U, F, uL, uR, fL, fR, err, ncta, s);
    case W_YC: return seg_launch<DIR, W_YC, MX>(P, U, F, uL, uR, fL, fR, err, ncta, s);
    default: return seg_launch<DIR, W_JS, MX>(P, U, F, uL, uR, fL, fR, err, ncta, s);
  }
}

template <int M, int DIR, int WT, bool MX>
void line_launch(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                 int* err, cudaStream_t s, int nv) {
  const int N = DIR == 0 ? P.N0 : P.N1;
  const int Pt = line_threads_m<M>(N);
  constexpr int T = line_threads_max();
  raise_smem_limit<k_crw_line<M, DIR, WT, MX>>((int)line_smem<M, MX>(T * M + 1, T));
  dim3 grid(DIR == 0 ? P.N1 : P.N0, nv, 2);
  k_crw_line<M, DIR, WT, MX><<<grid, Pt, line_smem<M, MX>(N, Pt), s>>>(P, U, F, uL, uR, fL, fR, err);
}

template <int M, int DIR, bool MX>
void line_launch_wt(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                    int* err, cudaStream_t s, int nv) {
  if (P.no_limiting) return line_launch<M, DIR, WT_NOLIM, MX>(P, U, F, uL, uR, fL, fR, err, s, nv);
  switch (P.weno_type) {
    case W_MAPPED: return line_launch<M, DIR, W_MAPPED, MX>(P, U, F, uL, uR, fL, fR, err, s, nv);
    case W_BORGES: return line_launch<M, DIR, W_BORGES, MX>(P, U, F, uL, uR, fL, fR, err, s, nv);
    case W_YC: return line_launch<M, DIR, W_YC, MX>(P, U, F, uL, uR, fL, fR, err, s, nv);
    default: return line_launch<M, DIR, W_JS, MX>(P, U, F, uL, uR, fL, fR, err, s, nv);
  }
}

template <int M>
void line_launch_m(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                   int dir, int* err, cudaStream_t s, int nv) {
  if (P.mixed) line_launch_wt<M, 0, true>(P, U, F, uL, uR, fL, fR, err, s, nv);
  else if (dir == 0) line_launch_wt<M, 0, false>(P, U, F, uL, uR, fL, fR, err, s, nv);
  else line_launch_wt<M, 1, false>(P, U, F, uL, uR, fL, fR, err, s, nv);
}

}  // namespace

// lines of 3 .. 4097 interfaces: 8 rows per thread from 128 interfaces up
// (up to 512 threads), 4 below
bool crweno_line_fits(int N) { return N >= 3 && line_threads_m<8>(N) <= line_threads_max(); }

// lines of 4098 .. 32769 interfaces: clusters of up to 8 CTAs
int launch_crweno_seg(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                      int dir, int* err, cudaStream_t s) {
  const int N = dir == 0 ? P.N0 : P.N1;
  if (crweno_cluster_size(N) < 2 || (P.mixed && dir != 0)) return -1;
  // CTAs of at most 256 threads (two per SM, so that one CTA's barrier
  // phases overlap the other's arithmetic) while eight of them cover the
  // line, else of 512: 28.9 vs 33.6 ms per launch at 8192^2
  const int chunks = (N - 1 + 7) / 8;
  int ncta = (chunks + 255) / 256;
  if (ncta > 8) ncta = (chunks + 511) / 512;
  if (P.mixed) seg_launch_wt<0, true>(P, U, F, uL, uR, fL, fR, err, ncta, s);
  else if (dir == 0) seg_launch_wt<0, false>(P, U, F, uL, uR, fL, fR, err, ncta, s);
  else seg_launch_wt<1, false>(P, U, F, uL, uR, fL, fR, err, ncta, s);
  return 0;
}

int launch_crweno_line(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL,
                       void* fR, int dir, int* err, cudaStream_t s) {
  const int N = dir == 0 ? P.N0 : P.N1;
  if (!crweno_line_fits(N) || (P.mixed && dir != 0)) return -1;
  if (N >= 128) line_launch_m<8>(P, U, F, uL, uR, fL, fR, dir, err, s, P.nvars);
  else line_launch_m<4>(P, U, F, uL, uR, fL, fR, dir, err, s, P.nvars);
  return 0;
}

}  // namespace piafs
