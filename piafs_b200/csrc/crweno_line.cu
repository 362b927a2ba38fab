// CRWENO5 interface reconstruction, one CTA per line, component and field,
// lines of up to 4097 interfaces (sm_100a): x lines (unit stride, also the y
// lines of a transposed state) and strided y lines.
//
// The method is that of k_crweno_pair (crweno.cu): Interp1PrimFifthOrderCRWENO
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
#include <type_traits>

#include "crweno_solve.cuh"
#include "kernels.h"

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
  // N + 1 interfaces over Pt threads: at most M + 1 each
#pragma unroll
  for (int it = 0; it <= M; it++) {
    const int i = k + it * Pt;
    if (i <= N) {
      oL[i * ist] = so[opad(i)];
      oR[i * ist] = so[ostride + opad(i)];
    }
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

int launch_crweno_line(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL,
                       void* fR, int dir, int* err, cudaStream_t s) {
  const int N = dir == 0 ? P.N0 : P.N1;
  if (!crweno_line_fits(N) || (P.mixed && dir != 0)) return -1;
  if (N >= 128) line_launch_m<8>(P, U, F, uL, uR, fL, fR, dir, err, s, P.nvars);
  else line_launch_m<4>(P, U, F, uL, uR, fL, fR, dir, err, s, P.nvars);
  return 0;
}

}  // namespace piafs
