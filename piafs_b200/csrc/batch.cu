// Batched simulations: many independent PIAFS runs advanced together (sm_100a).
//
// The reference runs an ensemble one member after another (one deck each,
// OutputSolution.cpp).  Here every member lives on the device at once and one
// persistent kernel per Runge-Kutta stage advances all of them: a CTA walks a
// device-side list of tiles (tile -> member), and for each tile it
//   1. loads the stage state on the tile plus a 3-cell halo into shared
//      memory, computing boundary ghosts on the fly from the member's zones
//      (bc_point, the rule of the boundary kernels),
//   2. reconstructs the WENO5 interface values of u and of the cell-centred
//      flux at every x and y interface of the tile (weno5_iface), upwinds
//      them (upwind_flow) and forms -dxinv (fI[+1] - fI) in both directions,
//   3. adds the viscous terms (2D, FirstDerivativeFirstOrder stencils on the
//      tile) and the photochemical source,
//   4. writes the stage derivative k_s and the next stage state
//      U_{s+1} = u + dt sum_j a_{s+1,j} k_j, or at the last stage
//      u <- u + dt sum_j b_j k_j.
// The expressions are those of the single-simulation kernels; a member's FP64
// result agrees with its deck run alone to rounding (the compiler contracts
// multiply-adds differently in the fused kernel), and it is bit for bit the
// same whatever other members share the batch, since a tile's arithmetic
// depends only on its own member.
// A per-step epilogue advances the members' clocks and retires members that
// reached their step count.  The tile list and the member table are device
// arrays the host rewrites between steps, so one CUDA graph of a step serves
// any mix of members (continuous batching).
//
// Stage buffers: stage s reads U_s (u for s = 0, else buffer (s-1) % 2) and
// writes U_{s+1} into buffer s % 2, so no tile overwrites state a neighbouring
// tile still reads as halo; the last stage updates u in place (pointwise),
// except for one-stage schemes, which write buffer 0 and swap it with u.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/piafs_gpu.h"
#include "deck.h"
#include "kernels.h"
#include "physics.cuh"
#include "source.cuh"

namespace piafs {
int set_last_error(int code, const std::string& msg);   // api.cu: piafs_gpu_last_error()
}

using namespace piafs;

namespace {

constexpr int BT = 256;          // threads of the stage kernel
constexpr int H = 3;             // halo (WENO5 stencil half-width)
constexpr int T1 = 256;          // points of a 1D tile

// Host-written description of one member.
struct BMember {
  DevParams P;
  double* X;                     // stage buffers (ghosted SoA planes)
  double* Y;
  double* k[MAX_STAGES];         // stage derivatives
  const double* dxinv;
  const double* imap;
  Zone zones[MAX_ZONES];
  int nzones;
  int nstages;
  double a[MAX_STAGES * MAX_STAGES];   // dt * A, row s = coefficients of stage s
  double b[MAX_STAGES];                // dt * b
  double c[MAX_STAGES];
  int tile_off, tnx, tny;
  int nsteps;
};
// Device-written state of one member.
struct BState {
  double* u;                     // solution u_n (swapped with X by one-stage schemes)
  double* X;
  double t;
  int iter;
  int active;
};

// ------------------------------------------------------------ ghost values
// Value of every variable at tile point (i, j) of stage state S: interior
// points from memory, edge ghosts (exactly one index outside the domain, at
// most 3 deep) from the last boundary zone that covers them, other points 0
// (corners; never used by the stencils).
__device__ __forceinline__ void load_point(const BMember& M, const double* S, int i, int j, double* out,
                                           int ostride) {
  const DevParams& P = M.P;
  const bool xin = i >= 0 && i < P.N0, yin = j >= 0 && j < P.N1;
  const int nv = P.nvars;
  if (xin && yin) {
    const long long p = pidx(P, i, j);
    for (int v = 0; v < nv; v++) out[v * ostride] = S[v * P.ps + p];
    return;
  }
  const bool edge = (yin && i >= -P.ghosts && i < P.N0 + P.ghosts) ||
                    (P.ndims == 2 && xin && j >= -P.ghosts && j < P.N1 + P.ghosts);
  if (!edge) {
    for (int v = 0; v < nv; v++) out[v * ostride] = 0.0;
    return;
  }
  // memory value first (what a slip wall leaves untouched), then the zone
  const long long p = pidx(P, i, j);
  for (int v = 0; v < nv; v++) out[v * ostride] = S[v * P.ps + p];
  for (int zi = M.nzones - 1; zi >= 0; zi--) {
    const Zone& z = M.zones[zi];
    if (i >= z.is[0] && i < z.ie[0] && j >= z.is[1] && j < z.ie[1]) {
      double tmp[32];
      bc_point(P, z, S, i, j, tmp, 1);
      const int nw = z.type == BC_SLIPWALL ? (P.ndims == 2 ? 4 : 3) : nv;
      for (int v = 0; v < nw; v++) out[v * ostride] = tmp[v];
      return;
    }
  }
}

// Upwind flux of every variable at the interface between the cells at smem
// offsets cell(r) = base + (r - 3) * st (r = 0..5 for cells i-3..i+2) of the
// tile state sU ([v][...], plane stride vs); result to so[v * sstride].
template <int MODEL, int UPW>
__device__ __forceinline__ void iface_flux(const DevParams& P, const double* sU, int vs, int base, int st, int dir,
                                           double* so, int sstride) {
  constexpr int NF = Flow<MODEL>::NF;
  double fc[4][6], vn[6];
#pragma unroll
  for (int r = 0; r < 6; r++) {
    const int c = base + (r - 3) * st;
    double f[4] = {0.0, 0.0, 0.0, 0.0}, w;
    if (MODEL == NS2D) ns2d_flux(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, dir, f, w);
    else euler1d_flux(sU[c], sU[vs + c], sU[2 * vs + c], P.gamma, f, w);
#pragma unroll
    for (int m = 0; m < NF; m++) fc[m][r] = f[m];
    vn[r] = w;
  }
  double uL[4], uR[4], fL[4], fR[4], ucl[4], ucr[4], fi[4], spa;
  int spm;
#pragma unroll
  for (int m = 0; m < NF; m++) {
    double a[6];
#pragma unroll
    for (int r = 0; r < 6; r++) a[r] = sU[m * vs + base + (r - 3) * st];
    weno5_iface(P, a, fc[m], uL[m], uR[m], fL[m], fR[m]);
    ucl[m] = a[2]; ucr[m] = a[3];
  }
  upwind_flow<MODEL, UPW, double>(uL, uR, fL, fR, ucl, ucr, P.gamma, dir, fi, &spa, &spm);
#pragma unroll
  for (int m = 0; m < NF; m++) so[m * sstride] = fi[m];
  for (int m = NF; m < P.nvars; m++) {
    double a[6], b[6], l, r, fl, fr;
#pragma unroll
    for (int q = 0; q < 6; q++) { a[q] = sU[m * vs + base + (q - 3) * st]; b[q] = __dmul_rn(vn[q], a[q]); }
    weno5_iface(P, a, b, l, r, fl, fr);
    so[m * sstride] = upwind_species(spm, spa, l, r, fl, fr);
  }
}

// the Runge-Kutta part of stage s at point p with stage derivatives k
__device__ __forceinline__ void rk_point(const BMember& M, const BState& Sd, int s, long long p, int nv) {
  const long long ps = M.P.ps;
  if (s < M.nstages - 1) {
    double* dst = (s % 2 == 0) ? M.X : M.Y;
    for (int v = 0; v < nv; v++) {
      const long long q = v * ps + p;
      double x = Sd.u[q];
      for (int j = 0; j <= s; j++) x += M.a[(s + 1) * MAX_STAGES + j] * M.k[j][q];
      dst[q] = x;
    }
  } else {
    double* dst = M.nstages == 1 ? Sd.X : Sd.u;
    for (int v = 0; v < nv; v++) {
      const long long q = v * ps + p;
      double x = Sd.u[q];
      for (int j = 0; j < M.nstages; j++) x += M.b[j] * M.k[j][q];
      dst[q] = x;
    }
  }
}

// ------------------------------------------------------------- 2D tile
// shared memory (doubles): sU [nv][TY+6][TX+6], sFx [nv][TY][TX+1],
// sFy [nv][TX][TY+2], Q [3][TY+2][TX+2], viscous fluxes [3][TY][TX+1] and
// [3][TY+1][TX]
template <int TX, int TY>
__host__ __device__ constexpr long long smem2d(int nv) {
  return (long long)nv * ((TY + 2 * H) * (TX + 2 * H) + TY * (TX + 1) + TX * (TY + 2)) +
         3LL * (TY + 2) * (TX + 2) + 3LL * TY * (TX + 1) + 3LL * (TY + 1) * TX;
}

template <int TX, int TY, int UPW>
__device__ void tile2d(const BMember& M, const BState& Sd, int s, int tx, int ty, double* smem) {
  const DevParams& P = M.P;
  constexpr int HX = TX + 2 * H, HY = TY + 2 * H, LX = TX + 1, LY = TY + 2;
  const int nv = P.nvars, N0 = P.N0, N1 = P.N1;
  const int i0 = tx * TX, j0 = ty * TY;
  const double* S = s == 0 ? Sd.u : ((s - 1) % 2 == 0 ? M.X : M.Y);
  const int vs = HX * HY;
  double* sU = smem;
  double* sFx = sU + nv * vs;
  double* sFy = sFx + nv * TY * LX;
  double* sQ = sFy + nv * TX * LY;              // [3][TY+2][TX+2]
  double* sVx = sQ + 3 * (TY + 2) * (TX + 2);   // [3][TY][TX+1]
  double* sVy = sVx + 3 * TY * (TX + 1);        // [3][TY+1][TX]
  const int tid = threadIdx.x;
  for (int e = tid; e < vs; e += BT) load_point(M, S, i0 - H + e % HX, j0 - H + e / HX, sU + e, vs);
  __syncthreads();
  // x interfaces (TX+1 per tile row)
  for (int e = tid; e < LX * TY; e += BT) {
    const int ii = e % LX, jj = e / LX, i = i0 + ii, j = j0 + jj;
    if (i > N0 || j >= N1) continue;
    iface_flux<NS2D, UPW>(P, sU, vs, (jj + H) * HX + ii + H, 1, 0, sFx + jj * LX + ii, TY * LX);
  }
  // y interfaces (TY+1 per tile column)
  for (int e = tid; e < TX * (TY + 1); e += BT) {
    const int ii = e % TX, jj = e / TX, i = i0 + ii, j = j0 + jj;
    if (j > N1 || i >= N0) continue;
    iface_flux<NS2D, UPW>(P, sU, vs, (jj + H) * HX + ii + H, HX, 1, sFy + ii * LY + jj, TX * LY);
  }
  // viscous fluxes (k_visc_source on this tile)
  const bool visc = P.viscous != 0;
  if (visc) {
    constexpr int QX = TX + 2, QY = TY + 2, FX = TX + 1, FY = TY + 1;
    for (int e = tid; e < QX * QY; e += BT) {
      const int a = e % QX, b = e / QX;
      const int i = i0 - 1 + a, j = j0 - 1 + b;
      double uu = 0.0, vv = 0.0, TT = 0.0;
      const bool xin = i >= 0 && i < N0, yin = j >= 0 && j < N1;
      if ((xin || yin) && i >= -P.ghosts && i < N0 + P.ghosts && j >= -P.ghosts && j < N1 + P.ghosts) {
        const int c = (b - 1 + H) * HX + (a - 1 + H);
        double rho, e_, pr;
        ns_flowvar(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, rho, uu, vv, e_, pr);
        TT = P.gamma * pr / rho;
      }
      sQ[e] = uu; sQ[QX * QY + e] = vv; sQ[2 * QX * QY + e] = TT;
    }
    __syncthreads();
    const double two_third = 2.0 / 3.0, inv_Re = 1.0 / P.Re, inv_Pr = 1.0 / P.Pr;
    const double igm1 = 1.0 / (P.gamma - 1.0);
    const double* su = sQ;
    const double* sv = sQ + QX * QY;
    const double* sT = sQ + 2 * QX * QY;
    for (int e = tid; e < FX * FY; e += BT) {
      const int a = e % FX, b = e / FX;
      const int i = i0 - 1 + a, j = j0 - 1 + b;
      const bool need_x = (b >= 1) && (j < N1) && (i < N0);
      const bool need_y = (a >= 1) && (i < N0) && (j < N1);
      if (!need_x && !need_y) continue;
      const int q = b * QX + a;
      const double dxi = M.dxinv[P.ghosts + i], dyi = M.dxinv[P.W0 + P.ghosts + j];
      const bool row_int = (j >= 0 && j < N1), col_int = (i >= 0 && i < N0);
      const double uc = su[q], vc = sv[q], Tc = sT[q];
      const double ux = row_int ? dxi * (su[q + 1] - uc) : 0.0;
      const double vx = row_int ? dxi * (sv[q + 1] - vc) : 0.0;
      const double Tx = row_int ? dxi * (sT[q + 1] - Tc) : 0.0;
      const double uy = col_int ? dyi * (su[q + QX] - uc) : 0.0;
      const double vy = col_int ? dyi * (sv[q + QX] - vc) : 0.0;
      const double Ty = col_int ? dyi * (sT[q + QX] - Tc) : 0.0;
      double mu, kappa;
      visc_coeffs<double>(P, Tc, mu, kappa);
      const double mre = mu * inv_Re, kre = kappa * inv_Re * igm1 * inv_Pr;
      if (need_x) {
        const double txx = two_third * mre * (2.0 * ux - vy), txy = mre * (uy + vx);
        double* f = sVx + (b - 1) * FX + a;
        f[0] = txx; f[TY * FX] = txy; f[2 * TY * FX] = uc * txx + vc * txy + kre * Tx;
      }
      if (need_y) {
        const double tyx = mre * (uy + vx), tyy = two_third * mre * (-ux + 2.0 * vy);
        double* f = sVy + b * TX + (a - 1);
        f[0] = tyx; f[FY * TX] = tyy; f[2 * FY * TX] = uc * tyx + vc * tyy + kre * Ty;
      }
    }
  }
  __syncthreads();
  // stage derivative and the Runge-Kutta combination, one point per thread
  const int pi = tid % TX, pj = tid / TX, i = i0 + pi, j = j0 + pj;
  if (pj >= TY || i >= N0 || j >= N1) return;
  const long long p = pidx(P, i, j);
  const long long ps = P.ps;
  double* ks = M.k[s];
  const double dxi = M.dxinv[P.ghosts + i], dyi = M.dxinv[P.W0 + P.ghosts + j];
  for (int m = 0; m < nv; m++) {
    const double hx = dxi * (sFx[m * TY * LX + pj * LX + pi + 1] - sFx[m * TY * LX + pj * LX + pi]);
    const double hy = dyi * (sFy[m * TX * LY + pi * LY + pj + 1] - sFy[m * TX * LY + pi * LY + pj]);
    const double h = hx + hy;
    ks[m * ps + p] = -h;
  }
  if (visc) {
    constexpr int FX = TX + 1, FY = TY + 1;
#pragma unroll
    for (int m = 0; m < 3; m++) {
      const double par = dxi * (sVx[m * TY * FX + pj * FX + pi + 1] - sVx[m * TY * FX + pj * FX + pi]) +
                         dyi * (sVy[m * FY * TX + (pj + 1) * TX + pi] - sVy[m * FY * TX + pj * TX + pi]);
      ks[(m + 1) * ps + p] += par;
    }
  }
  if (P.chem) {
    const double t = Sd.t + M.c[s] * P.dt;
    chem_source_point<double>(P, S, p, pulse_factor(P, t), M.imap[p], ks);
  }
  rk_point(M, Sd, s, p, nv);
}

// ------------------------------------------------------------- 1D tile
// shared memory (doubles): sU [nv][T1+6], sF [nv][T1+1]
__host__ __device__ constexpr long long smem1d(int nv) { return (long long)nv * ((T1 + 2 * H) + (T1 + 1)); }

template <int UPW>
__device__ void tile1d(const BMember& M, const BState& Sd, int s, int tx, double* smem) {
  const DevParams& P = M.P;
  constexpr int HX = T1 + 2 * H, LX = T1 + 1;
  const int nv = P.nvars, N0 = P.N0;
  const int i0 = tx * T1;
  const double* S = s == 0 ? Sd.u : ((s - 1) % 2 == 0 ? M.X : M.Y);
  double* sU = smem;
  double* sF = sU + nv * HX;
  const int tid = threadIdx.x;
  for (int e = tid; e < HX; e += BT) load_point(M, S, i0 - H + e, 0, sU + e, HX);
  __syncthreads();
  for (int e = tid; e < LX; e += BT) {
    const int i = i0 + e;
    if (i > N0) continue;
    iface_flux<EULER1D, UPW>(P, sU, HX, e + H, 1, 0, sF + e, LX);
  }
  __syncthreads();
  const int i = i0 + tid;
  if (i >= N0) return;
  const long long p = pidx(P, i, 0);
  double* ks = M.k[s];
  const double dxi = M.dxinv[P.ghosts + i];
  for (int m = 0; m < nv; m++) {
    const double h = dxi * (sF[m * LX + tid + 1] - sF[m * LX + tid]);
    ks[m * P.ps + p] = -h;
  }
  rk_point(M, Sd, s, p, nv);
}

// --------------------------------------------------------------- kernels
template <int TX, int TY>
__global__ void __launch_bounds__(BT) k_batch_stage(const BMember* __restrict__ mem, const BState* __restrict__ st,
                                                    const int* __restrict__ tile_member,
                                                    const int* __restrict__ ntiles, int s) {
  extern __shared__ double smem[];
  const int nt = *ntiles;
  for (int g = blockIdx.x; g < nt; g += gridDim.x) {
    const int m = tile_member[g];
    const BMember& M = mem[m];
    const BState Sd = st[m];
    if (!Sd.active || s >= M.nstages) continue;   // uniform over the CTA
    const int local = g - M.tile_off;
    if (M.P.ndims == 2) {
      const int tx = local % M.tnx, ty = local / M.tnx;
      switch (M.P.upwind) {
        case UPW_ROE: tile2d<TX, TY, UPW_ROE>(M, Sd, s, tx, ty, smem); break;
        case UPW_RF: tile2d<TX, TY, UPW_RF>(M, Sd, s, tx, ty, smem); break;
        case UPW_LLF: tile2d<TX, TY, UPW_LLF>(M, Sd, s, tx, ty, smem); break;
        default: tile2d<TX, TY, UPW_RUSANOV>(M, Sd, s, tx, ty, smem); break;
      }
    } else {
      switch (M.P.upwind) {
        case UPW_ROE: tile1d<UPW_ROE>(M, Sd, s, local, smem); break;
        case UPW_RF: tile1d<UPW_RF>(M, Sd, s, local, smem); break;
        case UPW_LLF: tile1d<UPW_LLF>(M, Sd, s, local, smem); break;
        default: tile1d<UPW_RUSANOV>(M, Sd, s, local, smem); break;
      }
    }
    __syncthreads();   // shared memory is reused by the next tile
  }
}

// clocks (k_advance_time), step counts, retirement; status[2m] = iter,
// status[2m+1] = active
__global__ void k_batch_epilogue(const BMember* __restrict__ mem, BState* __restrict__ st, int n,
                                 int* __restrict__ status) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  BState S = st[m];
  if (S.active) {
    S.t += mem[m].P.dt;
    S.iter += 1;
    if (mem[m].nstages == 1) { double* tmp = S.u; S.u = S.X; S.X = tmp; }
    if (S.iter >= mem[m].nsteps) S.active = 0;
    st[m] = S;
  }
  status[2 * m] = S.iter;
  status[2 * m + 1] = S.active;
}

// ------------------------------------------------------------- host side
struct HostMember {
  bool used = false;
  bool reported = false;
  Deck deck;
  BMember bm{};
  void* block = nullptr;     // one allocation: u, X, Y, k[], dxinv, imap
  size_t bytes = 0;
};

int nfail(int code, const std::string& m) { return piafs::set_last_error(code, m); }

#define BCK(call)                                                                               \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

struct TileShape { int tx, ty; };
constexpr TileShape kShapes[3] = {{32, 8}, {16, 16}, {64, 4}};

}  // namespace

struct piafs_gpu_batch {
  int precision = 0;
  unsigned long long budget = 0, used = 0;
  int device = 0, num_sms = 0;
  cudaStream_t stream = nullptr;
  std::vector<HostMember> members;     // slots
  int cap = 0;                         // slots on the device
  BMember* dmem = nullptr;
  BState* dstate = nullptr;
  int* dstatus = nullptr;
  int* hstatus = nullptr;              // pinned
  int* dtiles = nullptr;
  int* dntiles = nullptr;
  int tile_cap = 0, ntiles = 0;
  int shape = 0;                       // index into kShapes
  int max_nv = 0, max_stages = 0;
  bool dirty = true;                   // tile list / member table need upload
  cudaGraphExec_t graph = nullptr;
  int graph_shape = -1, graph_cap = -1, graph_nv = -1, graph_stages = -1, graph_grid = -1;
  long long steps = 0;
};

namespace {

long long smem_bytes(int shape, int nv) {
  long long d2 = 0;
  switch (shape) {
    case 0: d2 = smem2d<32, 8>(nv); break;
    case 1: d2 = smem2d<16, 16>(nv); break;
    default: d2 = smem2d<64, 4>(nv); break;
  }
  return std::max(d2, smem1d(nv)) * (long long)sizeof(double);
}

template <int TX, int TY>
cudaError_t launch_stage_shape(piafs_gpu_batch* B, int grid, int s) {
  const long long sm = smem_bytes(B->shape, B->max_nv);
  k_batch_stage<TX, TY><<<grid, BT, sm, B->stream>>>(B->dmem, B->dstate, B->dtiles, B->dntiles, s);
  return cudaGetLastError();
}

cudaError_t set_smem_attr(int shape, long long bytes) {
  switch (shape) {
    case 0: return cudaFuncSetAttribute(k_batch_stage<32, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    case 1: return cudaFuncSetAttribute(k_batch_stage<16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    default: return cudaFuncSetAttribute(k_batch_stage<64, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  }
}

int persistent_grid(piafs_gpu_batch* B) {
  const long long sm = smem_bytes(B->shape, std::max(B->max_nv, 1));
  int per_sm = 0;
  cudaError_t e;
  switch (B->shape) {
    case 0: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_stage<32, 8>, BT, sm); break;
    case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_stage<16, 16>, BT, sm); break;
    default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_stage<64, 4>, BT, sm); break;
  }
  if (e != cudaSuccess || per_sm < 1) per_sm = 1;
  return per_sm * B->num_sms;
}

// tiles of a member under the current shape
void member_tiles(const piafs_gpu_batch* B, BMember& m) {
  const TileShape ts = kShapes[B->shape];
  if (m.P.ndims == 2) { m.tnx = (m.P.N0 + ts.tx - 1) / ts.tx; m.tny = (m.P.N1 + ts.ty - 1) / ts.ty; }
  else { m.tnx = (m.P.N0 + T1 - 1) / T1; m.tny = 1; }
}

// rebuild the tile list over the members still stepping and upload the
// member table
int sync_tables(piafs_gpu_batch* B) {
  std::vector<int> tiles;
  for (int i = 0; i < (int)B->members.size(); i++) {
    HostMember& hm = B->members[i];
    if (!hm.used) continue;
    member_tiles(B, hm.bm);
    hm.bm.tile_off = (int)tiles.size();
    if (!hm.reported) tiles.insert(tiles.end(), (size_t)hm.bm.tnx * hm.bm.tny, i);
  }
  if ((int)tiles.size() > B->tile_cap) {
    int nc = std::max((int)tiles.size(), 2 * B->tile_cap);
    int* nt = nullptr;
    BCK(cudaMallocAsync(&nt, (size_t)nc * sizeof(int), B->stream));
    if (B->dtiles) BCK(cudaFreeAsync(B->dtiles, B->stream));
    B->dtiles = nt;
    B->tile_cap = nc;
    B->graph_cap = -1;   // kernel arguments changed
  }
  B->ntiles = (int)tiles.size();
  if (!tiles.empty())
    BCK(cudaMemcpyAsync(B->dtiles, tiles.data(), tiles.size() * sizeof(int), cudaMemcpyHostToDevice, B->stream));
  BCK(cudaMemcpyAsync(B->dntiles, &B->ntiles, sizeof(int), cudaMemcpyHostToDevice, B->stream));
  std::vector<BMember> tab(B->cap);
  for (int i = 0; i < (int)B->members.size(); i++)
    if (B->members[i].used) tab[i] = B->members[i].bm;
  BCK(cudaMemcpyAsync(B->dmem, tab.data(), (size_t)B->cap * sizeof(BMember), cudaMemcpyHostToDevice, B->stream));
  // the host copies must stay alive until the copies ran
  BCK(cudaStreamSynchronize(B->stream));
  B->dirty = false;
  return PIAFS_OK;
}

int grow_slots(piafs_gpu_batch* B, int need) {
  if (need <= B->cap) return PIAFS_OK;
  const int nc = std::max(need, std::max(16, 2 * B->cap));
  BMember* nm = nullptr;
  BState* ns = nullptr;
  int *nst = nullptr, *nhs = nullptr;
  BCK(cudaMallocAsync(&nm, (size_t)nc * sizeof(BMember), B->stream));
  BCK(cudaMallocAsync(&ns, (size_t)nc * sizeof(BState), B->stream));
  BCK(cudaMallocAsync(&nst, (size_t)nc * 2 * sizeof(int), B->stream));
  BCK(cudaMallocHost(&nhs, (size_t)nc * 2 * sizeof(int)));
  std::memset(nhs, 0, (size_t)nc * 2 * sizeof(int));
  BCK(cudaMemsetAsync(ns, 0, (size_t)nc * sizeof(BState), B->stream));
  BCK(cudaMemsetAsync(nst, 0, (size_t)nc * 2 * sizeof(int), B->stream));
  if (B->dstate) {
    BCK(cudaMemcpyAsync(ns, B->dstate, (size_t)B->cap * sizeof(BState), cudaMemcpyDeviceToDevice, B->stream));
    BCK(cudaMemcpyAsync(nst, B->dstatus, (size_t)B->cap * 2 * sizeof(int), cudaMemcpyDeviceToDevice, B->stream));
    BCK(cudaStreamSynchronize(B->stream));
    BCK(cudaFreeAsync(B->dmem, B->stream));
    BCK(cudaFreeAsync(B->dstate, B->stream));
    BCK(cudaFreeAsync(B->dstatus, B->stream));
    std::memcpy(nhs, B->hstatus, (size_t)B->cap * 2 * sizeof(int));
    cudaFreeHost(B->hstatus);
  }
  B->dmem = nm; B->dstate = ns; B->dstatus = nst; B->hstatus = nhs;
  B->cap = nc;
  B->graph_cap = -1;
  B->dirty = true;
  return PIAFS_OK;
}

int capture_graph(piafs_gpu_batch* B) {
  const int grid = persistent_grid(B);
  if (B->graph && B->graph_shape == B->shape && B->graph_cap == B->cap && B->graph_nv == B->max_nv &&
      B->graph_stages == B->max_stages && B->graph_grid == grid)
    return PIAFS_OK;
  if (B->graph) { cudaGraphExecDestroy(B->graph); B->graph = nullptr; }
  const long long sm = smem_bytes(B->shape, B->max_nv);
  BCK(set_smem_attr(B->shape, sm));
  cudaGraph_t g;
  BCK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < B->max_stages && e == cudaSuccess; s++) {
    switch (B->shape) {
      case 0: e = launch_stage_shape<32, 8>(B, grid, s); break;
      case 1: e = launch_stage_shape<16, 16>(B, grid, s); break;
      default: e = launch_stage_shape<64, 4>(B, grid, s); break;
    }
  }
  if (e == cudaSuccess) {
    k_batch_epilogue<<<(B->cap + 127) / 128, 128, 0, B->stream>>>(B->dmem, B->dstate, B->cap, B->dstatus);
    e = cudaGetLastError();
  }
  cudaError_t e2 = cudaStreamEndCapture(B->stream, &g);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("batch step capture: ") + cudaGetErrorString(e));
  BCK(e2);
  e = cudaGraphInstantiate(&B->graph, g, 0);
  cudaGraphDestroy(g);
  BCK(e);
  B->graph_shape = B->shape; B->graph_cap = B->cap; B->graph_nv = B->max_nv;
  B->graph_stages = B->max_stages; B->graph_grid = grid;
  return PIAFS_OK;
}

}  // namespace

extern "C" {

int piafs_gpu_batch_create(int precision, unsigned long long budget, piafs_gpu_batch** out) {
  if (!out) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  if (precision != PIAFS_PRECISION_FP64 && precision != PIAFS_PRECISION_MIXED)
    return nfail(PIAFS_ERR_ARGUMENT, "precision must be PIAFS_PRECISION_FP64 or PIAFS_PRECISION_MIXED");
  if (precision == PIAFS_PRECISION_MIXED)
    return nfail(PIAFS_ERR_UNSUPPORTED, "the batched path runs FP64 members in this build");
  auto* B = new piafs_gpu_batch();
  B->precision = precision;
  B->budget = budget;
  cudaError_t e = cudaGetDevice(&B->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&B->num_sms, cudaDevAttrMultiProcessorCount, B->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocAsync(&B->dntiles, sizeof(int), B->stream);
  if (e == cudaSuccess) {
    // keep freed member memory in the pool instead of returning it to the driver
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, B->device) == cudaSuccess) {
      unsigned long long thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  if (e != cudaSuccess) {
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
    return nfail(PIAFS_ERR_CUDA, std::string("batch set-up: ") + cudaGetErrorString(e));
  }
  if (int r = grow_slots(B, 16)) { delete B; return r; }
  *out = B;
  return PIAFS_OK;
}

void piafs_gpu_batch_destroy(piafs_gpu_batch* B) {
  if (!B) return;
  cudaStreamSynchronize(B->stream);
  if (B->graph) cudaGraphExecDestroy(B->graph);
  for (auto& m : B->members)
    if (m.block) cudaFreeAsync(m.block, B->stream);
  if (B->dmem) cudaFreeAsync(B->dmem, B->stream);
  if (B->dstate) cudaFreeAsync(B->dstate, B->stream);
  if (B->dstatus) cudaFreeAsync(B->dstatus, B->stream);
  if (B->dtiles) cudaFreeAsync(B->dtiles, B->stream);
  if (B->dntiles) cudaFreeAsync(B->dntiles, B->stream);
  cudaStreamSynchronize(B->stream);
  if (B->hstatus) cudaFreeHost(B->hstatus);
  cudaStreamDestroy(B->stream);
  delete B;
}

int piafs_gpu_batch_add(piafs_gpu_batch* B, const char* deck_dir, int nsteps, int* id) {
  if (!B || !deck_dir || !id) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  HostMember hm;
  std::string err;
  int r = read_deck(deck_dir, hm.deck, err);
  DevParams P;
  if (!r) r = make_params(hm.deck, P, err);
  if (r) return nfail(r, err);
  const Deck& d = hm.deck;
  if (P.scheme != WENO5) return nfail(PIAFS_ERR_UNSUPPORTED, "batched members use hyp_space_scheme weno5");
  if (!((P.ndims == 2 && P.model == NS2D) || (P.ndims == 1 && P.model == EULER1D && !P.chem)))
    return nfail(PIAFS_ERR_UNSUPPORTED, "batched members are 2D navierstokes2d or 1D euler1d without chemistry");
  if (P.nvars > 32) return nfail(PIAFS_ERR_UNSUPPORTED, "batched members have at most 32 variables");
  {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, B->device);
    if (smem_bytes(B->shape, std::max(B->max_nv, P.nvars)) > optin)
      return nfail(PIAFS_ERR_UNSUPPORTED, "too many variables for the batched stage kernel's shared-memory tile");
  }
  P.mixed = 0;
  const int ns = d.nstages;
  const size_t planes = (size_t)P.nvars * P.ps;
  const size_t ndx = d.dxinv.size(), nim = d.imap.size();
  const size_t bytes = ((3 + ns) * planes + ndx + nim) * sizeof(double);
  if (B->budget && B->used + bytes > B->budget)
    return nfail(PIAFS_ERR_MEMORY, "the batch's device memory budget cannot hold this member now");
  // slot
  int slot = -1;
  for (int i = 0; i < (int)B->members.size(); i++)
    if (!B->members[i].used) { slot = i; break; }
  if (slot < 0) { slot = (int)B->members.size(); B->members.emplace_back(); }
  if (int rr = grow_slots(B, slot + 1)) return rr;
  double* blk = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&blk, bytes, B->stream);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_MEMORY, std::string("member allocation: ") + cudaGetErrorString(e));
  BMember& bm = hm.bm;
  std::memset(&bm, 0, sizeof(bm));
  bm.P = P;
  double* u = blk;
  bm.X = blk + planes;
  bm.Y = blk + 2 * planes;
  for (int k = 0; k < ns; k++) bm.k[k] = blk + (3 + k) * planes;
  double* dx = blk + (3 + ns) * planes;
  double* im = dx + ndx;
  bm.dxinv = dx;
  bm.imap = nim ? im : nullptr;
  bm.nzones = (int)d.zones.size();
  for (int z = 0; z < bm.nzones; z++) bm.zones[z] = d.zones[z];
  bm.nstages = ns;
  for (int s = 0; s < MAX_STAGES; s++) {
    for (int j = 0; j < MAX_STAGES; j++) bm.a[s * MAX_STAGES + j] = d.dt * d.A[s * MAX_STAGES + j];
    bm.b[s] = d.dt * d.b[s];
    bm.c[s] = d.c[s];
  }
  bm.nsteps = nsteps > 0 ? nsteps : d.n_iter;
  // upload: initial state (AoS with ghosts) into u, X and Y (the ghost
  // entries of the stage buffers must hold what the state's ghosts hold)
  double* stage = nullptr;
  e = cudaMallocAsync((void**)&stage, d.u0.size() * sizeof(double), B->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(stage, d.u0.data(), d.u0.size() * sizeof(double), cudaMemcpyHostToDevice, B->stream);
  if (e == cudaSuccess) { launch_aos_to_soa(stage, u, P.npg, P.nvars, P.ps, B->stream); e = cudaGetLastError(); }
  if (e == cudaSuccess) e = cudaMemcpyAsync(bm.X, u, planes * sizeof(double), cudaMemcpyDeviceToDevice, B->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(bm.Y, u, planes * sizeof(double), cudaMemcpyDeviceToDevice, B->stream);
  for (int k = 0; k < ns && e == cudaSuccess; k++) e = cudaMemsetAsync(bm.k[k], 0, planes * sizeof(double), B->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dx, d.dxinv.data(), ndx * sizeof(double), cudaMemcpyHostToDevice, B->stream);
  if (e == cudaSuccess && nim) e = cudaMemcpyAsync(im, d.imap.data(), nim * sizeof(double), cudaMemcpyHostToDevice, B->stream);
  BState st{};
  st.u = u; st.X = bm.X; st.t = d.restart_iter * d.dt; st.iter = 0; st.active = bm.nsteps > 0 ? 1 : 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(B->dstate + slot, &st, sizeof(BState), cudaMemcpyHostToDevice, B->stream);
  int stat[2] = {0, st.active};
  if (e == cudaSuccess) e = cudaMemcpyAsync(B->dstatus + 2 * slot, stat, sizeof(stat), cudaMemcpyHostToDevice, B->stream);
  if (stage) cudaFreeAsync(stage, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);   // host sources must outlive the copies
  if (e != cudaSuccess) {
    cudaFreeAsync(blk, B->stream);
    return nfail(PIAFS_ERR_CUDA, std::string("member upload: ") + cudaGetErrorString(e));
  }
  B->hstatus[2 * slot] = 0;
  B->hstatus[2 * slot + 1] = st.active;
  hm.used = true;
  hm.reported = st.active == 0;
  hm.block = blk;
  hm.bytes = bytes;
  hm.deck.u0.clear();
  hm.deck.u0.shrink_to_fit();
  hm.deck.imap.clear();
  hm.deck.imap.shrink_to_fit();
  B->used += bytes;
  B->max_nv = std::max(B->max_nv, P.nvars);
  B->max_stages = std::max(B->max_stages, ns);
  B->members[slot] = std::move(hm);
  B->dirty = true;
  *id = slot;
  return PIAFS_OK;
}

int piafs_gpu_batch_step(piafs_gpu_batch* B, int nsteps) {
  if (!B || nsteps < 0) return nfail(PIAFS_ERR_ARGUMENT, "bad argument");
  if (B->dirty) if (int r = sync_tables(B)) return r;
  if (B->ntiles == 0 || nsteps == 0) return PIAFS_OK;
  if (int r = capture_graph(B)) return r;
  for (int n = 0; n < nsteps; n++) BCK(cudaGraphLaunch(B->graph, B->stream));
  BCK(cudaMemcpyAsync(B->hstatus, B->dstatus, (size_t)B->cap * 2 * sizeof(int), cudaMemcpyDeviceToHost, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  B->steps += nsteps;
  return PIAFS_OK;
}

int piafs_gpu_batch_poll(piafs_gpu_batch* B, int* done, int cap, int* n) {
  if (!B || !n || (cap > 0 && !done)) return nfail(PIAFS_ERR_ARGUMENT, "bad argument");
  int k = 0;
  for (int i = 0; i < (int)B->members.size() && k < cap; i++) {
    HostMember& hm = B->members[i];
    if (!hm.used || hm.reported) continue;
    if (B->hstatus[2 * i + 1] == 0 && B->hstatus[2 * i] >= hm.bm.nsteps) {
      hm.reported = true;
      done[k++] = i;
      B->dirty = true;   // drop its tiles
    }
  }
  *n = k;
  return PIAFS_OK;
}

int piafs_gpu_batch_member(piafs_gpu_batch* B, int id, double* t, int* iter, int* done) {
  if (!B || id < 0 || id >= (int)B->members.size() || !B->members[id].used)
    return nfail(PIAFS_ERR_ARGUMENT, "no such member");
  BState st;
  BCK(cudaMemcpyAsync(&st, B->dstate + id, sizeof(BState), cudaMemcpyDeviceToHost, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  if (t) *t = st.t;
  if (iter) *iter = st.iter;
  if (done) *done = st.active ? 0 : 1;
  return PIAFS_OK;
}

int piafs_gpu_batch_get_solution(piafs_gpu_batch* B, int id, double* out) {
  if (!B || !out || id < 0 || id >= (int)B->members.size() || !B->members[id].used)
    return nfail(PIAFS_ERR_ARGUMENT, "no such member");
  const DevParams& P = B->members[id].bm.P;
  BState st;
  BCK(cudaMemcpyAsync(&st, B->dstate + id, sizeof(BState), cudaMemcpyDeviceToHost, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  const size_t n = (size_t)P.N0 * P.N1 * P.nvars;
  double* tmp = nullptr;
  BCK(cudaMallocAsync((void**)&tmp, n * sizeof(double), B->stream));
  launch_soa_to_interior(P, st.u, tmp, B->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, B->stream);
  cudaFreeAsync(tmp, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("member solution: ") + cudaGetErrorString(e));
  return PIAFS_OK;
}

int piafs_gpu_batch_get_stage_derivative(piafs_gpu_batch* B, int id, int stage, double* out) {
  if (!B || !out || id < 0 || id >= (int)B->members.size() || !B->members[id].used)
    return nfail(PIAFS_ERR_ARGUMENT, "no such member");
  const BMember& bm = B->members[id].bm;
  if (stage < 0 || stage >= bm.nstages) return nfail(PIAFS_ERR_ARGUMENT, "no such stage");
  const DevParams& P = bm.P;
  const size_t n = (size_t)P.N0 * P.N1 * P.nvars;
  double* tmp = nullptr;
  BCK(cudaMallocAsync((void**)&tmp, n * sizeof(double), B->stream));
  launch_soa_to_interior(P, bm.k[stage], tmp, B->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, B->stream);
  cudaFreeAsync(tmp, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("stage derivative: ") + cudaGetErrorString(e));
  return PIAFS_OK;
}

int piafs_gpu_batch_remove(piafs_gpu_batch* B, int id) {
  if (!B || id < 0 || id >= (int)B->members.size() || !B->members[id].used)
    return nfail(PIAFS_ERR_ARGUMENT, "no such member");
  HostMember& hm = B->members[id];
  BState st{};
  BCK(cudaMemcpyAsync(B->dstate + id, &st, sizeof(BState), cudaMemcpyHostToDevice, B->stream));
  BCK(cudaFreeAsync(hm.block, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  B->used -= hm.bytes;
  B->hstatus[2 * id] = 0;
  B->hstatus[2 * id + 1] = 0;
  hm = HostMember();
  B->dirty = true;
  return PIAFS_OK;
}

int piafs_gpu_batch_get_info(piafs_gpu_batch* B, piafs_gpu_batch_info* info) {
  if (!B || !info) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  if (B->dirty) if (int r = sync_tables(B)) return r;
  std::memset(info, 0, sizeof(*info));
  for (auto& m : B->members)
    if (m.used) { info->members++; if (!m.reported) info->active++; }
  info->tiles = B->ntiles;
  info->tile_x = kShapes[B->shape].tx;
  info->tile_y = kShapes[B->shape].ty;
  info->steps = B->steps;
  info->bytes_in_use = B->used;
  info->budget_bytes = B->budget;
  info->launches_per_step = B->max_stages + 1;
  return PIAFS_OK;
}

int piafs_gpu_batch_tune(piafs_gpu_batch* B, int force_tile_x) {
  if (!B) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  if (force_tile_x) {
    int k = -1;
    for (int i = 0; i < 3; i++)
      if (kShapes[i].tx == force_tile_x) k = i;
    if (k < 0) return nfail(PIAFS_ERR_ARGUMENT, "tile_x must be 32, 16 or 64");
    B->shape = k;
    B->dirty = true;
    return PIAFS_OK;
  }
  return nfail(PIAFS_ERR_UNSUPPORTED, "automatic tuning is not available in this build");
}

}  // extern "C"
