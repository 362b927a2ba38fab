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
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <thread>
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

constexpr int H = 3;             // halo (WENO5 stencil half-width)

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
// (corners; never used by the stencils).  A slip wall sets the flow variables
// and leaves the others as they are in memory, as the boundary kernel does.
__device__ __forceinline__ void load_point(const BMember& M, const double* S, int i, int j, double* out,
                                           int ostride) {
  const DevParams& P = M.P;
  const bool xin = i >= 0 && i < P.N0, yin = j >= 0 && j < P.N1;
  const int nv = P.nvars;
  const bool edge = !(xin && yin) && ((yin && i >= -P.ghosts && i < P.N0 + P.ghosts) ||
                                      (P.ndims == 2 && xin && j >= -P.ghosts && j < P.N1 + P.ghosts));
  if (!(xin && yin) && !edge) {
    for (int v = 0; v < nv; v++) out[v * ostride] = 0.0;
    return;
  }
  const long long p = pidx(P, i, j);
  for (int v = 0; v < nv; v++) out[v * ostride] = S[v * P.ps + p];
  if (!edge) return;
  for (int zi = M.nzones - 1; zi >= 0; zi--) {
    const Zone& z = M.zones[zi];
    if (i >= z.is[0] && i < z.ie[0] && j >= z.is[1] && j < z.ie[1]) {
      bc_point(P, z, S, i, j, out, ostride);
      return;
    }
  }
}

// Cell-centred fluxes of every variable at a tile cell (ns2d_flux /
// euler1d_flux, passive variables vn u_m) into f[m * fstride]; vn returned.
template <int MODEL>
__device__ __forceinline__ double cell_flux(const DevParams& P, const double* sU, int vs, int c, int dir, double* f,
                                            int fstride) {
  constexpr int NF = Flow<MODEL>::NF;
  double fl[4] = {0.0, 0.0, 0.0, 0.0}, vn;
  if (MODEL == NS2D) ns2d_flux(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, dir, fl, vn);
  else euler1d_flux(sU[c], sU[vs + c], sU[2 * vs + c], P.gamma, fl, vn);
#pragma unroll
  for (int m = 0; m < NF; m++) f[m * fstride] = fl[m];
  for (int m = NF; m < P.nvars; m++) f[m * fstride] = __dmul_rn(vn, sU[m * vs + c]);
  return vn;
}

// The four WENO5 values of one variable at one interface: u at u[(r-3)*ust]
// and its flux at f[(r-3)*fst] for the cells r = 0..5 (i-3..i+2).
__device__ __forceinline__ void iface_weno(const DevParams& P, const double* u, int ust, const double* f, int fst,
                                           double& uL, double& uR, double& fL, double& fR) {
  double a[6], b[6];
#pragma unroll
  for (int r = 0; r < 6; r++) { a[r] = u[(r - 3) * ust]; b[r] = f[(r - 3) * fst]; }
  weno5_iface(P, a, b, uL, uR, fL, fR);
}

// Characteristic / scalar upwinding of the flow variables at one interface
// from their WENO values rec[k * ks + m * ms] (k: uL, uR, fL, fR) and the cell
// states left / right (ucl, ucr at stride vs); flux to so[m * sstride],
// passive-variable scheme data to *spa / *spm.
template <int MODEL, int UPW>
__device__ __noinline__ void iface_upwind_flow(const DevParams& P, const double* rec, int ks, int ms,
                                               const double* ucl, const double* ucr, int vs, int dir, double* so,
                                               int sstride, double* spa, int* spm) {
  constexpr int NF = Flow<MODEL>::NF;
  double uL[4], uR[4], fL[4], fR[4], cl[4], cr[4], fi[4];
#pragma unroll
  for (int m = 0; m < NF; m++) {
    uL[m] = rec[m * ms]; uR[m] = rec[ks + m * ms]; fL[m] = rec[2 * ks + m * ms]; fR[m] = rec[3 * ks + m * ms];
    cl[m] = ucl[m * vs]; cr[m] = ucr[m * vs];
  }
  upwind_flow<MODEL, UPW, double>(uL, uR, fL, fR, cl, cr, P.gamma, dir, fi, spa, spm);
#pragma unroll
  for (int m = 0; m < NF; m++) so[m * sstride] = fi[m];
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
// One tile of TX x TY points, worked by BT threads in phases separated by
// barriers; each phase is a list of small items over both directions, so
// every thread stays light and the phases stay balanced:
//   load     the stage state on the tile + 3-cell halo (boundary ghosts on
//            the fly)
//   fluxes   flow-variable fluxes and the normal velocity at every stencil
//            cell of either direction
//   WENO     WENO5 values of the flow variables, item = (interface, var)
//   upwind   characteristic/scalar upwinding, item = interface
//   passive  WENO5 + scalar upwinding of a passive variable (flux vn u_m),
//            item = (interface, var)
//   viscous  Q, viscous face fluxes (k_visc_source on the tile)
//   point    stage derivative, chemistry, Runge-Kutta combination
// Interfaces are numbered x first (f < NXI: row jj, position ii) then y.
// Shared memory (doubles): sU [nv][HY][HX]; interface fluxes fx [nv][NXI] and
// fy [nv][NYI]; a work region, reused by the viscous phase: cell data
// [5][NCX] + [5][NCY], WENO values [4][4][NXI+NYI], passive speed and scheme
// [NXI+NYI] each.
template <int TX, int TY>
struct Tile2D {
  static constexpr int HX = TX + 6, HY = TY + 6;
  static constexpr int NXI = TY * (TX + 1), NYI = TX * (TY + 1), NI = NXI + NYI;
  static constexpr int NCX = TY * HX, NCY = TX * HY;            // stencil cells per direction
  static constexpr int VISC = 3 * (TY + 2) * (TX + 2) + 3 * TY * (TX + 1) + 3 * (TY + 1) * TX;
  static constexpr int WORK0 = 5 * (NCX + NCY) + 16 * NI + 2 * NI;
  static constexpr int WORK = WORK0 > VISC ? WORK0 : VISC;
  __host__ __device__ static constexpr long long smem(int nv) {
    return (long long)nv * (HX * HY + NXI + NYI) + WORK;
  }
};
template <int TX, int TY>
__host__ __device__ constexpr long long smem2d(int nv) { return Tile2D<TX, TY>::smem(nv); }

template <int TX, int TY, int UPW, int BT>
__device__ __forceinline__ void tile2d(const BMember& M, const BState& Sd, int s, int tx, int ty, double* smem) {
  typedef Tile2D<TX, TY> T;
  constexpr int HX = T::HX, HY = T::HY, NXI = T::NXI, NYI = T::NYI, NI = T::NI, NCX = T::NCX, NCY = T::NCY;
  const DevParams& P = M.P;
  const int nv = P.nvars, N0 = P.N0, N1 = P.N1;
  const int i0 = tx * TX, j0 = ty * TY;
  const double* S = s == 0 ? Sd.u : ((s - 1) % 2 == 0 ? M.X : M.Y);
  constexpr int vs = HX * HY;
  double* sU = smem;
  double* fx = sU + nv * vs;                   // [m][jj * (TX+1) + ii]
  double* fy = fx + nv * NXI;                  // [m][ii * (TY+1) + jj]
  double* wk = fy + nv * NYI;                  // work region
  double* cx = wk;                             // [5][NCX]: 4 flow fluxes + vn, x cells
  double* cy = cx + 5 * NCX;                   // [5][NCY]
  double* rec = cy + 5 * NCY;                  // [k][m][NI]
  double* spa = rec + 16 * NI;                 // [NI]
  int* spm = (int*)(spa + NI);                 // [NI]
  const int tid = threadIdx.x;
  for (int e = tid; e < vs; e += BT) load_point(M, S, i0 - H + e % HX, j0 - H + e / HX, sU + e, vs);
  __syncthreads();
  // cell data: x cells (row jj, column a): c = (jj+H)*HX + a; y cells
  // (column ii, row b): c = b*HX + ii + H
  for (int e = tid; e < NCX + NCY; e += BT) {
    const bool xd = e < NCX;
    const int g = xd ? e : e - NCX;
    const int c = xd ? (g / HX + H) * HX + g % HX : (g % HY) * HX + g / HY + H;
    double f[4], vn;
    ns2d_flux(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, xd ? 0 : 1, f, vn);
    double* o = xd ? cx + g : cy + g;
    const int st = xd ? NCX : NCY;
#pragma unroll
    for (int m = 0; m < 4; m++) o[m * st] = f[m];
    o[4 * st] = vn;
  }
  __syncthreads();
  // geometry of interface f: its cell i (right of the interface) in sU
  // (base, stride ust along the line), in the cell data (cb, plane cst) and
  // whether it is inside the member
  auto geo = [&](int f, int& base, int& ust, const double*& cd, int& cst, int& dir) -> bool {
    if (f < NXI) {
      const int ii = f % (TX + 1), jj = f / (TX + 1);
      base = (jj + H) * HX + ii + H; ust = 1; cd = cx + jj * HX + ii + H; cst = NCX; dir = 0;
      return i0 + ii <= N0 && j0 + jj < N1;
    }
    const int g = f - NXI, jj = g % (TY + 1), ii = g / (TY + 1);
    base = (jj + H) * HX + ii + H; ust = HX; cd = cy + ii * HY + jj + H; cst = NCY; dir = 1;
    return j0 + jj <= N1 && i0 + ii < N0;
  };
  for (int e = tid; e < 4 * NI; e += BT) {
    const int m = e / NI, f = e % NI;
    int base, ust, cst, dir;
    const double* cd;
    if (!geo(f, base, ust, cd, cst, dir)) continue;
    iface_weno(P, sU + m * vs + base, ust, cd + m * cst, 1, rec[(0 * 4 + m) * NI + f], rec[(1 * 4 + m) * NI + f],
               rec[(2 * 4 + m) * NI + f], rec[(3 * 4 + m) * NI + f]);
  }
  __syncthreads();
  for (int f = tid; f < NI; f += BT) {
    int base, ust, cst, dir;
    const double* cd;
    if (!geo(f, base, ust, cd, cst, dir)) continue;
    double* so = f < NXI ? fx + f : fy + (f - NXI);
    iface_upwind_flow<NS2D, UPW>(P, rec + f, 4 * NI, NI, sU + base - ust, sU + base, vs, dir, so,
                                 f < NXI ? NXI : NYI, spa + f, spm + f);
  }
  __syncthreads();
  const int np = nv - 4;
  for (int e = tid; e < np * NI; e += BT) {
    const int m = 4 + e / NI, f = e % NI;
    int base, ust, cst, dir;
    const double* cd;
    if (!geo(f, base, ust, cd, cst, dir)) continue;
    const double* u = sU + m * vs + base;
    const double* vn = cd + 4 * cst;
    double a[6], b[6], l, r, fl, fr;
#pragma unroll
    for (int q = 0; q < 6; q++) { a[q] = u[(q - 3) * ust]; b[q] = __dmul_rn(vn[q - 3], a[q]); }
    weno5_iface(P, a, b, l, r, fl, fr);
    const double h = upwind_species(spm[f], spa[f], l, r, fl, fr);
    if (f < NXI) fx[m * NXI + f] = h;
    else fy[m * NYI + f - NXI] = h;
  }
  __syncthreads();
  // viscous fluxes (k_visc_source on this tile), in the work region
  const bool visc = P.viscous != 0;
  constexpr int QX = TX + 2, QY = TY + 2, FX = TX + 1, FY = TY + 1;
  double* sQ = wk;                              // [3][QY][QX]
  double* sVx = sQ + 3 * QY * QX;               // [3][TY][FX]
  double* sVy = sVx + 3 * TY * FX;              // [3][FY][TX]
  if (visc) {
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
    __syncthreads();
  }
  // stage derivative and the Runge-Kutta combination, one point per thread
  if (tid >= TX * TY) return;
  const int pi = tid % TX, pj = tid / TX, i = i0 + pi, j = j0 + pj;
  if (i >= N0 || j >= N1) return;
  const long long p = pidx(P, i, j);
  const long long ps = P.ps;
  double* ks = M.k[s];
  const double dxi = M.dxinv[P.ghosts + i], dyi = M.dxinv[P.W0 + P.ghosts + j];
  constexpr int LX = TX + 1, LY = TY + 1;
  for (int m = 0; m < nv; m++) {
    const double hx = dxi * (fx[m * NXI + pj * LX + pi + 1] - fx[m * NXI + pj * LX + pi]);
    const double hy = dyi * (fy[m * NYI + pi * LY + pj + 1] - fy[m * NYI + pi * LY + pj]);
    const double h = hx + hy;
    ks[m * ps + p] = -h;
  }
  if (visc) {
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
// A 1D tile has T1 points, one per thread.  Shared memory (doubles): sU
// [nv][T1+6], cell fluxes [nv][T1+6], interface fluxes [nv][T1+1], flow WENO
// values [4][3][T1+1], passive speed and scheme
template <int T1>
__host__ __device__ constexpr long long smem1d(int nv) {
  return (long long)nv * (2 * (T1 + 2 * H) + (T1 + 1)) + 14LL * (T1 + 1);
}

template <int UPW, int BT>
__device__ __forceinline__ void tile1d(const BMember& M, const BState& Sd, int s, int tx, double* smem) {
  constexpr int T1 = BT;
  const DevParams& P = M.P;
  constexpr int HX = T1 + 2 * H, LX = T1 + 1, NF = 3;
  const int nv = P.nvars, N0 = P.N0;
  const int i0 = tx * T1;
  const double* S = s == 0 ? Sd.u : ((s - 1) % 2 == 0 ? M.X : M.Y);
  double* sU = smem;
  double* cf = sU + nv * HX;                 // [m][HX]
  double* sF = cf + nv * HX;                 // [m][LX]
  double* rec = sF + nv * LX;                // [k][m][LX]
  double* spa = rec + 12 * LX;
  int* spm = (int*)(spa + LX);
  const int tid = threadIdx.x;
  for (int e = tid; e < HX; e += BT) load_point(M, S, i0 - H + e, 0, sU + e, HX);
  __syncthreads();
  for (int e = tid; e < HX; e += BT) cell_flux<EULER1D>(P, sU, HX, e, 0, cf + e, HX);
  __syncthreads();
  for (int e = tid; e < NF * LX; e += BT) {
    const int m = e / LX, f = e % LX;
    if (i0 + f > N0) continue;
    iface_weno(P, sU + m * HX + f + H, 1, cf + m * HX + f + H, 1, rec[(0 * NF + m) * LX + f],
               rec[(1 * NF + m) * LX + f], rec[(2 * NF + m) * LX + f], rec[(3 * NF + m) * LX + f]);
  }
  __syncthreads();
  for (int f = tid; f < LX; f += BT) {
    if (i0 + f > N0) continue;
    iface_upwind_flow<EULER1D, UPW>(P, rec + f, NF * LX, LX, sU + f + H - 1, sU + f + H, HX, 0, sF + f, LX,
                                    spa + f, spm + f);
  }
  __syncthreads();
  for (int e = tid; e < (nv - NF) * LX; e += BT) {
    const int m = NF + e / LX, f = e % LX;
    if (i0 + f > N0) continue;
    double l, r, fl, fr;
    iface_weno(P, sU + m * HX + f + H, 1, cf + m * HX + f + H, 1, l, r, fl, fr);
    sF[m * LX + f] = upwind_species(spm[f], spa[f], l, r, fl, fr);
  }
  __syncthreads();
  const int i = i0 + tid;
  if (tid >= T1 || i >= N0) return;
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
template <int TX, int TY, int BT, int MINB>
__global__ void __launch_bounds__(BT, MINB) k_batch_stage(const BMember* __restrict__ mem,
                                                          const BState* __restrict__ st,
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
        case UPW_ROE: tile2d<TX, TY, UPW_ROE, BT>(M, Sd, s, tx, ty, smem); break;
        case UPW_RF: tile2d<TX, TY, UPW_RF, BT>(M, Sd, s, tx, ty, smem); break;
        case UPW_LLF: tile2d<TX, TY, UPW_LLF, BT>(M, Sd, s, tx, ty, smem); break;
        default: tile2d<TX, TY, UPW_RUSANOV, BT>(M, Sd, s, tx, ty, smem); break;
      }
    } else {
      switch (M.P.upwind) {
        case UPW_ROE: tile1d<UPW_ROE, BT>(M, Sd, s, local, smem); break;
        case UPW_RF: tile1d<UPW_RF, BT>(M, Sd, s, local, smem); break;
        case UPW_LLF: tile1d<UPW_LLF, BT>(M, Sd, s, local, smem); break;
        default: tile1d<UPW_RUSANOV, BT>(M, Sd, s, local, smem); break;
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

// ------------------------------------------------------- request fields
// SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): a counter-based stream, value k of seed s.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Initial fields of a request (interior points; ghosts stay zero), the
// fields of the package's case generators: 1D density wave and 2D
// photochemical beam (see piafs_gpu_request).
__global__ void k_request_init(DevParams P, int kind, double amp, double radius, double noise,
                               unsigned long long seed, double* __restrict__ u, double* __restrict__ imap) {
  const long long n = (long long)P.N0 * P.N1;
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = (int)(k % P.N0), j = (int)(k / P.N0);
  const long long p = pidx(P, i, j), ps = P.ps;
  const double g = P.gamma;
  if (kind == PIAFS_REQUEST_EULER1D_WAVE) {
    const double x = (double)i / P.N0;
    const double rho = 1.0 + amp * sin(2.0 * 3.141592653589793 * x);
    u[p] = rho;
    u[ps + p] = rho;
    u[2 * ps + p] = 1.0 / (g - 1.0) + 0.5 * rho;
    return;
  }
  const double x = (i + 0.5) / P.N0, y = (j + 0.5) / P.N1;
  const double r01 = (double)(splitmix64(seed * 0x100000001B3ull + (unsigned long long)k) >> 11) * 0x1.0p-53;
  const double rho = 1.0 + noise * (2.0 * r01 - 1.0);
  const double pr = 1.0 / g;
  u[p] = rho;
  u[ps + p] = 0.0;
  u[2 * ps + p] = 0.0;
  u[3 * ps + p] = pr / (g - 1.0);
  for (int v = 4; v < P.nvars; v++) u[v * ps + p] = 0.0;
  for (int iz = 0; (P.chem ? iz < P.nz : false) && 4 + P.zstride * iz + 1 < P.nvars; iz++) {
    u[(4 + P.zstride * iz) * ps + p] = 1.0;          // O2 (normalised)
    u[(5 + P.zstride * iz) * ps + p] = 0.005;        // O3 = f_O3 / f_O2
  }
  if (imap) {
    const double dx = x - 0.5, dy = y - 0.5;
    imap[p] = amp * exp(-(dx * dx + dy * dy) / (radius * radius));
  }
}

// Deterministic sum of a member's interior solution: per-block partial sums
// in a fixed tree order, then one block over the partials in index order.
constexpr int CS_THREADS = 256, CS_BLOCKS = 256;
__global__ void k_checksum_partial(DevParams P, const double* __restrict__ u, double* __restrict__ part) {
  __shared__ double sh[CS_THREADS];
  const long long n = (long long)P.N0 * P.N1 * P.nvars;
  double acc = 0.0;
  for (long long e = blockIdx.x * (long long)CS_THREADS + threadIdx.x; e < n; e += (long long)CS_BLOCKS * CS_THREADS) {
    const long long pt = e / P.nvars;
    const int v = (int)(e - pt * P.nvars);
    acc += u[v * P.ps + pidx(P, (int)(pt % P.N0), (int)(pt / P.N0))];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = CS_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_checksum_final(const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < CS_BLOCKS; b++) s += part[b];
    *out = s;
  }
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

// Launch configurations the tuner chooses from: 2D tile shape, threads per
// CTA (also the points of a 1D tile) and the CTAs per SM the compiler is
// asked to fit; 256-thread tiles are small enough for two CTAs per SM.
struct TileShape { int tx, ty, nt, minb; };
constexpr int kNumShapes = 5;
constexpr TileShape kShapes[kNumShapes] = {
    {16, 16, 512, 1}, {32, 8, 512, 1}, {16, 8, 256, 2}, {32, 4, 256, 2}, {8, 16, 256, 2}};

template <int TX, int TY, int NT, int MINB>
struct StageOps {
  static long long smem(int nv) {
    return std::max(smem2d<TX, TY>(nv), smem1d<NT>(nv)) * (long long)sizeof(double);
  }
  static cudaError_t attr(long long bytes) {
    return cudaFuncSetAttribute(k_batch_stage<TX, TY, NT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes);
  }
  static int per_sm(long long bytes) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<TX, TY, NT, MINB>, NT, bytes) != cudaSuccess)
      n = 0;
    return n;
  }
  static void launch(int grid, long long bytes, cudaStream_t st, const BMember* m, const BState* s, const int* tl,
                     const int* nt, int stage) {
    k_batch_stage<TX, TY, NT, MINB><<<grid, NT, bytes, st>>>(m, s, tl, nt, stage);
  }
};
#define PIAFS_SHAPE_SWITCH(idx, CALL)                              \
  switch (idx) {                                                   \
    case 0: { typedef StageOps<16, 16, 512, 1> Ops; CALL; } break; \
    case 1: { typedef StageOps<32, 8, 512, 1> Ops; CALL; } break;  \
    case 2: { typedef StageOps<16, 8, 256, 2> Ops; CALL; } break;  \
    case 3: { typedef StageOps<32, 4, 256, 2> Ops; CALL; } break;  \
    default: { typedef StageOps<8, 16, 256, 2> Ops; CALL; } break; \
  }

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
  long long r = 0;
  PIAFS_SHAPE_SWITCH(shape, r = Ops::smem(nv));
  return r;
}

int persistent_grid(piafs_gpu_batch* B) {
  // PIAFS_GPU_BATCH_GRID=n overrides the number of persistent CTAs
  if (const char* g = std::getenv("PIAFS_GPU_BATCH_GRID")) {
    const int n = std::atoi(g);
    if (n > 0) return n;
  }
  const long long sm = smem_bytes(B->shape, std::max(B->max_nv, 1));
  int per_sm = 0;
  PIAFS_SHAPE_SWITCH(B->shape, per_sm = Ops::per_sm(sm));
  if (per_sm < 1) per_sm = 1;
  return per_sm * B->num_sms;
}

// tiles of a member under the current shape
void member_tiles(const piafs_gpu_batch* B, BMember& m) {
  const TileShape ts = kShapes[B->shape];
  if (m.P.ndims == 2) { m.tnx = (m.P.N0 + ts.tx - 1) / ts.tx; m.tny = (m.P.N1 + ts.ty - 1) / ts.ty; }
  else { m.tnx = (m.P.N0 + ts.nt - 1) / ts.nt; m.tny = 1; }
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
  {
    cudaError_t ea = cudaSuccess;
    PIAFS_SHAPE_SWITCH(B->shape, ea = Ops::attr(sm));
    BCK(ea);
  }
  cudaGraph_t g;
  BCK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < B->max_stages && e == cudaSuccess; s++) {
    PIAFS_SHAPE_SWITCH(B->shape, Ops::launch(grid, sm, B->stream, B->dmem, B->dstate, B->dtiles, B->dntiles, s));
    e = cudaGetLastError();
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

namespace {
// Parse and check one member's deck (host only; safe to run in parallel).
int parse_member(const char* deck_dir, HostMember& hm, DevParams& P, std::string& err) {
  int r = read_deck(deck_dir, hm.deck, err);
  if (!r) r = make_params(hm.deck, P, err);
  if (r) return r;
  if (P.scheme != WENO5) { err = "batched members use hyp_space_scheme weno5"; return PIAFS_ERR_UNSUPPORTED; }
  if (!((P.ndims == 2 && P.model == NS2D) || (P.ndims == 1 && P.model == EULER1D && !P.chem))) {
    err = "batched members are 2D navierstokes2d or 1D euler1d without chemistry";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (P.nvars > 32) { err = "batched members have at most 32 variables"; return PIAFS_ERR_UNSUPPORTED; }
  return 0;
}
}  // namespace

namespace {
int admit_member(piafs_gpu_batch* B, HostMember&& hm, DevParams P, int nsteps, int* id,
                 const piafs_gpu_request* req = nullptr) {
  const Deck& d = hm.deck;
  {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, B->device);
    if (smem_bytes(B->shape, std::max(B->max_nv, P.nvars)) > optin)
      return nfail(PIAFS_ERR_UNSUPPORTED, "too many variables for the batched stage kernel's shared-memory tile");
  }
  P.mixed = 0;
  const int ns = d.nstages;
  const size_t planes = (size_t)P.nvars * P.ps;
  const size_t ndx = d.dxinv.size(), nim = req ? (P.chem ? (size_t)P.npg : 0) : d.imap.size();
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
  // entries of the stage buffers must hold what the state's ghosts hold);
  // a request's fields are generated on the device instead
  double* stage = nullptr;
  if (req) {
    e = cudaMemsetAsync(u, 0, planes * sizeof(double), B->stream);
    if (e == cudaSuccess && nim) e = cudaMemsetAsync(im, 0, nim * sizeof(double), B->stream);
    if (e == cudaSuccess) {
      const long long npt = (long long)P.N0 * P.N1;
      k_request_init<<<(unsigned)((npt + 255) / 256), 256, 0, B->stream>>>(
          P, req->kind, req->amp, req->beam_radius, req->noise, req->seed, u, nim ? im : nullptr);
      e = cudaGetLastError();
    }
  } else {
    e = cudaMallocAsync((void**)&stage, d.u0.size() * sizeof(double), B->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(stage, d.u0.data(), d.u0.size() * sizeof(double), cudaMemcpyHostToDevice, B->stream);
    if (e == cudaSuccess) { launch_aos_to_soa(stage, u, P.npg, P.nvars, P.ps, B->stream); e = cudaGetLastError(); }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(bm.X, u, planes * sizeof(double), cudaMemcpyDeviceToDevice, B->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(bm.Y, u, planes * sizeof(double), cudaMemcpyDeviceToDevice, B->stream);
  for (int k = 0; k < ns && e == cudaSuccess; k++) e = cudaMemsetAsync(bm.k[k], 0, planes * sizeof(double), B->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dx, d.dxinv.data(), ndx * sizeof(double), cudaMemcpyHostToDevice, B->stream);
  if (e == cudaSuccess && nim && !req)
    e = cudaMemcpyAsync(im, d.imap.data(), nim * sizeof(double), cudaMemcpyHostToDevice, B->stream);
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
}  // namespace

namespace {

std::string fmt17(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

// The in-memory deck of a request: the key files the package's case
// generators write for the same parameters (cases.euler1d_density_wave,
// cases.ns2d_photochem_beam) and the interior grid.
int request_deck(const piafs_gpu_request& q, DeckMemory& m, std::string& err) {
  if (q.n < 8 || q.nsteps < 1 || !(q.dt > 0.0)) { err = "request: bad size, step count or dt"; return PIAFS_ERR_ARGUMENT; }
  const std::string n = std::to_string(q.n), ns = std::to_string(q.nsteps);
  if (q.kind == PIAFS_REQUEST_EULER1D_WAVE) {
    m.files["solver.inp"] =
        "begin\n ndims 1\n nvars 3\n size " + n + "\n ghost 3\n n_iter " + ns +
        "\n time_scheme rk\n time_scheme_type ssprk3\n hyp_space_scheme weno5\n hyp_interp_type components\n"
        " dt " + fmt17(q.dt) + "\n screen_op_iter " + ns + "\n file_op_iter " + ns +
        "\n op_file_format none\n ip_file_type binary\n op_overwrite no\n model euler1d\nend\n";
    m.files["boundary.inp"] = "2\nperiodic 0 1 0 0\nperiodic 0 -1 0 0\n";
    m.files["physics.inp"] = "begin\n gamma 1.4\n upwinding roe\nend\n";
    m.grid.resize(q.n);
    for (int i = 0; i < q.n; i++) m.grid[i] = (double)i / q.n;
    return 0;
  }
  if (q.kind == PIAFS_REQUEST_NS2D_BEAM) {
    if (!(q.Re > 0.0) || !(q.beam_radius > 0.0)) { err = "request: Re and beam_radius must be positive"; return PIAFS_ERR_ARGUMENT; }
    // Re ~ 1/sin(theta): theta = 4.2117e-5 rad gives Re = 1e4
    const double s = std::sin(4.2117e-5) * 1e4 / q.Re;
    const double theta = std::asin(s < 1.0 ? s : 1.0);
    m.files["solver.inp"] =
        "begin\n ndims 2\n nvars 11\n size " + n + " " + n + "\n ghost 3\n n_iter " + ns +
        "\n time_scheme rk\n time_scheme_type ssprk3\n hyp_space_scheme weno5\n hyp_interp_type components\n"
        " par_space_scheme 2\n dt " + fmt17(q.dt) + "\n screen_op_iter " + ns + "\n file_op_iter " + ns +
        "\n op_file_format none\n ip_file_type binary\n op_overwrite no\n model navierstokes2d\nend\n";
    m.files["boundary.inp"] =
        "4\nperiodic 0 1 0 0 -1e+99 1e+99\nperiodic 0 -1 0 0 -1e+99 1e+99\n"
        "slip-wall 1 1 -1e+99 1e+99 0 0\n 0 0\nslip-wall 1 -1 -1e+99 1e+99 0 0\n 0 0\n";
    m.files["physics.inp"] = "begin\n gamma 1.4\n upwinding llf-char\n Pr 0.72\n Re " + fmt17(q.Re) +
                             "\n include_chemistry yes\n write_output no\nend\n";
    m.files["chemistry.inp"] = "begin\n theta " + fmt17(theta) + "\nend\n";
    m.grid.resize(2 * (size_t)q.n);
    for (int i = 0; i < q.n; i++) m.grid[i] = m.grid[q.n + i] = (i + 0.5) / q.n;
    return 0;
  }
  err = "request: unknown kind";
  return PIAFS_ERR_ARGUMENT;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
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
  DevParams P;
  std::string err;
  if (int r = parse_member(deck_dir, hm, P, err)) return nfail(r, err);
  return admit_member(B, std::move(hm), P, nsteps, id);
}

int piafs_gpu_batch_add_many(piafs_gpu_batch* B, const char* const* deck_dirs, int n, const int* nsteps, int* ids,
                             int* n_added) {
  if (!B || (n > 0 && (!deck_dirs || !ids)) || n < 0 || !n_added) return nfail(PIAFS_ERR_ARGUMENT, "bad argument");
  *n_added = 0;
  std::vector<HostMember> hms(n);
  std::vector<DevParams> Ps(n);
  std::vector<std::string> errs(n);
  std::vector<int> rcs(n, 0);
  // decks are parsed by a pool of host threads, then admitted in order
  const int nt = std::max(1, std::min<int>(n, (int)std::thread::hardware_concurrency()));
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int w = 0; w < nt; w++)
    pool.emplace_back([&]() {
      for (int k = next++; k < n; k = next++) rcs[k] = parse_member(deck_dirs[k], hms[k], Ps[k], errs[k]);
    });
  for (auto& th : pool) th.join();
  for (int k = 0; k < n; k++) {
    if (rcs[k]) return nfail(rcs[k], std::string(deck_dirs[k]) + ": " + errs[k]);
    if (int r = admit_member(B, std::move(hms[k]), Ps[k], nsteps ? nsteps[k] : 0, ids + k)) return r;
    *n_added = k + 1;
  }
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

int piafs_gpu_batch_get_buffer(piafs_gpu_batch* B, int id, int which, double* out) {
  if (!B || !out || id < 0 || id >= (int)B->members.size() || !B->members[id].used || which < 0 || which > 2)
    return nfail(PIAFS_ERR_ARGUMENT, "bad argument");
  const BMember& bm = B->members[id].bm;
  BState st;
  BCK(cudaMemcpyAsync(&st, B->dstate + id, sizeof(BState), cudaMemcpyDeviceToHost, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  const double* src = which == 0 ? st.u : which == 1 ? bm.X : bm.Y;
  const DevParams& P = bm.P;
  double* tmp = nullptr;
  const size_t n = (size_t)P.npg * P.nvars;
  BCK(cudaMallocAsync((void**)&tmp, n * sizeof(double), B->stream));
  launch_soa_to_aos(src, tmp, P.npg, P.nvars, P.ps, B->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, B->stream);
  cudaFreeAsync(tmp, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("buffer: ") + cudaGetErrorString(e));
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
  info->min_ctas_per_sm = kShapes[B->shape].minb;
  return PIAFS_OK;
}

int piafs_gpu_batch_tune(piafs_gpu_batch* B, int force_tile_x) {
  if (!B) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  if (force_tile_x) {
    int k = -1;
    for (int i = 0; i < kNumShapes && k < 0; i++)
      if (kShapes[i].tx == force_tile_x) k = i;
    if (k < 0) return nfail(PIAFS_ERR_ARGUMENT, "tile_x must be 32, 16 or 64");
    B->shape = k;
    B->dirty = true;
    return PIAFS_OK;
  }
  // Time every launch configuration on the current members (one warm-up
  // step, then two timed steps each) and keep the fastest.  The members'
  // solution, clocks and step counts are saved before and restored after
  // every trial, so tuning leaves the batch as it found it.
  if (B->dirty) if (int r = sync_tables(B)) return r;
  if (B->ntiles == 0) return PIAFS_OK;
  std::vector<BState> saved(B->cap);
  BCK(cudaMemcpyAsync(saved.data(), B->dstate, (size_t)B->cap * sizeof(BState), cudaMemcpyDeviceToHost, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  std::vector<std::pair<double*, size_t>> copies;   // (device copy, doubles) per member slot
  copies.resize(B->members.size(), {nullptr, 0});
  cudaError_t e = cudaSuccess;
  for (size_t i = 0; i < B->members.size() && e == cudaSuccess; i++) {
    const HostMember& hm = B->members[i];
    if (!hm.used) continue;
    const size_t n = (size_t)hm.bm.P.nvars * hm.bm.P.ps;
    e = cudaMallocAsync((void**)&copies[i].first, n * sizeof(double), B->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(copies[i].first, saved[i].u, n * sizeof(double), cudaMemcpyDeviceToDevice, B->stream);
    copies[i].second = n;
  }
  auto restore = [&]() -> cudaError_t {
    cudaError_t r = cudaSuccess;
    for (size_t i = 0; i < copies.size() && r == cudaSuccess; i++)
      if (copies[i].first)
        r = cudaMemcpyAsync(saved[i].u, copies[i].first, copies[i].second * sizeof(double),
                            cudaMemcpyDeviceToDevice, B->stream);
    if (r == cudaSuccess)
      r = cudaMemcpyAsync(B->dstate, saved.data(), (size_t)B->cap * sizeof(BState), cudaMemcpyHostToDevice,
                          B->stream);
    if (r == cudaSuccess) r = cudaStreamSynchronize(B->stream);
    return r;
  };
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, B->device);
  const int keep = B->shape;
  int best = keep;
  float best_ms = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  for (int c = 0; c < kNumShapes && e == cudaSuccess; c++) {
    if (smem_bytes(c, B->max_nv) > optin) continue;
    B->shape = c;
    B->dirty = true;
    if (int r = sync_tables(B)) { e = cudaErrorUnknown; (void)r; break; }
    if (int r = capture_graph(B)) { e = cudaErrorUnknown; (void)r; break; }
    e = cudaGraphLaunch(B->graph, B->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e0, B->stream);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) e = cudaGraphLaunch(B->graph, B->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e1, B->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && ms < best_ms) { best_ms = ms; best = c; }
    if (e == cudaSuccess) e = restore();
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  for (auto& cp : copies)
    if (cp.first) cudaFreeAsync(cp.first, B->stream);
  cudaStreamSynchronize(B->stream);
  B->shape = e == cudaSuccess ? best : keep;
  B->dirty = true;
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("tuning: ") + cudaGetErrorString(e));
  return sync_tables(B);
}

int piafs_gpu_batch_set_launch(piafs_gpu_batch* B, int tile_x, int tile_y, int minb) {
  if (!B) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  for (int i = 0; i < kNumShapes; i++)
    if (kShapes[i].tx == tile_x && kShapes[i].ty == tile_y && kShapes[i].minb == minb) {   // shapes are unique
      int optin = 0;
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, B->device);
      if (smem_bytes(i, B->max_nv) > optin)
        return nfail(PIAFS_ERR_UNSUPPORTED, "this tile does not fit the members' variables in shared memory");
      B->shape = i;
      B->dirty = true;
      return PIAFS_OK;
    }
  return nfail(PIAFS_ERR_ARGUMENT, "no such launch configuration");
}

int piafs_gpu_batch_add_request(piafs_gpu_batch* B, const piafs_gpu_request* req, int* id) {
  if (!B || !req || !id) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  DeckMemory mem;
  std::string err;
  if (int r = request_deck(*req, mem, err)) return nfail(r, err);
  HostMember hm;
  DevParams P;
  int r = read_deck_memory(mem, hm.deck, err);
  if (!r) r = make_params(hm.deck, P, err);
  if (r) return nfail(r, err);
  return admit_member(B, std::move(hm), P, req->nsteps, id, req);
}

int piafs_gpu_batch_checksum(piafs_gpu_batch* B, int id, double* sum) {
  if (!B || !sum || id < 0 || id >= (int)B->members.size() || !B->members[id].used)
    return nfail(PIAFS_ERR_ARGUMENT, "no such member");
  const DevParams& P = B->members[id].bm.P;
  BState st;
  BCK(cudaMemcpyAsync(&st, B->dstate + id, sizeof(BState), cudaMemcpyDeviceToHost, B->stream));
  double* part = nullptr;
  BCK(cudaMallocAsync((void**)&part, (CS_BLOCKS + 1) * sizeof(double), B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  k_checksum_partial<<<CS_BLOCKS, CS_THREADS, 0, B->stream>>>(P, st.u, part);
  k_checksum_final<<<1, 32, 0, B->stream>>>(part, part + CS_BLOCKS);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(sum, part + CS_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, B->stream);
  cudaFreeAsync(part, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("checksum: ") + cudaGetErrorString(e));
  return PIAFS_OK;
}

int piafs_gpu_serve_trace(const piafs_gpu_request* reqs, const double* arrival_s, int n, int precision,
                          unsigned long long budget, int steps_per_round, piafs_gpu_serve_result* out) {
  if (n < 0 || (n > 0 && (!reqs || !arrival_s || !out)) || steps_per_round < 1)
    return nfail(PIAFS_ERR_ARGUMENT, "bad argument");
  for (int k = 1; k < n; k++)
    if (arrival_s[k] < arrival_s[k - 1]) return nfail(PIAFS_ERR_ARGUMENT, "arrival times must be nondecreasing");
  piafs_gpu_batch* B = nullptr;
  if (int r = piafs_gpu_batch_create(precision, budget, &B)) return r;
  std::vector<int> slot_req;     // member id -> request index
  int next = 0, finished = 0, rc = PIAFS_OK;
  const double t0 = now_s();
  for (int k = 0; k < n; k++) {
    out[k].arrival_s = arrival_s[k];
    out[k].admitted_s = out[k].finished_s = -1.0;
    out[k].steps = 0;
    out[k].checksum = 0.0;
  }
  std::vector<int> done(4096);
  while (finished < n && rc == PIAFS_OK) {
    // admission: arrived requests in order, while the budget holds them
    double t = now_s() - t0;
    while (next < n && arrival_s[next] <= t) {
      int id = -1;
      const int r = piafs_gpu_batch_add_request(B, reqs + next, &id);
      if (r == PIAFS_ERR_MEMORY) {
        piafs_gpu_batch_info bi;
        if ((rc = piafs_gpu_batch_get_info(B, &bi))) break;
        if (bi.members == 0)   // alone it does not fit: it never will
          rc = nfail(PIAFS_ERR_MEMORY, "a request needs more device memory than the whole HBM budget");
        break;
      }
      if (r) { rc = r; break; }
      if ((int)slot_req.size() <= id) slot_req.resize(id + 1, -1);
      slot_req[id] = next;
      out[next].admitted_s = now_s() - t0;
      next++;
      t = now_s() - t0;
    }
    if (rc) break;
    piafs_gpu_batch_info info;
    if ((rc = piafs_gpu_batch_get_info(B, &info))) break;
    if (info.active > 0) {
      if ((rc = piafs_gpu_batch_step(B, steps_per_round))) break;
    } else if (info.members == 0) {
      if (next >= n) break;
      // nothing resident: wait for the next arrival
      std::this_thread::sleep_for(std::chrono::duration<double>(std::min(std::max(arrival_s[next] - t, 0.0), 1e-3)));
      continue;
    }
    // retire finished requests
    int nd = 0;
    if ((rc = piafs_gpu_batch_poll(B, done.data(), (int)done.size(), &nd))) break;
    for (int q = 0; q < nd && rc == PIAFS_OK; q++) {
      const int id = done[q], k = slot_req[id];
      double cs = 0.0, tm = 0.0;
      int it = 0, dn = 0;
      rc = piafs_gpu_batch_checksum(B, id, &cs);
      if (!rc) rc = piafs_gpu_batch_member(B, id, &tm, &it, &dn);
      if (!rc) rc = piafs_gpu_batch_remove(B, id);
      out[k].checksum = cs;
      out[k].steps = it;
      out[k].finished_s = now_s() - t0;
      finished++;
    }
  }
  piafs_gpu_batch_destroy(B);
  return rc;
}

}  // extern "C"
