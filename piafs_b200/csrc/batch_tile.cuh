// Device side of the batched stage kernel (see batch.cu for the engine).
//
// One persistent kernel per Runge-Kutta stage walks a device list of tiles
// (tile -> member).  For each tile a CTA
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
// The FP64 expressions are those of the single-simulation kernels.  MX
// (mixed precision) follows the single-simulation mixed path: the state,
// the cell fluxes and the Runge-Kutta combination stay FP64; the WENO
// weights and values, the upwind fluxes (deviation form), the viscous
// stencils and the chemistry source are FP32.  Values enter FP32 relative to
// a reference of the tile (the state and fluxes at its first interior cell,
// subtracted in FP64; 1D: the tile's first cell), so the O(1) background never
// goes through FP32 rounding; the divergence differences the interface fluxes
// along grid lines of the tile, where the reference cancels.
#pragma once
#include <type_traits>

#include "kernels.h"
#include "physics.cuh"
#include "source.cuh"

namespace piafs {
namespace batch {

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

// Launch configurations the tuner chooses from: 2D tile shape, threads per
// CTA (also the points of a 1D tile) and the CTAs per SM the compiler is
// asked to fit.  The 15- and 7-row tiles have at most as many interfaces as
// threads (16x15: 255 + 256 = 511 for 512 threads; 32x7: 231 + 256; 16x7:
// 119 + 128 for 256), so the per-interface phases run in one round.
struct TileShape { int tx, ty, nt, minb; };
constexpr int kNumShapes = 8;
constexpr TileShape kShapes[kNumShapes] = {{16, 16, 512, 1}, {32, 8, 512, 1}, {16, 8, 256, 2}, {32, 4, 256, 2},
                                           {8, 16, 256, 2},  {16, 15, 512, 1}, {32, 7, 512, 1}, {16, 7, 256, 2}};

__host__ __device__ constexpr long long al16(long long b) { return (b + 15) / 16 * 16; }

#ifdef __CUDACC__
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
  // six loads in flight before their stores (the stores could alias S as far
  // as the compiler knows, which would serialise the loads)
  const long long ps = P.ps;
  for (int v0 = 0; v0 < nv; v0 += 6) {
    const double* q = S + v0 * ps + p;
    double* o = out + v0 * ostride;
    const int r = nv - v0;
    const double a0 = q[0], a1 = r > 1 ? q[ps] : 0.0, a2 = r > 2 ? q[2 * ps] : 0.0;
    const double a3 = r > 3 ? q[3 * ps] : 0.0, a4 = r > 4 ? q[4 * ps] : 0.0, a5 = r > 5 ? q[5 * ps] : 0.0;
    o[0] = a0;
    if (r > 1) o[ostride] = a1;
    if (r > 2) o[2 * ostride] = a2;
    if (r > 3) o[3 * ostride] = a3;
    if (r > 4) o[4 * ostride] = a4;
    if (r > 5) o[5 * ostride] = a5;
  }
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
// and its flux at f[(r-3)*fst] for the cells r = 0..5 (i-3..i+2); MX: taken
// relative to ur / fr in FP64, then reconstructed in FP32.
template <bool MX>
__device__ __forceinline__ void iface_weno(const DevParams& P, const double* u, int ust, const double* f, int fst,
                                           double ur, double fr, typename std::conditional<MX, float, double>::type& uL,
                                           typename std::conditional<MX, float, double>::type& uR,
                                           typename std::conditional<MX, float, double>::type& fL,
                                           typename std::conditional<MX, float, double>::type& fR) {
  typedef typename std::conditional<MX, float, double>::type T;
  T a[6], b[6];
#pragma unroll
  for (int r = 0; r < 6; r++) {
    if (MX) { a[r] = (T)(u[(r - 3) * ust] - ur); b[r] = (T)(f[(r - 3) * fst] - fr); }
    else { a[r] = u[(r - 3) * ust]; b[r] = f[(r - 3) * fst]; }
  }
  weno5_iface(P, a, b, uL, uR, fL, fR);
}

// Characteristic / scalar upwinding of the flow variables at one interface
// from their WENO values rec[k * ks + m * ms] (k: uL, uR, fL, fR) and the cell
// states left / right (ucl, ucr at stride vs); flux to so[m * sstride],
// passive-variable scheme data to *spa / *spm.  MX: rec holds FP32 values
// relative to the reference state uref (stride vs), and the flux comes back
// relative to the reference flux (upwind_flow_dev).
template <int MODEL, int UPW, bool MX>
__device__ __noinline__ void iface_upwind_flow(const DevParams& P,
                                               const typename std::conditional<MX, float, double>::type* rec, int ks,
                                               int ms, const double* ucl, const double* ucr, const double* uref,
                                               int vs, int dir, typename std::conditional<MX, float, double>::type* so,
                                               int sstride, typename std::conditional<MX, float, double>::type* spa,
                                               int* spm) {
  typedef typename std::conditional<MX, float, double>::type T;
  constexpr int NF = Flow<MODEL>::NF;
  T uL[4], uR[4], fL[4], fR[4], cl[4], cr[4], fi[4];
#pragma unroll
  for (int m = 0; m < NF; m++) {
    uL[m] = rec[m * ms]; uR[m] = rec[ks + m * ms]; fL[m] = rec[2 * ks + m * ms]; fR[m] = rec[3 * ks + m * ms];
    cl[m] = (T)ucl[m * vs]; cr[m] = (T)ucr[m * vs];
  }
  if (MX) {
    T aL[4], aR[4];
    if (MODEL == NS2D && (UPW == UPW_LLF || UPW == UPW_RF)) {
#pragma unroll
      for (int m = 0; m < NF; m++) { const T r = (T)uref[m * vs]; aL[m] = r + uL[m]; aR[m] = r + uR[m]; }
      upwind_flow_dev<MODEL, UPW, T>(uL, uR, fL, fR, aL, aR, cl, cr, (T)P.gamma, dir, fi, spa, spm);
    } else {
      upwind_flow_dev<MODEL, UPW, T>(uL, uR, fL, fR, uL, uR, cl, cr, (T)P.gamma, dir, fi, spa, spm);
    }
  } else {
    upwind_flow<MODEL, UPW, T>(uL, uR, fL, fR, cl, cr, (T)P.gamma, dir, fi, spa, spm);
  }
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
#endif  // __CUDACC__

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
// Interfaces are numbered x first (f < NXI: row jj, position ii) then y
// (row jj, column ii), x fastest in both.
// Shared memory (bytes, regions 16-byte aligned): sU [nv][HY][HX] (FP64);
// interface fluxes fx [nv][TY][TX+1] and fy [nv][TY+1][TX] (T); a work
// region, reused by the viscous phase: cell data, WENO values [4][4][NI] (T),
// passive speed (T) and scheme (int) [NI] each.  T is FP64, or FP32 under MX.
// FP64 cell data: 4 flow fluxes and vn, [5][TY][HX] for x cells and
// [5][HY][TX] for y cells.  MX: the state and every cell flux (flow fluxes and
// the passive fluxes vn u_m) enter FP32 once per cell, relative to the tile's
// reference values (state, x and y fluxes at the tile's first interior cell,
// subtracted in FP64): state deviations [nv][HY][HX] and flux deviations
// [nv][TY][HX] + [nv][HY][TX].  A per-tile constant is constant along every
// grid line of the tile, so reconstruction and upwinding are unchanged by it
// and the divergence cancels it.
template <int TX, int TY, bool MX>
struct Tile2D {
  typedef typename std::conditional<MX, float, double>::type T;
  static constexpr int HX = TX + 6, HY = TY + 6;
  static constexpr int NXI = TY * (TX + 1), NYI = TX * (TY + 1), NI = NXI + NYI;
  static constexpr int NCX = TY * HX, NCY = TX * HY;            // stencil cells per direction
  static constexpr long long VISC =
      al16((3LL * (TY + 2) * (TX + 2) + 3LL * TY * (TX + 1) + 3LL * (TY + 1) * TX) * (long long)sizeof(T));
  static constexpr long long REC = al16(16LL * NI * (long long)sizeof(T));
  static constexpr long long SPA = al16((long long)NI * (long long)sizeof(T));
  // work region: [MX: FP32 state deviations] cell data, WENO values, passive
  // speed and scheme
  __host__ __device__ static constexpr long long suf_bytes(int nv) { return MX ? al16(4LL * nv * HX * HY) : 0; }
  __host__ __device__ static constexpr long long cell_bytes(int nv) {
    return MX ? al16(4LL * nv * (NCX + NCY)) : al16(5LL * (NCX + NCY) * 8);
  }
  __host__ __device__ static constexpr long long work(int nv) {
    return suf_bytes(nv) + cell_bytes(nv) + REC + SPA + al16(4LL * NI) > VISC
               ? suf_bytes(nv) + cell_bytes(nv) + REC + SPA + al16(4LL * NI)
               : VISC;
  }
  __host__ __device__ static constexpr long long su_bytes(int nv) { return al16((long long)nv * HX * HY * 8); }
  __host__ __device__ static constexpr long long fx_bytes(int nv) { return al16((long long)nv * NXI * sizeof(T)); }
  __host__ __device__ static constexpr long long fy_bytes(int nv) { return al16((long long)nv * NYI * sizeof(T)); }
  __host__ __device__ static constexpr long long smem(int nv) {
    return su_bytes(nv) + fx_bytes(nv) + fy_bytes(nv) + work(nv);
  }
};

// ------------------------------------------------------------- 1D tile
// A 1D tile has T1 points, one per thread.  Shared memory (bytes): sU and
// the cell fluxes [nv][T1+6] (FP64), interface fluxes [nv][T1+1] (T), flow
// WENO values [4][3][T1+1] (T), passive speed (T) and scheme (int).
template <int T1, bool MX>
struct Tile1D {
  typedef typename std::conditional<MX, float, double>::type T;
  static constexpr int HX = T1 + 2 * H, LX = T1 + 1;
  __host__ __device__ static constexpr long long smem(int nv) {
    return al16(2LL * nv * HX * 8) + al16((long long)nv * LX * sizeof(T)) + al16(12LL * LX * sizeof(T)) +
           al16((long long)LX * sizeof(T)) + al16(4LL * LX);
  }
};

#ifdef __CUDACC__
// photochemical source of one layer at a point whose state is u[v * us]
// (shared memory), added to the point's stage derivative kv[] in registers
// (the arithmetic and the order of chem_source_point for nz = 1)
template <typename T>
__device__ __forceinline__ void chem_source_kv(const DevParams& P, const double* u, int us, double hnu_factor,
                                               double imap_p, double* kv) {
  T src[5], Q;
  chem_layer<T>(P, chem_hnu0<T>(P, hnu_factor, imap_p), (T)u[4 * us], (T)u[5 * us], (T)u[6 * us], (T)u[7 * us],
                (T)u[8 * us], (T)u[9 * us], (T)u[10 * us], src, Q);
#pragma unroll
  for (int k = 0; k < 5; k++) kv[5 + k] += (double)src[k];
  kv[3] += (double)Q;
}

template <int TX, int TY, int UPW, int BT, bool MX>
__device__ __forceinline__ void tile2d(const BMember& M, const BState& Sd, int s, int tx, int ty, char* smem) {
  typedef Tile2D<TX, TY, MX> L;
  typedef typename L::T T;
  constexpr int HX = L::HX, HY = L::HY, NXI = L::NXI, NYI = L::NYI, NI = L::NI, NCX = L::NCX, NCY = L::NCY;
  const DevParams& P = M.P;
  const int nv = P.nvars, N0 = P.N0, N1 = P.N1;
  const int i0 = tx * TX, j0 = ty * TY;
  const double* S = s == 0 ? Sd.u : ((s - 1) % 2 == 0 ? M.X : M.Y);
  constexpr int vs = HX * HY;
  double* sU = (double*)smem;
  T* fx = (T*)(smem + L::su_bytes(nv));                  // [m][jj * (TX+1) + ii]
  T* fy = (T*)((char*)fx + L::fx_bytes(nv));             // [m][jj * TX + ii]
  char* wk = (char*)fy + L::fy_bytes(nv);                // work region
  float* sUf = (float*)wk;                               // MX: [nv][HY][HX] state deviations
  char* cw = wk + L::suf_bytes(nv);
  double* cx = (double*)cw;                              // FP64: [5][NCX]: 4 flow fluxes + vn, x cells [jj][a]
  double* cy = cx + 5 * NCX;                             // FP64: [5][NCY]: y cells [b][ii]
  float* cxf = (float*)cw;                               // MX: [nv][NCX] flux deviations, x cells
  float* cyf = cxf + nv * NCX;                           // MX: [nv][NCY], y cells
  T* rec = (T*)(cw + L::cell_bytes(nv));                 // [k][m][NI]
  T* spa = (T*)((char*)rec + L::REC);                    // [NI]
  int* spm = (int*)((char*)spa + L::SPA);                // [NI]
  const int tid = threadIdx.x;
  constexpr int c0 = H * HX + H;                         // the tile's first interior cell
  for (int e = tid; e < vs; e += BT) load_point(M, S, i0 - H + e % HX, j0 - H + e / HX, sU + e, vs);
  __syncthreads();
  // cell data: x cells (row jj, column a): c = (jj+H)*HX + a, index jj*HX + a;
  // y cells (row b, column ii): c = b*HX + ii + H, index b*TX + ii
  if constexpr (MX) {
    double fr0[4], fr1[4], vr0, vr1;                     // reference fluxes (x, y) at c0
    ns2d_flux(sU[c0], sU[vs + c0], sU[2 * vs + c0], sU[3 * vs + c0], P.gamma, 0, fr0, vr0);
    ns2d_flux(sU[c0], sU[vs + c0], sU[2 * vs + c0], sU[3 * vs + c0], P.gamma, 1, fr1, vr1);
    for (int e = tid; e < nv * vs; e += BT) sUf[e] = (float)(sU[e] - sU[(e / vs) * vs + c0]);
    for (int e = tid; e < NCX + NCY; e += BT) {
      const bool xd = e < NCX;
      const int g = xd ? e : e - NCX;
      const int c = xd ? (g / HX + H) * HX + g % HX : (g / TX) * HX + g % TX + H;
      double f[4], vn;
      ns2d_flux(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, xd ? 0 : 1, f, vn);
      float* o = xd ? cxf + g : cyf + g;
      const int st = xd ? NCX : NCY;
      const double* fr = xd ? fr0 : fr1;
      const double vr = xd ? vr0 : vr1;
#pragma unroll
      for (int m = 0; m < 4; m++) o[m * st] = (float)(f[m] - fr[m]);
      for (int m = 4; m < nv; m++)
        o[m * st] = (float)(__dmul_rn(vn, sU[m * vs + c]) - __dmul_rn(vr, sU[m * vs + c0]));
    }
  } else {
    for (int e = tid; e < NCX + NCY; e += BT) {
      const bool xd = e < NCX;
      const int g = xd ? e : e - NCX;
      const int c = xd ? (g / HX + H) * HX + g % HX : (g / TX) * HX + g % TX + H;
      double f[4], vn;
      ns2d_flux(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, xd ? 0 : 1, f, vn);
      double* o = xd ? cx + g : cy + g;
      const int st = xd ? NCX : NCY;
#pragma unroll
      for (int m = 0; m < 4; m++) o[m * st] = f[m];
      o[4 * st] = vn;
    }
  }
  __syncthreads();
  // geometry of interface f: its cell i (right of the interface) in sU
  // (base, stride ust along the line), in its direction's cell data (index
  // cdo, plane cst, stride cls along the line) and whether it is inside the
  // member.  Consecutive interfaces of either direction are consecutive in x,
  // so a warp's shared-memory accesses are unit-stride.
  auto geo = [&](int f, int& base, int& ust, int& cdo, int& cst, int& cls, int& dir) -> bool {
    if (f < NXI) {
      const int ii = f % (TX + 1), jj = f / (TX + 1);
      base = (jj + H) * HX + ii + H; ust = 1; cdo = jj * HX + ii + H; cst = NCX; cls = 1; dir = 0;
      return i0 + ii <= N0 && j0 + jj < N1;
    }
    const int g = f - NXI, ii = g % TX, jj = g / TX;
    base = (jj + H) * HX + ii + H; ust = HX; cdo = (jj + H) * TX + ii; cst = NCY; cls = TX; dir = 1;
    return j0 + jj <= N1 && i0 + ii < N0;
  };
  // a thread takes NW items at a time and finishes them together (their loads
  // and arithmetic are independent, so their latencies overlap); items past
  // the end or outside the member are computed on in-tile data and dropped
  constexpr int NW = 2;
  auto load_stencil = [&](int m, int base, int ust, int cdo, int cst, int cls, int dir, T* a, T* b) {
    if constexpr (MX) {
      const float* u = sUf + m * vs + base;
      const float* fc = (dir ? cyf : cxf) + m * cst + cdo;
#pragma unroll
      for (int r = 0; r < 6; r++) { a[r] = u[(r - 3) * ust]; b[r] = fc[(r - 3) * cls]; }
    } else {
      const double* u = sU + m * vs + base;
      if (m < 4) {
        const double* fc = (dir ? cy : cx) + m * cst + cdo;
#pragma unroll
        for (int r = 0; r < 6; r++) { a[r] = u[(r - 3) * ust]; b[r] = fc[(r - 3) * cls]; }
      } else {
        const double* vn = (dir ? cy : cx) + 4 * cst + cdo;
#pragma unroll
        for (int r = 0; r < 6; r++) { a[r] = u[(r - 3) * ust]; b[r] = __dmul_rn(vn[(r - 3) * cls], a[r]); }
      }
    }
  };
  for (int e0 = tid; e0 < 4 * NI; e0 += NW * BT) {
    T a[NW][6], b[NW][6], o[NW][4];
    int at[NW];
    bool ok[NW];
#pragma unroll
    for (int w = 0; w < NW; w++) {
      const int e = min(e0 + w * BT, 4 * NI - 1);
      const int m = e / NI, f = e % NI;
      int base, ust, cdo, cst, cls, dir;
      ok[w] = geo(f, base, ust, cdo, cst, cls, dir) && e0 + w * BT < 4 * NI;
      at[w] = m * NI + f;
      load_stencil(m, base, ust, cdo, cst, cls, dir, a[w], b[w]);
    }
    weno5_iface_n<NW, T>(P, a, b, o);
#pragma unroll
    for (int w = 0; w < NW; w++)
      if (ok[w]) {
        rec[at[w]] = o[w][0]; rec[at[w] + 4 * NI] = o[w][1]; rec[at[w] + 8 * NI] = o[w][2];
        rec[at[w] + 12 * NI] = o[w][3];
      }
  }
  __syncthreads();
  for (int f = tid; f < NI; f += BT) {
    int base, ust, cdo, cst, cls, dir;
    if (!geo(f, base, ust, cdo, cst, cls, dir)) continue;
    T* so = f < NXI ? fx + f : fy + (f - NXI);
    iface_upwind_flow<NS2D, UPW, MX>(P, rec + f, 4 * NI, NI, sU + base - ust, sU + base, sU + c0, vs, dir, so,
                                     f < NXI ? NXI : NYI, spa + f, spm + f);
  }
  __syncthreads();
  const int npi = (nv - 4) * NI;
  for (int e0 = tid; e0 < npi; e0 += NW * BT) {
    T a[NW][6], b[NW][6], o[NW][4];
    int fi[NW], mi[NW];
    bool ok[NW];
#pragma unroll
    for (int w = 0; w < NW; w++) {
      const int e = min(e0 + w * BT, npi - 1);
      const int m = 4 + e / NI, f = e % NI;
      int base, ust, cdo, cst, cls, dir;
      ok[w] = geo(f, base, ust, cdo, cst, cls, dir) && e0 + w * BT < npi;
      fi[w] = f; mi[w] = m;
      load_stencil(m, base, ust, cdo, cst, cls, dir, a[w], b[w]);
    }
    weno5_iface_n<NW, T>(P, a, b, o);
#pragma unroll
    for (int w = 0; w < NW; w++)
      if (ok[w]) {
        const int f = fi[w];
        const T h = upwind_species(spm[f], spa[f], o[w][0], o[w][1], o[w][2], o[w][3]);
        if (f < NXI) fx[mi[w] * NXI + f] = h;
        else fy[mi[w] * NYI + f - NXI] = h;
      }
  }
  __syncthreads();
  // viscous fluxes (k_visc_source on this tile), in the work region; MX:
  // temperature relative to the tile's first point
  const bool visc = P.viscous != 0;
  constexpr int QX = TX + 2, QY = TY + 2, FX = TX + 1, FY = TY + 1;
  T* sQ = (T*)wk;                               // [3][QY][QX]
  T* sVx = sQ + 3 * QY * QX;                    // [3][TY][FX]
  T* sVy = sVx + 3 * TY * FX;                   // [3][FY][TX]
  if (visc) {
    double Tref = 0.0;
    if (MX) {
      const int c = H * HX + H;
      double rho, uu, vv, e_, pr;
      ns_flowvar(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, rho, uu, vv, e_, pr);
      Tref = P.gamma * pr / rho;
    }
    for (int e = tid; e < QX * QY; e += BT) {
      const int a = e % QX, b = e / QX;
      const int i = i0 - 1 + a, j = j0 - 1 + b;
      double uu = 0.0, vv = 0.0, TT = Tref;
      const bool xin = i >= 0 && i < N0, yin = j >= 0 && j < N1;
      if ((xin || yin) && i >= -P.ghosts && i < N0 + P.ghosts && j >= -P.ghosts && j < N1 + P.ghosts) {
        const int c = (b - 1 + H) * HX + (a - 1 + H);
        double rho, e_, pr;
        ns_flowvar(sU[c], sU[vs + c], sU[2 * vs + c], sU[3 * vs + c], P.gamma, rho, uu, vv, e_, pr);
        TT = P.gamma * pr / rho;
      }
      sQ[e] = (T)uu; sQ[QX * QY + e] = (T)vv; sQ[2 * QX * QY + e] = (T)(TT - Tref);
    }
    __syncthreads();
    const T two_third = T(2.0 / 3.0), inv_Re = (T)(1.0 / P.Re), inv_Pr = (T)(1.0 / P.Pr);
    const T igm1 = (T)(1.0 / (P.gamma - 1.0));
    const T* su = sQ;
    const T* sv = sQ + QX * QY;
    const T* sT = sQ + 2 * QX * QY;
    for (int e = tid; e < FX * FY; e += BT) {
      const int a = e % FX, b = e / FX;
      const int i = i0 - 1 + a, j = j0 - 1 + b;
      const bool need_x = (b >= 1) && (j < N1) && (i < N0);
      const bool need_y = (a >= 1) && (i < N0) && (j < N1);
      if (!need_x && !need_y) continue;
      const int q = b * QX + a;
      const T dxi = (T)M.dxinv[P.ghosts + i], dyi = (T)M.dxinv[P.W0 + P.ghosts + j];
      const bool row_int = (j >= 0 && j < N1), col_int = (i >= 0 && i < N0);
      const T uc = su[q], vc = sv[q], Tc = sT[q];
      const T ux = row_int ? dxi * (su[q + 1] - uc) : T(0);
      const T vx = row_int ? dxi * (sv[q + 1] - vc) : T(0);
      const T Tx = row_int ? dxi * (sT[q + 1] - Tc) : T(0);
      const T uy = col_int ? dyi * (su[q + QX] - uc) : T(0);
      const T vy = col_int ? dyi * (sv[q + QX] - vc) : T(0);
      const T Ty = col_int ? dyi * (sT[q + QX] - Tc) : T(0);
      T mu, kappa;
      visc_coeffs<T>(P, MX ? (T)Tref + Tc : Tc, mu, kappa);
      const T mre = mu * inv_Re, kre = kappa * inv_Re * igm1 * inv_Pr;
      if (need_x) {
        const T txx = two_third * mre * (T(2) * ux - vy), txy = mre * (uy + vx);
        T* f = sVx + (b - 1) * FX + a;
        f[0] = txx; f[TY * FX] = txy; f[2 * TY * FX] = uc * txx + vc * txy + kre * Tx;
      }
      if (need_y) {
        const T tyx = mre * (uy + vx), tyy = two_third * mre * (-ux + T(2) * vy);
        T* f = sVy + b * TX + (a - 1);
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
  constexpr int LX = TX + 1;
  // the stage derivative of one variable: hyperbolic (and viscous) part
  auto hyp_visc = [&](int m) -> double {
    const T* ax = fx + m * NXI + pj * LX + pi;
    const T* ay = fy + m * NYI + pj * TX + pi;
    double h;
    if (MX) {
      const T hx = (T)dxi * (ax[1] - ax[0]), hy = (T)dyi * (ay[TX] - ay[0]);
      h = (double)(hx + hy);
    } else {
      const double hx = dxi * (ax[1] - ax[0]);
      const double hy = dyi * (ay[TX] - ay[0]);
      h = hx + hy;
    }
    double k = -h;
    if (visc && m >= 1 && m <= 3) {
      const int n = m - 1;
      if (MX) {
        const T par = (T)dxi * (sVx[n * TY * FX + pj * FX + pi + 1] - sVx[n * TY * FX + pj * FX + pi]) +
                      (T)dyi * (sVy[n * FY * TX + (pj + 1) * TX + pi] - sVy[n * FY * TX + pj * TX + pi]);
        k += (double)par;
      } else {
        const double par = dxi * (sVx[n * TY * FX + pj * FX + pi + 1] - sVx[n * TY * FX + pj * FX + pi]) +
                           dyi * (sVy[n * FY * TX + (pj + 1) * TX + pi] - sVy[n * FY * TX + pj * TX + pi]);
        k += par;
      }
    }
    return k;
  };
  const double t = Sd.t + M.c[s] * P.dt;
  // Every variable in registers (the common counts: NS2D with one chemistry
  // layer, 11, and without chemistry, 4): the earlier stages' part of the
  // Runge-Kutta combination first, all of its loads in flight together, then
  // this stage's derivative, then the stores.
  auto fast = [&](auto nvc) {
    constexpr int NV = decltype(nvc)::value;
    const int c = (pj + H) * HX + pi + H;                // the point's cell in sU
    const bool last = s == M.nstages - 1;
    double xa[NV], kv[NV];
#pragma unroll
    for (int m = 0; m < NV; m++) xa[m] = s == 0 ? sU[m * vs + c] : Sd.u[m * ps + p];
    for (int q = 0; q < s; q++) {
      const double cq = last ? M.b[q] : M.a[(s + 1) * MAX_STAGES + q];
      const double* kq = M.k[q] + p;
      double tq[NV];
#pragma unroll
      for (int m = 0; m < NV; m++) tq[m] = kq[m * ps];
#pragma unroll
      for (int m = 0; m < NV; m++) xa[m] += cq * tq[m];
    }
#pragma unroll
    for (int m = 0; m < NV; m++) kv[m] = hyp_visc(m);
    if (NV == 11) chem_source_kv<T>(P, sU + c, vs, pulse_factor(P, t), M.imap[p], kv);
    const double cs = last ? M.b[s] : M.a[(s + 1) * MAX_STAGES + s];
    double* dst = last ? (M.nstages == 1 ? Sd.X : Sd.u) : (s % 2 == 0 ? M.X : M.Y);
#pragma unroll
    for (int m = 0; m < NV; m++) { ks[m * ps + p] = kv[m]; dst[m * ps + p] = xa[m] + cs * kv[m]; }
  };
  if (nv == 11 && P.chem && P.nz == 1) { fast(std::integral_constant<int, 11>()); return; }
  if (nv == 4 && !P.chem) { fast(std::integral_constant<int, 4>()); return; }
  for (int m = 0; m < nv; m++) ks[m * ps + p] = hyp_visc(m);
  if (P.chem) chem_source_point<T>(P, S, p, pulse_factor(P, t), M.imap[p], ks);
  rk_point(M, Sd, s, p, nv);
}

template <int UPW, int BT, bool MX>
__device__ __forceinline__ void tile1d(const BMember& M, const BState& Sd, int s, int tx, char* smem) {
  typedef Tile1D<BT, MX> L;
  typedef typename L::T T;
  constexpr int T1 = BT, HX = L::HX, LX = L::LX, NF = 3;
  const DevParams& P = M.P;
  const int nv = P.nvars, N0 = P.N0;
  const int i0 = tx * T1;
  const double* S = s == 0 ? Sd.u : ((s - 1) % 2 == 0 ? M.X : M.Y);
  double* sU = (double*)smem;
  double* cf = sU + nv * HX;                            // [m][HX]
  T* sF = (T*)(smem + al16(2LL * nv * HX * 8));         // [m][LX]
  T* rec = (T*)((char*)sF + al16((long long)nv * LX * sizeof(T)));   // [k][m][LX]
  T* spa = (T*)((char*)rec + al16(12LL * LX * sizeof(T)));
  int* spm = (int*)((char*)spa + al16((long long)LX * sizeof(T)));
  const int tid = threadIdx.x;
  for (int e = tid; e < HX; e += BT) load_point(M, S, i0 - H + e, 0, sU + e, HX);
  __syncthreads();
  for (int e = tid; e < HX; e += BT) cell_flux<EULER1D>(P, sU, HX, e, 0, cf + e, HX);
  __syncthreads();
  // MX: the line's reference is the tile's first interior cell (index H)
  for (int e = tid; e < NF * LX; e += BT) {
    const int m = e / LX, f = e % LX;
    if (i0 + f > N0) continue;
    const double ur = MX ? sU[m * HX + H] : 0.0, fr = MX ? cf[m * HX + H] : 0.0;
    iface_weno<MX>(P, sU + m * HX + f + H, 1, cf + m * HX + f + H, 1, ur, fr, rec[(0 * NF + m) * LX + f],
                   rec[(1 * NF + m) * LX + f], rec[(2 * NF + m) * LX + f], rec[(3 * NF + m) * LX + f]);
  }
  __syncthreads();
  for (int f = tid; f < LX; f += BT) {
    if (i0 + f > N0) continue;
    iface_upwind_flow<EULER1D, UPW, MX>(P, rec + f, NF * LX, LX, sU + f + H - 1, sU + f + H, sU + H, HX, 0, sF + f,
                                        LX, spa + f, spm + f);
  }
  __syncthreads();
  for (int e = tid; e < (nv - NF) * LX; e += BT) {
    const int m = NF + e / LX, f = e % LX;
    if (i0 + f > N0) continue;
    T l, r, fl, fr;
    const double ur = MX ? sU[m * HX + H] : 0.0, frf = MX ? cf[m * HX + H] : 0.0;
    iface_weno<MX>(P, sU + m * HX + f + H, 1, cf + m * HX + f + H, 1, ur, frf, l, r, fl, fr);
    sF[m * LX + f] = upwind_species(spm[f], spa[f], l, r, fl, fr);
  }
  __syncthreads();
  const int i = i0 + tid;
  if (tid >= T1 || i >= N0) return;
  const long long p = pidx(P, i, 0);
  double* ks = M.k[s];
  const double dxi = M.dxinv[P.ghosts + i];
  for (int m = 0; m < nv; m++) {
    double h;
    if (MX) h = (double)((T)dxi * (sF[m * LX + tid + 1] - sF[m * LX + tid]));
    else h = dxi * (sF[m * LX + tid + 1] - sF[m * LX + tid]);
    ks[m * P.ps + p] = -h;
  }
  rk_point(M, Sd, s, p, nv);
}

// --------------------------------------------------------------- kernel
template <int TX, int TY, int BT, int MINB, bool MX>
__global__ void __launch_bounds__(BT, MINB) k_batch_stage(const BMember* __restrict__ mem,
                                                          const BState* __restrict__ st,
                                                          const int* __restrict__ tile_member,
                                                          const int* __restrict__ ntiles, int s) {
  extern __shared__ double smem_d[];
  char* smem = (char*)smem_d;
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
        case UPW_ROE: tile2d<TX, TY, UPW_ROE, BT, MX>(M, Sd, s, tx, ty, smem); break;
        case UPW_RF: tile2d<TX, TY, UPW_RF, BT, MX>(M, Sd, s, tx, ty, smem); break;
        case UPW_LLF: tile2d<TX, TY, UPW_LLF, BT, MX>(M, Sd, s, tx, ty, smem); break;
        default: tile2d<TX, TY, UPW_RUSANOV, BT, MX>(M, Sd, s, tx, ty, smem); break;
      }
    } else {
      switch (M.P.upwind) {
        case UPW_ROE: tile1d<UPW_ROE, BT, MX>(M, Sd, s, local, smem); break;
        case UPW_RF: tile1d<UPW_RF, BT, MX>(M, Sd, s, local, smem); break;
        case UPW_LLF: tile1d<UPW_LLF, BT, MX>(M, Sd, s, local, smem); break;
        default: tile1d<UPW_RUSANOV, BT, MX>(M, Sd, s, local, smem); break;
      }
    }
    __syncthreads();   // shared memory is reused by the next tile
  }
}
#endif  // __CUDACC__

// ------------------------------------------------------- launch tables
// Per-precision operations on the stage kernel of launch configuration
// `shape` (an index into kShapes).  Each precision is instantiated in its own
// translation unit (batch_stage_fp64.cu, batch_stage_mixed.cu).
template <bool MX>
struct StageTable {
  static long long smem(int shape, int nv);                       // dynamic shared memory, bytes
  static cudaError_t attr(int shape, long long bytes);            // raise the kernel's limit
  static int per_sm(int shape, long long bytes);                  // resident CTAs per SM
  static void launch(int shape, int grid, long long bytes, cudaStream_t st, const BMember* m, const BState* s,
                     const int* tiles, const int* ntiles, int stage);
};

#ifdef PIAFS_BATCH_STAGE_IMPL
template <int TX, int TY, int NT, int MINB, bool MX>
struct StageOps {
  static long long smem(int nv) { return std::max(Tile2D<TX, TY, MX>::smem(nv), Tile1D<NT, MX>::smem(nv)); }
  static cudaError_t attr(long long bytes) {
    return cudaFuncSetAttribute(k_batch_stage<TX, TY, NT, MINB, MX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes);
  }
  static int per_sm(long long bytes) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<TX, TY, NT, MINB, MX>, NT, bytes) !=
        cudaSuccess)
      n = 0;
    return n;
  }
  static void launch(int grid, long long bytes, cudaStream_t st, const BMember* m, const BState* s, const int* tl,
                     const int* nt, int stage) {
    k_batch_stage<TX, TY, NT, MINB, MX><<<grid, NT, bytes, st>>>(m, s, tl, nt, stage);
  }
};
#define PIAFS_SHAPE_SWITCH(idx, MX, CALL)                               \
  switch (idx) {                                                        \
    case 0: { typedef StageOps<16, 16, 512, 1, MX> Ops; CALL; } break;  \
    case 1: { typedef StageOps<32, 8, 512, 1, MX> Ops; CALL; } break;   \
    case 2: { typedef StageOps<16, 8, 256, 2, MX> Ops; CALL; } break;   \
    case 3: { typedef StageOps<32, 4, 256, 2, MX> Ops; CALL; } break;   \
    case 4: { typedef StageOps<8, 16, 256, 2, MX> Ops; CALL; } break;   \
    case 5: { typedef StageOps<16, 15, 512, 1, MX> Ops; CALL; } break;  \
    case 6: { typedef StageOps<32, 7, 512, 1, MX> Ops; CALL; } break;   \
    default: { typedef StageOps<16, 7, 256, 2, MX> Ops; CALL; } break;  \
  }

template <bool MX>
long long StageTable<MX>::smem(int shape, int nv) {
  long long r = 0;
  PIAFS_SHAPE_SWITCH(shape, MX, r = Ops::smem(nv));
  return r;
}
template <bool MX>
cudaError_t StageTable<MX>::attr(int shape, long long bytes) {
  cudaError_t e = cudaSuccess;
  PIAFS_SHAPE_SWITCH(shape, MX, e = Ops::attr(bytes));
  return e;
}
template <bool MX>
int StageTable<MX>::per_sm(int shape, long long bytes) {
  int r = 0;
  PIAFS_SHAPE_SWITCH(shape, MX, r = Ops::per_sm(bytes));
  return r;
}
template <bool MX>
void StageTable<MX>::launch(int shape, int grid, long long bytes, cudaStream_t st, const BMember* m,
                            const BState* s, const int* tiles, const int* ntiles, int stage) {
  PIAFS_SHAPE_SWITCH(shape, MX, Ops::launch(grid, bytes, st, m, s, tiles, ntiles, stage));
}
#undef PIAFS_SHAPE_SWITCH
#endif  // PIAFS_BATCH_STAGE_IMPL

}  // namespace batch
}  // namespace piafs
