// Hot-path kernels of the PIAFS GPU path (sm_100a).
//
// Per RK stage the host enqueues, for each direction d:
//   k_flux          cell-centred flux F_d(U) at every point (FFunction);
//                   for the y pass of 2D Navier-Stokes k_transpose_flux_y
//                   (transposed state and its y flux)
//   k_weno5 or      interface values uL,uR,fL,fR (InterpolateInterfacesHyp
//   k_crw_line        with the weights of SetInterpLimiterVar fused in;
//                     crweno_line.cu, crweno.cu)
//   k_upwind_div2d  upwind flux at the interfaces of both directions +
//   (k_upwind_div   conservative difference into the stage derivative
//    in 1D)         (Upwind + HyperbolicFunction's dxinv*(fI[j+1]-fI[j]))
// then k_visc_source (ParabolicFunction + SourceFunction) and the RK
// kernels k_stage / k_update2 (TimeRK).  All state is FP64.
#include <cstdio>
#include <type_traits>
#include "kernels.h"
#include "physics.cuh"
#include "source.cuh"

namespace piafs {

// ============================================================ layout helpers
__global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, long long npg,
                             int nv, long long ps) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= npg * nv) return;
  long long p = idx / nv;
  int v = (int)(idx - p * nv);
  soa[v * ps + p] = aos[idx];
}
__global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, long long npg,
                             int nv, long long ps) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= npg * nv) return;
  long long p = idx / nv;
  int v = (int)(idx - p * nv);
  aos[idx] = soa[v * ps + p];
}
// interior points only, op-file order (point-major, dim0 fastest)
__global__ void k_soa_to_interior(DevParams P, const double* __restrict__ soa, double* __restrict__ out) {
  long long n = (long long)P.N0 * P.N1 * P.nvars;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long long pt = idx / P.nvars;
  int v = (int)(idx - pt * P.nvars);
  int i = (int)(pt % P.N0), j = (int)(pt / P.N0);
  out[idx] = soa[v * P.ps + pidx(P, i, j)];
}
__global__ void k_interior_to_soa(DevParams P, const double* __restrict__ in, double* __restrict__ soa) {
  long long n = (long long)P.N0 * P.N1 * P.nvars;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long long pt = idx / P.nvars;
  int v = (int)(idx - pt * P.nvars);
  int i = (int)(pt % P.N0), j = (int)(pt / P.N0);
  soa[v * P.ps + pidx(P, i, j)] = in[idx];
}
// interface arrays: AoS (reference) <-> SoA (device)
__global__ void k_iface_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, long long ni,
                                   int nv, long long pis) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= ni * nv) return;
  long long q = idx / nv;
  int v = (int)(idx - q * nv);
  soa[v * pis + q] = aos[idx];
}
__global__ void k_iface_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, long long ni,
                                   int nv, long long pis) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= ni * nv) return;
  long long q = idx / nv;
  int v = (int)(idx - q * nv);
  aos[idx] = soa[v * pis + q];
}

// Plane-wise transpose of a ghosted state: in[v][j][i] (i fastest, W0 x W1)
// to out[v][i][j] (j fastest), through 32 x 32 shared-memory tiles.  The
// y-direction CRWENO5 pass runs on the transposed copy so that its lines are
// contiguous in memory.
__global__ void k_transpose_planes(const double* __restrict__ in, double* __restrict__ out, int W0, int W1,
                                   long long ps) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const double* a = in + blockIdx.z * ps;
  double* b = out + blockIdx.z * ps;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int i = i0 + threadIdx.x, j = j0 + r;
    if (i < W0 && j < W1) tile[r][threadIdx.x] = a[(long long)j * W0 + i];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int j = j0 + threadIdx.x, i = i0 + r;
    if (i < W0 && j < W1) b[(long long)i * W1 + j] = tile[threadIdx.x][r];
  }
}

// The y pass's transposed state and its y flux in one pass (2D
// Navier-Stokes): a 32 x 32 tile of points with all variables, the flow
// variables kept in shared memory for the flux, every variable written
// transposed to UT and its y flux (ns2d_flux; vn U_m for the passive ones,
// as k_flux forms them) to FT -- one read of U where the transpose and
// k_flux read it twice.
__global__ void __launch_bounds__(256) k_transpose_flux_y(DevParams P, const double* __restrict__ U,
                                                          double* __restrict__ UT, double* __restrict__ FT) {
  __shared__ double flow[4][32][33];
  __shared__ double tile[32][33];
  const int W0 = P.W0, W1 = P.W1;
  const long long ps = P.ps;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
  for (int m = 0; m < 4; m++)
    for (int r = ty; r < 32; r += 8) {
      const int i = i0 + tx, j = j0 + r;
      if (i < W0 && j < W1) flow[m][r][tx] = U[m * ps + (long long)j * W0 + i];
    }
  __syncthreads();
  // point (i = i0 + r, j = j0 + tx): writes along j are coalesced
  double vn[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int r = ty + 8 * k;
    const int j = j0 + tx, i = i0 + r;
    vn[k] = 0.0;
    if (i < W0 && j < W1) {
      double f[4];
      ns2d_flux(flow[0][tx][r], flow[1][tx][r], flow[2][tx][r], flow[3][tx][r], P.gamma, 1, f, vn[k]);
      const long long q = (long long)i * W1 + j;
#pragma unroll
      for (int m = 0; m < 4; m++) {
        UT[m * ps + q] = flow[m][tx][r];
        FT[m * ps + q] = f[m];
      }
    }
  }
  // passive variables one tile at a time, the next tile's loads in flight
  // while the current one is written
  double nxt[4];
  auto load = [&](int m) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int r = ty + 8 * k, i = i0 + tx, j = j0 + r;
      nxt[k] = (m < P.nvars && i < W0 && j < W1) ? U[m * ps + (long long)j * W0 + i] : 0.0;
    }
  };
  load(4);
  for (int m = 4; m < P.nvars; m++) {
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) tile[ty + 8 * k][tx] = nxt[k];
    load(m + 1);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int r = ty + 8 * k;
      const int j = j0 + tx, i = i0 + r;
      if (i < W0 && j < W1) {
        const long long q = (long long)i * W1 + j;
        const double x = tile[tx][r];
        UT[m * ps + q] = x;
        FT[m * ps + q] = __dmul_rn(vn[k], x);
      }
    }
  }
}

// ================================================================ boundaries
// One zone of ApplyBoundaryConditions: BCPeriodicU (BCPeriodic.c:22-62),
// BCExtrapolateU (BCExtrapolate.c:16-50), BCSlipWallU (BCSlipWall.c:24-136).
// Only the ghost slab of the zone is written; corner ghosts are never touched.
__global__ void k_bc_zone(DevParams P, double* __restrict__ u, Zone z) {
  int ni = z.ie[0] - z.is[0], nj = z.ie[1] - z.is[1];
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)ni * nj) return;
  const int g0 = z.is[0] + (int)(idx % ni), g1 = z.is[1] + (int)(idx / ni);
  bc_point(P, z, u, g0, g1, u + pidx(P, g0, g1), P.ps);
}
__global__ void k_stage(long long n, double* __restrict__ Us, const double* __restrict__ u,
                        const double* __restrict__ d0, double a0, const double* __restrict__ d1, double a1,
                        const double* __restrict__ d2, double a2, int nterms) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = u[i];
  if (nterms > 0) x += a0 * d0[i];
  if (nterms > 1) x += a1 * d1[i];
  if (nterms > 2) x += a2 * d2[i];
  Us[i] = x;
}

// u += sum_s (dt b_s) Udot_s (TimeRK.c:86-99); optionally accumulates
// sum (u_old - u_new)^2 over interior points (TimePostStep.c:36-54)
__global__ void k_update(DevParams P, double* __restrict__ u, const double* __restrict__ d0, double b0,
                         const double* __restrict__ d1, double b1, const double* __restrict__ d2, double b2,
                         const double* __restrict__ d3, double b3, int ns, double* __restrict__ norm_acc) {
  long long n = (long long)P.nvars * P.ps;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double sq = 0.0;
  if (i < n) {
    double old = u[i], x = old;
    if (ns > 0) x += b0 * d0[i];
    if (ns > 1) x += b1 * d1[i];
    if (ns > 2) x += b2 * d2[i];
    if (ns > 3) x += b3 * d3[i];
    u[i] = x;
    if (norm_acc) {
      long long p = i % P.ps;
      if (p < P.npg) {
        int ii = (int)(p % P.W0) - P.ghosts, jj = (int)(p / P.W0) - P.g1;
        if (ii >= 0 && ii < P.N0 && jj >= 0 && jj < P.N1) { double d = old - x; sq = d * d; }
      }
    }
  }
  if (norm_acc) {
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    __shared__ double ws[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = sq;
    __syncthreads();
    if (w == 0) {
      sq = lane < (blockDim.x >> 5) ? ws[lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
      if (lane == 0) atomicAdd(norm_acc, sq);
    }
  }
}

// k_update for ns stages, two consecutive values (one double2) per thread:
// the same arithmetic per value, more bytes in flight per thread
template <int NS>
__global__ void k_update2(DevParams P, double* __restrict__ u, const double* __restrict__ d0, double b0,
                          const double* __restrict__ d1, double b1, const double* __restrict__ d2, double b2,
                          const double* __restrict__ d3, double b3, double* __restrict__ norm_acc) {
  const long long n2 = (long long)P.nvars * P.ps / 2;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double sq = 0.0;
  if (i < n2) {
    const double2 old = reinterpret_cast<const double2*>(u)[i];
    double2 x = old;
    const double* dd[4] = {d0, d1, d2, d3};
    const double bb[4] = {b0, b1, b2, b3};
    double2 v[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) v[k] = reinterpret_cast<const double2*>(dd[k])[i];
#pragma unroll
    for (int k = 0; k < NS; k++) { x.x += bb[k] * v[k].x; x.y += bb[k] * v[k].y; }
    reinterpret_cast<double2*>(u)[i] = x;
    if (norm_acc) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const long long p = (2 * i + h) % P.ps;
        if (p < P.npg) {
          const int ii = (int)(p % P.W0) - P.ghosts, jj = (int)(p / P.W0) - P.g1;
          if (ii >= 0 && ii < P.N0 && jj >= 0 && jj < P.N1) {
            const double d = h == 0 ? old.x - x.x : old.y - x.y;
            sq += d * d;
          }
        }
      }
    }
  }
  if (norm_acc) {
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    __shared__ double ws[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = sq;
    __syncthreads();
    if (w == 0) {
      sq = lane < (blockDim.x >> 5) ? ws[lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
      if (lane == 0) atomicAdd(norm_acc, sq);
    }
  }
}

// max local CFL over interior points (NavierStokes2DComputeCFL.c:19-56,
// Euler1DComputeCFL.c).  Non-negative doubles order like their bit patterns.
__global__ void k_cfl(DevParams P, const double* __restrict__ u, const double* __restrict__ dxinv,
                      unsigned long long* __restrict__ out) {
  long long n = (long long)P.N0 * P.N1;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double m = 0.0;
  if (idx < n) {
    int i = (int)(idx % P.N0), j = (int)(idx / P.N0);
    long long p = pidx(P, i, j);
    if (P.model == NS2D) {
      double rho, vx, vy, e, pr;
      ns_flowvar(u[p], u[P.ps + p], u[2 * P.ps + p], u[3 * P.ps + p], P.gamma, rho, vx, vy, e, pr);
      double c = sqrt(P.gamma * pr / rho);
      double lx = (absv(vx) + c) * P.dt * dxinv[P.ghosts + i];
      double ly = (absv(vy) + c) * P.dt * dxinv[P.W0 + P.ghosts + j];
      m = maxv(lx, ly);
    } else {
      double rho, v, e, pr;
      eu_flowvar(u[p], u[P.ps + p], u[2 * P.ps + p], P.gamma, rho, v, e, pr);
      double c = sqrt(P.gamma * pr / rho);
      m = (absv(v) + c) * P.dt * dxinv[P.ghosts + i];
    }
    if (!(m >= 0.0)) m = 0.0;
  }
  for (int o = 16; o > 0; o >>= 1) m = maxv(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// ===================================================================== flux
// NavierStokes2DFlux (NavierStokes2DFlux.c:24-52) / Euler1DFlux, every point
template <int MODEL, int DIR>
__global__ void k_flux(DevParams P, const double* __restrict__ U, double* __restrict__ F) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= P.npg) return;
  const long long ps = P.ps;
  double f[4], vn;
  if (MODEL == NS2D) {
    ns2d_flux(U[p], U[ps + p], U[2 * ps + p], U[3 * ps + p], P.gamma, DIR, f, vn);
    for (int m = 0; m < 4; m++) F[m * ps + p] = f[m];
    for (int m = 4; m < P.nvars; m++) F[m * ps + p] = __dmul_rn(vn, U[m * ps + p]);
  } else {
    euler1d_flux(U[p], U[ps + p], U[2 * ps + p], P.gamma, f, vn);
    for (int m = 0; m < 3; m++) F[m * ps + p] = f[m];
    for (int m = 3; m < P.nvars; m++) F[m * ps + p] = __dmul_rn(vn, U[m * ps + p]);
  }
}

// decode interface index q of direction DIR into (position along dir, line)
template <int DIR>
__device__ __forceinline__ void iface_decode(const DevParams& P, long long q, int& i, int& l) {
  if (DIR == 0) { i = (int)(q % (P.N0 + 1)); l = (int)(q / (P.N0 + 1)); }
  else          { l = (int)(q % P.N0);       i = (int)(q / P.N0); }
}
template <int DIR>
__device__ __forceinline__ long long cell_of(const DevParams& P, int i, int l) {
  return DIR == 0 ? pidx(P, i, l) : pidx(P, l, i);
}

// ==================================================================== WENO5
// Interp1PrimFifthOrderWENO (Interp1PrimFifthOrderWENO.c:77-171) for the four
// (upw, uflag) combinations with the weights of
// WENOFifthOrderCalculateWeights fused in; one thread per (interface, var).
// MX (mixed precision): cells relative to the line's first interior value
// (FP64 subtraction), weights and values in FP32, stored as FP32 relative to
// that reference, as in the mixed CRWENO5 kernel.
template <int DIR, bool MX>
__global__ void k_weno5(DevParams P, const double* __restrict__ U, const double* __restrict__ F,
                        void* __restrict__ uLv, void* __restrict__ uRv, void* __restrict__ fLv,
                        void* __restrict__ fRv) {
  typedef typename std::conditional<MX, float, double>::type R;
  const long long ni = P.nint[DIR];
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= ni * P.nvars) return;
  int v = (int)(idx / ni);
  long long q = idx - (long long)v * ni;
  int i, l;
  iface_decode<DIR>(P, q, i, l);
  const long long st = DIR == 0 ? 1 : P.W0;
  const long long c0 = cell_of<DIR>(P, i, l);    // cell i (right of the interface)
  const double* u = U + (long long)v * P.ps + c0;
  const double* f = F + (long long)v * P.ps + c0;
  double ru = 0.0, rf = 0.0;
  if (MX) {
    const long long l0 = cell_of<DIR>(P, 0, l);
    ru = U[(long long)v * P.ps + l0]; rf = F[(long long)v * P.ps + l0];
  }
  R a[6], b[6];     // cells i-3 .. i+2
#pragma unroll
  for (int r = 0; r < 6; r++) { a[r] = (R)(u[(r - 3) * st] - ru); b[r] = (R)(f[(r - 3) * st] - rf); }
  const long long o = (long long)v * P.pis + q;
  R* uL = (R*)uLv; R* uR = (R*)uRv; R* fL = (R*)fLv; R* fR = (R*)fRv;
  weno5_iface(P, a, b, uL[o], uR[o], fL[o], fR[o]);
}

// ======================================================== WENO5 (characteristic)
// Interp1PrimFifthOrderWENOChar (Interp1PrimFifthOrderWENOChar.c:92-200) with
// the weights of WENOFifthOrderCalculateWeightsChar
// (WENOFifthOrderCalculateWeights.c:761-1409): at each interface the flow
// variables of the six stencil cells, of u and of the flux f alike, are
// projected on the left eigenvectors of the Roe average of the two cells
// beside the interface, each characteristic field is WENO5-reconstructed
// (weights from its own projected values) for both biases, and the results
// go back through the right eigenvectors.  The passive variables have unit
// eigenvectors (navierstokes2d.h:243-247), so their reconstruction is the
// component one.  One thread per interface.  (The reference takes the
// average of the cells in the order of each bias; it is the same state to
// rounding, and one average serves both biases here.)
template <int MODEL, int DIR>
__global__ void k_weno5_char(DevParams P, const double* __restrict__ U, const double* __restrict__ F,
                             double* __restrict__ uL, double* __restrict__ uR, double* __restrict__ fL,
                             double* __restrict__ fR) {
  constexpr int NF = Flow<MODEL>::NF;
  const long long ni = P.nint[DIR];
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= ni) return;
  int i, l;
  iface_decode<DIR>(P, q, i, l);
  const long long st = DIR == 0 ? 1 : P.W0;
  const long long c0 = cell_of<DIR>(P, i, l);    // cell i (right of the interface)
  const long long ps = P.ps;
  double cl[4], cr[4], ua[4], L[4][4], R[4][4];
#pragma unroll
  for (int m = 0; m < NF; m++) { cl[m] = U[m * ps + c0 - st]; cr[m] = U[m * ps + c0]; }
  Flow<MODEL>::roe_avg(cl, cr, P.gamma, ua);
  Flow<MODEL>::eigvec(ua, P.gamma, DIR, L, R);
#pragma unroll
  for (int fld = 0; fld < 2; fld++) {
    const double* src = fld ? F : U;
    double w[NF][6];                              // characteristic values, cells i-3 .. i+2
#pragma unroll
    for (int r = 0; r < 6; r++) {
      double cv[4];
#pragma unroll
      for (int m = 0; m < NF; m++) cv[m] = src[m * ps + c0 + (r - 3) * st];
#pragma unroll
      for (int v = 0; v < NF; v++) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < NF; k++) acc += L[v][k] * cv[k];
        w[v][r] = acc;
      }
    }
    double vl[4], vr[4];
#pragma unroll
    for (int v = 0; v < NF; v++) weno5_pair(P, w[v], vl[v], vr[v]);
    double* oL = fld ? fL : uL;
    double* oR = fld ? fR : uR;
#pragma unroll
    for (int k = 0; k < NF; k++) {
      double sl = 0.0, sr = 0.0;
#pragma unroll
      for (int v = 0; v < NF; v++) { sl += R[k][v] * vl[v]; sr += R[k][v] * vr[v]; }
      oL[k * P.pis + q] = sl;
      oR[k * P.pis + q] = sr;
    }
  }
  for (int m = NF; m < P.nvars; m++) {
    double a[6], b[6];
#pragma unroll
    for (int r = 0; r < 6; r++) { a[r] = U[m * ps + c0 + (r - 3) * st]; b[r] = F[m * ps + c0 + (r - 3) * st]; }
    const long long o = (long long)m * P.pis + q;
    weno5_iface(P, a, b, uL[o], uR[o], fL[o], fR[o]);
  }
}

// ============================================================ upwind + div
// Upwind (NavierStokes2DUpwind*/Euler1DUpwind*) at the interfaces of a tile,
// then hyp += dxinv (fI[j+1] - fI[j]) (HyperbolicFunction.c:97-112) and the
// stage derivative rhs = -hyp (TimeRHSFunctionExplicit.c:64-66).
// mode 0: rhs = -hyp_x (first direction); 1: rhs <- -((-rhs) + hyp_y);
// mode 2: out = hyp_x; 3: out <- out + hyp_y (the hyperbolic term alone).
// Tile: DIR 0: 128 cells of one row; DIR 1: 32 columns x 8 rows.
// MX (mixed precision, 1D): FP32 interface values relative to the line's
// reference, fluxes in deviation form (upwind_flow_dev), FP32 differences.
template <int MODEL, int UPW, int DIR, bool MX>
__global__ void __launch_bounds__(256) k_upwind_div(DevParams P, const double* __restrict__ U,
                                                    const void* __restrict__ uLv, const void* __restrict__ uRv,
                                                    const void* __restrict__ fLv, const void* __restrict__ fRv,
                                                    const double* __restrict__ dxinv, double* __restrict__ rhs,
                                                    int mode) {
  typedef typename std::conditional<MX, float, double>::type T;
  extern __shared__ double sfd[];
  T* sfi = (T*)sfd;
  const T* uL = (const T*)uLv; const T* uR = (const T*)uRv;
  const T* fL = (const T*)fLv; const T* fR = (const T*)fRv;
  constexpr int NF = Flow<MODEL>::NF;
  const int TX = DIR == 0 ? 128 : 32, TY = DIR == 0 ? 1 : 8;
  const int TL = DIR == 0 ? TX : TY;             // cells along the line in the tile
  const int TW = DIR == 0 ? 1 : TX;              // lines in the tile
  const int nvars = P.nvars;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int N = DIR == 0 ? P.N0 : P.N1;
  const int nl = DIR == 0 ? P.N1 : P.N0;
  // tile origin
  const int i0 = DIR == 0 ? blockIdx.x * TX : blockIdx.y * TY;     // along the line
  const int l0 = DIR == 0 ? blockIdx.y : blockIdx.x * TX;          // first line
  const double g = P.gamma;
  // interfaces i0 .. i0+TL for lines l0 .. l0+TW-1
  const int nIf = (TL + 1) * TW;
  const int tid = tx + TX * ty, nth = TX * TY;
  for (int e = tid; e < nIf; e += nth) {
    int li, ii;
    if (DIR == 0) { ii = e; li = 0; } else { li = e % TW; ii = e / TW; }
    const int i = i0 + ii, l = l0 + li;
    if (i > N || l >= nl) continue;
    const long long q = DIR == 0 ? (long long)i + (long long)(P.N0 + 1) * l : (long long)l + (long long)P.N0 * i;
    const long long pL = cell_of<DIR>(P, i - 1, l), pR = cell_of<DIR>(P, i, l);
    T a[4], b[4], c[4], d[4], ucl[4], ucr[4], fi[4], spa;
    int spm;
#pragma unroll
    for (int m = 0; m < NF; m++) {
      a[m] = uL[m * P.pis + q]; b[m] = uR[m * P.pis + q];
      c[m] = fL[m * P.pis + q]; d[m] = fR[m * P.pis + q];
      if (UPW != UPW_LLF || MODEL == EULER1D) { ucl[m] = (T)U[m * P.ps + pL]; ucr[m] = (T)U[m * P.ps + pR]; }
    }
    if (MX) upwind_flow_dev<MODEL, UPW, T>(a, b, c, d, a, b, ucl, ucr, (T)g, DIR, fi, &spa, &spm);
    else upwind_flow<MODEL, UPW, T>(a, b, c, d, ucl, ucr, (T)g, DIR, fi, &spa, &spm);
    T* so = sfi + (long long)(ii * TW + li);
    const int vs = (TL + 1) * TW;
#pragma unroll
    for (int m = 0; m < NF; m++) so[m * vs] = fi[m];
    for (int m = NF; m < nvars; m++)
      so[m * vs] = upwind_species(spm, spa, uL[m * P.pis + q], uR[m * P.pis + q], fL[m * P.pis + q], fR[m * P.pis + q]);
  }
  __syncthreads();
  // divergence for the tile's cells
  int ii, li;
  if (DIR == 0) { ii = tx; li = 0; } else { li = tx; ii = ty; }
  const int i = i0 + ii, l = l0 + li;
  if (i >= N || l >= nl) return;
  const long long p = cell_of<DIR>(P, i, l);
  const int off = DIR == 0 ? 0 : P.W0;
  const T dxi = (T)dxinv[off + P.ghosts + i];
  const int vs = (TL + 1) * TW;
  for (int m = 0; m < nvars; m++) {
    const double h = (double)(dxi * (sfi[m * vs + (ii + 1) * TW + li] - sfi[m * vs + ii * TW + li]));
    double* r = rhs + (long long)m * P.ps + p;
    if (mode == 0) *r = -h;
    else if (mode == 1) *r = -((-*r) + h);
    else if (mode == 2) *r = h;
    else *r = *r + h;
  }
}

// Upwind flux of all components at one interface q of direction DIR into
// so[m * sm_stride] (NavierStokes2DUpwind*); cells pL / pR are the cells left
// and right of the interface in `cells`.  MX: the interface arrays hold
// floats relative to the line's reference values, uref (absolute, FP64) are
// those references for the flow variables, the flux is computed in FP32 in
// deviation form and stored relative to the line's flux reference.
template <int UPW, int DIR, bool MX>
__device__ __forceinline__ void iface_upwind(const DevParams& P, const void* __restrict__ uLv,
                                             const void* __restrict__ uRv, const void* __restrict__ fLv,
                                             const void* __restrict__ fRv, long long q,
                                             const double* __restrict__ cells, long long pL, long long pR,
                                             const double* uref,
                                             typename std::conditional<MX, float, double>::type* so, int sm_stride) {
  typedef typename std::conditional<MX, float, double>::type T;
  constexpr int NF = Flow<NS2D>::NF;
  const T* uL = (const T*)uLv; const T* uR = (const T*)uRv;
  const T* fL = (const T*)fLv; const T* fR = (const T*)fRv;
  T a[4], b[4], c[4], d[4], ucl[4], ucr[4], fi[4], spa;
  int spm;
#pragma unroll
  for (int m = 0; m < NF; m++) {
    a[m] = uL[m * P.pis + q]; b[m] = uR[m * P.pis + q];
    c[m] = fL[m * P.pis + q]; d[m] = fR[m * P.pis + q];
    if (UPW != UPW_LLF) { ucl[m] = (T)cells[m * P.ps + pL]; ucr[m] = (T)cells[m * P.ps + pR]; }
  }
  if (MX) {
    T aL[4], aR[4];
    if (UPW == UPW_LLF || UPW == UPW_RF) {
#pragma unroll
      for (int m = 0; m < NF; m++) { const T r = (T)uref[m]; aL[m] = r + a[m]; aR[m] = r + b[m]; }
    }
    upwind_flow_dev<NS2D, UPW, T>(a, b, c, d, aL, aR, ucl, ucr, (T)P.gamma, DIR, fi, &spa, &spm);
  } else {
    upwind_flow<NS2D, UPW, T>(a, b, c, d, ucl, ucr, (T)P.gamma, DIR, fi, &spa, &spm);
  }
#pragma unroll
  for (int m = 0; m < NF; m++) so[m * sm_stride] = fi[m];
  if (P.pack_sp) {
    // passive variables packed by the line solve: uL - uR, fL + fR
    int m = NF;
    for (; m + 4 <= P.nvars; m += 4) {
      T du[4], sf[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const long long o = (long long)(m + k) * P.pis + q;
        du[k] = uL[o]; sf[k] = fL[o];
      }
#pragma unroll
      for (int k = 0; k < 4; k++) so[(m + k) * sm_stride] = upwind_species_packed(spm, spa, du[k], sf[k]);
    }
    for (; m < P.nvars; m++)
      so[m * sm_stride] = upwind_species_packed(spm, spa, uL[m * P.pis + q], fL[m * P.pis + q]);
    return;
  }
  // passive variables four at a time, their sixteen loads in flight together
  int m = NF;
  for (; m + 4 <= P.nvars; m += 4) {
    T l[4], r[4], fl[4], fr[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const long long o = (long long)(m + k) * P.pis + q;
      l[k] = uL[o]; r[k] = uR[o]; fl[k] = fL[o]; fr[k] = fR[o];
    }
#pragma unroll
    for (int k = 0; k < 4; k++) so[(m + k) * sm_stride] = upwind_species(spm, spa, l[k], r[k], fl[k], fr[k]);
  }
  for (; m < P.nvars; m++)
    so[m * sm_stride] = upwind_species(spm, spa, uL[m * P.pis + q], uR[m * P.pis + q], fL[m * P.pis + q],
                                       fR[m * P.pis + q]);
}

// Both directions of the 2D hyperbolic term in one pass: upwind fluxes at the
// x and y interfaces of a 16 x 15 tile (one of each per thread), then
// hyp = dxinv_x (fIx[i+1] - fIx[i]) + dxinv_y (fIy[j+1] - fIy[j])
// (HyperbolicFunction.c:97-112, the x term first) and rhs = -hyp (neg = 1,
// TimeRHSFunctionExplicit.c:64-66) or out = hyp (neg = 0): the same sum, in
// the same order, that the per-direction kernels accumulate, with the stage
// derivative written once.  The y-interface arrays are in the transposed
// layout (q = j + (N1+1) i, cell values from UT) when YT, else in the
// standard one (q = i + N0 j, cell values from U).  MX: mixed precision (FP32
// interface values relative to their line's reference, FP32 fluxes and
// differences, FP64 result).
template <int UPW, bool YT, bool MX, bool HYIN>
__global__ void __launch_bounds__(256, 3) k_upwind_div2d(DevParams P, const double* __restrict__ U,
                                                      const double* __restrict__ UT,
                                                      const void* __restrict__ xuL, const void* __restrict__ xuR,
                                                      const void* __restrict__ xfL, const void* __restrict__ xfR,
                                                      const void* __restrict__ yuL, const void* __restrict__ yuR,
                                                      const void* __restrict__ yfL, const void* __restrict__ yfR,
                                                      const double* __restrict__ dxinv, double* __restrict__ rhs,
                                                      int neg, const void* __restrict__ hyin, int n0) {
  typedef typename std::conditional<MX, float, double>::type T;
  extern __shared__ double sfd[];
  T* sf = (T*)sfd;
  constexpr int TI = 16, TJ = 15, LX = TI + 1, LY = TJ + 2;   // LY padded against bank conflicts
  constexpr int NX = LX * TJ, NY = TI * LY;
  const int nvars = P.nvars, N0 = P.N0, N1 = P.N1, g = P.ghosts;
  const int i0 = blockIdx.x * TI, j0 = blockIdx.y * TJ;
  const int tid = threadIdx.x;
  T* sx = sf;               // x-interface fluxes [m][row jj][ii = 0..TI]
  T* sy = sf + nvars * NX;  // y-interface fluxes [m][column ii][jj = 0..TJ]
  double uref[4];
  if (tid < NX) {                // (TI + 1) x TJ x-interfaces
    const int ii = tid % LX, jj = tid / LX;
    const int i = i0 + ii, j = j0 + jj;
    if (i <= N0 && j < N1) {
      const long long pR = pidx(P, i, j);
      if (MX && (UPW == UPW_LLF || UPW == UPW_RF)) {
        const long long p0 = pidx(P, 0, j);
#pragma unroll
        for (int m = 0; m < 4; m++) uref[m] = U[m * P.ps + p0];
      }
      iface_upwind<UPW, 0, MX>(P, xuL, xuR, xfL, xfR, i + (long long)(N0 + 1) * j, U, pR - 1, pR, uref,
                               sx + jj * LX + ii, NX);
    }
  }
  if (!HYIN) {                   // TI x (TJ + 1) y-interfaces
    int ii, jj;
    if (YT) { jj = tid % (TJ + 1); ii = tid / (TJ + 1); }
    else { ii = tid % TI; jj = tid / TI; }
    const int i = i0 + ii, j = j0 + jj;
    if (j <= N1 && i < N0) {
      if (MX && (UPW == UPW_LLF || UPW == UPW_RF)) {
        const long long p0 = pidx(P, i, 0);
#pragma unroll
        for (int m = 0; m < 4; m++) uref[m] = U[m * P.ps + p0];
      }
      if (YT) {
        const long long pR = (long long)(j + g) + (long long)P.W1 * (i + g);
        iface_upwind<UPW, 1, MX>(P, yuL, yuR, yfL, yfR, j + (long long)(N1 + 1) * i, UT, pR - 1, pR, uref,
                                 sy + ii * LY + jj, NY);
      } else {
        const long long pR = pidx(P, i, j);
        iface_upwind<UPW, 1, MX>(P, yuL, yuR, yfL, yfR, i + (long long)N0 * j, U, pR - P.W0, pR, uref,
                                 sy + ii * LY + jj, NY);
      }
    }
  }
  __syncthreads();
  if (tid >= TI * TJ) return;
  const int ii = tid % TI, jj = tid / TI;
  const int i = i0 + ii, j = j0 + jj;
  if (i >= N0 || j >= N1) return;
  const long long p = pidx(P, i, j);
  const T dxi = (T)dxinv[g + i], dyi = (T)dxinv[P.W0 + g + j];
  // HYIN: the y term of column i comes from the slab that owns it, as
  // hyin[((i / n0) nvars + m) N1 + j) n0 + i % n0] (k_slab_upwind_y)
  const T* hyv = (const T*)hyin;
  const long long hbase = HYIN ? (long long)(i / n0) * nvars * N1 * n0 + (long long)j * n0 + i % n0 : 0;
  for (int m = 0; m < nvars; m++) {
    // hyp = dxinv_x dfx + dxinv_y dfy as dxinv_x dfx fused onto the rounded y
    // term, on both paths
    const T dfx = sx[m * NX + jj * LX + ii + 1] - sx[m * NX + jj * LX + ii];
    const T hy = HYIN ? hyv[hbase + (long long)m * N1 * n0]
                      : mul_rn(dyi, sy[m * NY + ii * LY + jj + 1] - sy[m * NY + ii * LY + jj]);
    const double h = (double)fma_rn(dxi, dfx, hy);
    rhs[(long long)m * P.ps + p] = neg ? -h : h;
  }
}

// The y term of the 2D hyperbolic divergence on a column slab of a grid
// decomposed along y (columns [c0, c0 + N0) of the whole grid, all N1 rows,
// in the transposed layout: cell values from UT, interface q = j + (N1 + 1) c):
// the upwind fluxes at the y interfaces of a 16 x 15 tile as in
// k_upwind_div2d, then dyinv_j (fIy[j+1] - fIy[j]) for every variable,
// written for the row slab that owns row j: hy[((r nvars + m) n1 + j - r n1)
// N0 + c], r = j / n1.  The product is rounded on its own; k_upwind_div2d
// fuses the x term's product onto it.
template <int UPW, bool MX>
__global__ void __launch_bounds__(256, 3) k_slab_upwind_y(DevParams P, const double* __restrict__ UT,
                                                       const void* __restrict__ yuL, const void* __restrict__ yuR,
                                                       const void* __restrict__ yfL, const void* __restrict__ yfR,
                                                       const double* __restrict__ dyinv, void* __restrict__ hy,
                                                       int n1) {
  typedef typename std::conditional<MX, float, double>::type T;
  extern __shared__ double sfd[];
  T* sy = (T*)sfd;
  constexpr int TI = 16, TJ = 15, LY = TJ + 2, NY = TI * LY;
  const int nvars = P.nvars, N0 = P.N0, N1 = P.N1, g = P.ghosts;
  const int i0 = blockIdx.x * TI, j0 = blockIdx.y * TJ;
  const int tid = threadIdx.x;
  double uref[4];
  {
    const int jj = tid % (TJ + 1), ii = tid / (TJ + 1);
    const int i = i0 + ii, j = j0 + jj;
    if (ii < TI && j <= N1 && i < N0) {
      const long long line = (long long)P.W1 * (i + g);
      if (MX && (UPW == UPW_LLF || UPW == UPW_RF)) {
#pragma unroll
        for (int m = 0; m < 4; m++) uref[m] = UT[m * P.ps + g + line];
      }
      const long long pR = (long long)(j + g) + line;
      iface_upwind<UPW, 1, MX>(P, yuL, yuR, yfL, yfR, j + (long long)(N1 + 1) * i, UT, pR - 1, pR, uref,
                               sy + ii * LY + jj, NY);
    }
  }
  __syncthreads();
  if (tid >= TI * TJ) return;
  const int ii = tid % TI, jj = tid / TI;
  const int i = i0 + ii, j = j0 + jj;
  if (i >= N0 || j >= N1) return;
  const T dyi = (T)dyinv[g + j];
  const int r = j / n1;
  T* out = (T*)hy + ((long long)r * nvars * n1 + (j - (long long)r * n1)) * N0 + i;
  for (int m = 0; m < nvars; m++)
    out[(long long)m * n1 * N0] = mul_rn(dyi, sy[m * NY + ii * LY + jj + 1] - sy[m * NY + ii * LY + jj]);
}

// ===================================================== viscous + chemistry
// FirstDerivativeFourthOrderCentral (FirstDerivativeFourthOrder.c:68-127) at
// index i of a line with N interior points and g ghosts, f(k) the value at
// i + k: the central stencil inside, the reference's biased ones at the two
// outermost points of each end (not divided by the grid spacing).  The
// reference writes the left rows, then the interior, then the right rows, so
// the right rows are tested first.
template <typename T, typename Fn>
__device__ __forceinline__ T d4(int i, int N, int g, Fn f) {
  const T c = T(1.0 / 12.0);
  if (i == N + g - 1) return (T(3) * f(-4) - T(16) * f(-3) + T(36) * f(-2) - T(48) * f(-1) + T(25) * f(0)) * c;
  if (i == N + g - 2) return (-f(-3) + T(6) * f(-2) - T(18) * f(-1) + T(10) * f(0) + T(3) * f(1)) * c;
  if (i == -g) return (T(-25) * f(0) + T(48) * f(1) - T(36) * f(2) + T(16) * f(3) - T(3) * f(4)) * c;
  if (i == -g + 1) return (T(-3) * f(-1) - T(10) * f(0) + T(18) * f(1) - T(6) * f(2) + f(3)) * c;
  return (f(-2) - T(8) * f(-1) + T(8) * f(1) - f(2)) * c;
}

// NavierStokes2DParabolicFunction (NavierStokes2DParabolicFunction.c:41-204)
// with FirstDerivativeFirstOrder (bias +1 on Q, -1 on the fluxes), fused with
// SourceFunction -> ChemistrySource (ChemistrySolve.c:18-115) and the RHS
// accumulation rhs += par; rhs += source (TimeRHSFunctionExplicit.c:67-74).
// Tile: 32 x 8 interior points.  Cross-derivative terms at ghost columns/rows
// are zero, as the reference computes derivatives on interior lines only.
// MX (mixed precision): velocities and temperature, their differences, the
// viscous fluxes and the chemistry in FP32; the temperature is held relative
// to the tile's first point (taken in FP64) so that its differences keep
// FP32's relative precision; the result is added to the FP64 rhs.  Six
// CTAs per SM (40 registers): the tile's two phases and its memory latency
// overlap across more CTAs (0.33 vs 0.38 ms per launch at 2048^2).
template <bool MX>
__global__ void __launch_bounds__(256, 6) k_visc_source(DevParams P, const double* __restrict__ U,
                                                     const double* __restrict__ dxinv,
                                                     const double* __restrict__ imap,
                                                     const double* __restrict__ tdev, double cstage,
                                                     double* __restrict__ rhs, int do_chem,
                                                     double* __restrict__ hnu) {
  typedef typename std::conditional<MX, float, double>::type T;
  constexpr int BX = 32, BY = 8, QX = BX + 2, QY = BY + 2, FX = BX + 1, FY = BY + 1;
  __shared__ T su[QY][QX], sv[QY][QX], sT[QY][QX];
  __shared__ T fx[3][BY][FX];   // FVx at i in [i0-1, i0+BX), rows j0..j0+BY-1
  __shared__ T fy[3][FY][BX];   // FVy at j in [j0-1, j0+BY), cols i0..i0+BX-1
  const int i0 = blockIdx.x * BX, j0 = blockIdx.y * BY;
  const int tid = threadIdx.x + BX * threadIdx.y;
  const long long ps = P.ps;
  if (P.viscous) {
    double Tref = 0.0;
    if (MX) {
      const long long p0 = pidx(P, i0, j0);
      double rho, uu, vv, e_, pr;
      ns_flowvar(U[p0], U[ps + p0], U[2 * ps + p0], U[3 * ps + p0], P.gamma, rho, uu, vv, e_, pr);
      Tref = P.gamma * pr / rho;
    }
    // Q = (u, v, T = gamma p / rho) on [i0-1, i0+BX] x [j0-1, j0+BY]
    for (int e = tid; e < QX * QY; e += BX * BY) {
      const int a = e % QX, b = e / QX;
      const int i = i0 - 1 + a, j = j0 - 1 + b;
      double uu = 0.0, vv = 0.0, TT = Tref;
      if (i >= -P.ghosts && i < P.N0 + P.ghosts && j >= -P.ghosts && j < P.N1 + P.ghosts) {
        const long long p = pidx(P, i, j);
        double rho, e_, pr;
        ns_flowvar(U[p], U[ps + p], U[2 * ps + p], U[3 * ps + p], P.gamma, rho, uu, vv, e_, pr);
        TT = P.gamma * pr / rho;
      }
      su[b][a] = (T)uu; sv[b][a] = (T)vv; sT[b][a] = (T)(TT - Tref);
    }
    __syncthreads();
    const T two_third = T(2.0 / 3.0), inv_Re = (T)(1.0 / P.Re), inv_Pr = (T)(1.0 / P.Pr);
    const T igm1 = (T)(1.0 / (P.gamma - 1.0));
    // viscous fluxes on [i0-1, i0+BX) x [j0-1, j0+BY) (corner cell unused)
    for (int e = tid; e < FX * FY; e += BX * BY) {
      const int a = e % FX, b = e / FX;       // a: i - (i0-1), b: j - (j0-1)
      const int i = i0 - 1 + a, j = j0 - 1 + b;
      const bool need_x = (b >= 1) && (j < P.N1) && (i < P.N0);   // FVx at interior rows
      const bool need_y = (a >= 1) && (i < P.N0) && (j < P.N1);   // FVy at interior columns
      if (!need_x && !need_y) continue;
      const int qa = a, qb = b;               // (i, j) in the Q tile
      const T dxi = (T)dxinv[P.ghosts + i], dyi = (T)dxinv[P.W0 + P.ghosts + j];
      // interior rows of the whole grid (a row slab's ghost rows inside it are
      // interior rows)
      const bool row_int = (j + P.jg0 >= 0 && j + P.jg0 < P.N1g), col_int = (i >= 0 && i < P.N0);
      const T uc = su[qb][qa], vc = sv[qb][qa], Tc = sT[qb][qa];
      // first differences (QDerivX only on interior rows, QDerivY only on interior columns)
      const T ux = row_int ? dxi * (su[qb][qa + 1] - uc) : T(0);
      const T vx = row_int ? dxi * (sv[qb][qa + 1] - vc) : T(0);
      const T Tx = row_int ? dxi * (sT[qb][qa + 1] - Tc) : T(0);
      const T uy = col_int ? dyi * (su[qb + 1][qa] - uc) : T(0);
      const T vy = col_int ? dyi * (sv[qb + 1][qa] - vc) : T(0);
      const T Ty = col_int ? dyi * (sT[qb + 1][qa] - Tc) : T(0);
      T mu, kappa;
      visc_coeffs<T>(P, MX ? (T)Tref + Tc : Tc, mu, kappa);
      const T mre = mu * inv_Re, kre = kappa * inv_Re * igm1 * inv_Pr;
      if (need_x) {
        const T txx = two_third * mre * (T(2) * ux - vy), txy = mre * (uy + vx);
        fx[0][b - 1][a] = txx; fx[1][b - 1][a] = txy; fx[2][b - 1][a] = uc * txx + vc * txy + kre * Tx;
      }
      if (need_y) {
        const T tyx = mre * (uy + vx), tyy = two_third * mre * (-ux + T(2) * vy);
        fy[0][b][a - 1] = tyx; fy[1][b][a - 1] = tyy; fy[2][b][a - 1] = uc * tyx + vc * tyy + kre * Ty;
      }
    }
    __syncthreads();
  }
  const int a = threadIdx.x, b = threadIdx.y;
  const int i = i0 + a, j = j0 + b;
  if (i >= P.N0 || j >= P.N1) return;
  const long long p = pidx(P, i, j);
  if (P.viscous) {
    const T dxi = (T)dxinv[P.ghosts + i], dyi = (T)dxinv[P.W0 + P.ghosts + j];
#pragma unroll
    for (int m = 0; m < 3; m++) {
      const T par = dxi * (fx[m][b][a + 1] - fx[m][b][a]) + dyi * (fy[m][b + 1][a] - fy[m][b][a]);
      rhs[(m + 1) * ps + p] += (double)par;
    }
  }
  if (do_chem) {
    const double t = *tdev + cstage * P.dt;
    chem_source_point<T>(P, U, p, pulse_factor(P, t), imap[p], rhs, hnu);
  }
}

// k_visc_source with par_space_scheme 4: the first derivatives of Q and of
// the viscous fluxes by FirstDerivativeFourthOrderCentral (d4; the bias is
// ignored), NavierStokes2DParabolicFunction.c:41-204 otherwise unchanged.
// Tile: 32 x 8 interior points; the viscous fluxes reach two points beyond
// it, their derivatives of Q two more.  As in the reference, QDerivX exists on
// interior rows and QDerivY on interior columns only (zero elsewhere), so no
// corner ghost is read.
template <bool MX>
__global__ void __launch_bounds__(256) k_visc4_source(DevParams P, const double* __restrict__ U,
                                                      const double* __restrict__ dxinv,
                                                      const double* __restrict__ imap,
                                                      const double* __restrict__ tdev, double cstage,
                                                      double* __restrict__ rhs, int do_chem,
                                                      double* __restrict__ hnu) {
  typedef typename std::conditional<MX, float, double>::type T;
  constexpr int BX = 32, BY = 8, HQ = 4, HF = 2;
  constexpr int QX = BX + 2 * HQ, QY = BY + 2 * HQ, FXW = BX + 2 * HF, FYH = BY + 2 * HF;
  __shared__ T su[QY][QX], sv[QY][QX], sT[QY][QX];
  __shared__ T fx[3][BY][FXW];   // FVx at i in [i0-2, i0+BX+2), rows j0..j0+BY-1
  __shared__ T fy[3][FYH][BX];   // FVy at j in [j0-2, j0+BY+2), cols i0..i0+BX-1
  const int i0 = blockIdx.x * BX, j0 = blockIdx.y * BY;
  const int tid = threadIdx.x + BX * threadIdx.y;
  const long long ps = P.ps;
  const int g = P.ghosts, N0 = P.N0, N1 = P.N1;
  double Tref = 0.0;
  if (MX) {
    const long long p0 = pidx(P, i0, j0);
    double rho, uu, vv, e_, pr;
    ns_flowvar(U[p0], U[ps + p0], U[2 * ps + p0], U[3 * ps + p0], P.gamma, rho, uu, vv, e_, pr);
    Tref = P.gamma * pr / rho;
  }
  // Q = (u, v, T = gamma p / rho) on [i0-4, i0+BX+4) x [j0-4, j0+BY+4)
  for (int e = tid; e < QX * QY; e += BX * BY) {
    const int a = e % QX, b = e / QX;
    const int i = i0 - HQ + a, j = j0 - HQ + b;
    double uu = 0.0, vv = 0.0, TT = Tref;
    if (i >= -g && i < N0 + g && j >= -g && j < N1 + g) {
      const long long p = pidx(P, i, j);
      double rho, e_, pr;
      ns_flowvar(U[p], U[ps + p], U[2 * ps + p], U[3 * ps + p], P.gamma, rho, uu, vv, e_, pr);
      TT = P.gamma * pr / rho;
    }
    su[b][a] = (T)uu; sv[b][a] = (T)vv; sT[b][a] = (T)(TT - Tref);
  }
  __syncthreads();
  const T two_third = T(2.0 / 3.0), inv_Re = (T)(1.0 / P.Re), inv_Pr = (T)(1.0 / P.Pr);
  const T igm1 = (T)(1.0 / (P.gamma - 1.0));
  // the viscous flux of direction `dir` at (i, j) from the scaled first
  // derivatives of Q (QDerivX on interior rows, QDerivY on interior columns)
  auto vflux = [&](int i, int j, int dir, T* out, int ostride) {
    const int qa = i - (i0 - HQ), qb = j - (j0 - HQ);
    const bool row_int = (j >= 0 && j < N1), col_int = (i >= 0 && i < N0);
    T ux = T(0), vx = T(0), Tx = T(0), uy = T(0), vy = T(0), Ty = T(0);
    if (row_int) {
      const T dxi = (T)dxinv[g + i];
      ux = d4<T>(i, N0, g, [&](int k) { return su[qb][qa + k]; }) * dxi;
      vx = d4<T>(i, N0, g, [&](int k) { return sv[qb][qa + k]; }) * dxi;
      Tx = d4<T>(i, N0, g, [&](int k) { return sT[qb][qa + k]; }) * dxi;
    }
    if (col_int) {
      const T dyi = (T)dxinv[P.W0 + g + j];
      uy = d4<T>(j, N1, g, [&](int k) { return su[qb + k][qa]; }) * dyi;
      vy = d4<T>(j, N1, g, [&](int k) { return sv[qb + k][qa]; }) * dyi;
      Ty = d4<T>(j, N1, g, [&](int k) { return sT[qb + k][qa]; }) * dyi;
    }
    const T uc = su[qb][qa], vc = sv[qb][qa], Tc = sT[qb][qa];
    T mu, kappa;
    visc_coeffs<T>(P, MX ? (T)Tref + Tc : Tc, mu, kappa);
    const T mre = mu * inv_Re, kre = kappa * inv_Re * igm1 * inv_Pr;
    if (dir == 0) {
      const T txx = two_third * mre * (T(2) * ux - vy), txy = mre * (uy + vx);
      out[0] = txx; out[ostride] = txy; out[2 * ostride] = uc * txx + vc * txy + kre * Tx;
    } else {
      const T tyx = mre * (uy + vx), tyy = two_third * mre * (-ux + T(2) * vy);
      out[0] = tyx; out[ostride] = tyy; out[2 * ostride] = uc * tyx + vc * tyy + kre * Ty;
    }
  };
  for (int e = tid; e < BY * FXW; e += BX * BY) {        // x fluxes on interior rows
    const int a = e % FXW, b = e / FXW;
    const int i = i0 - HF + a, j = j0 + b;
    if (j < N1 && i >= -g && i < N0 + g) vflux(i, j, 0, &fx[0][b][a], BY * FXW);
  }
  for (int e = tid; e < FYH * BX; e += BX * BY) {        // y fluxes on interior columns
    const int a = e % BX, b = e / BX;
    const int i = i0 + a, j = j0 - HF + b;
    if (i < N0 && j >= -g && j < N1 + g) vflux(i, j, 1, &fy[0][b][a], FYH * BX);
  }
  __syncthreads();
  const int a = threadIdx.x, b = threadIdx.y;
  const int i = i0 + a, j = j0 + b;
  if (i >= N0 || j >= N1) return;
  const long long p = pidx(P, i, j);
  const T dxi = (T)dxinv[g + i], dyi = (T)dxinv[P.W0 + g + j];
#pragma unroll
  for (int m = 0; m < 3; m++) {
    const T dfx = d4<T>(i, N0, g, [&](int k) { return fx[m][b][a + HF + k]; });
    const T dfy = d4<T>(j, N1, g, [&](int k) { return fy[m][b + HF + k][a]; });
    const T par = dxi * dfx + dyi * dfy;
    rhs[(m + 1) * ps + p] += (double)par;
  }
  if (do_chem) {
    const double t = *tdev + cstage * P.dt;
    chem_source_point<T>(P, U, p, pulse_factor(P, t), imap[p], rhs, hnu);
  }
}

// BCSpongeSource (BCSponge.c:42-73) added to the RHS: at the interior points
// of the box [is0, ie0) x [is1, ie1), rhs_v -= sigma (u_v - uref_v), sigma the
// ramp value at the point's index along the sponge dimension.
__global__ void k_sponge(DevParams P, const double* __restrict__ U, double* __restrict__ rhs, int dim, int is0,
                         int ie0, int is1, int ie1, const double* __restrict__ sigma,
                         const double* __restrict__ uref) {
  const int n0 = ie0 - is0, n1 = ie1 - is1;
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)n0 * n1) return;
  const int i = is0 + (int)(k % n0), j = is1 + (int)(k / n0);
  const long long p = pidx(P, i, j);
  const double sg = sigma[dim == 0 ? i - is0 : j - is1];
  for (int v = 0; v < P.nvars; v++) rhs[v * P.ps + p] -= sg * (U[v * P.ps + p] - uref[v]);
}

// chemistry source alone (1D, or 2D without viscosity)
template <bool MX>
__global__ void k_source(DevParams P, const double* __restrict__ U, const double* __restrict__ imap,
                         const double* __restrict__ tdev, double cstage, double* __restrict__ rhs,
                         double* __restrict__ hnu) {
  long long n = (long long)P.N0 * P.N1;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int i = (int)(idx % P.N0), j = (int)(idx / P.N0);
  long long p = pidx(P, i, j);
  const double t = *tdev + cstage * P.dt;
  chem_source_point<typename std::conditional<MX, float, double>::type>(P, U, p, pulse_factor(P, t), imap[p], rhs,
                                                                        hnu);
}

__global__ void k_advance_time(double* tdev, double dt) { *tdev += dt; }

// =================================================================== batched
// tridiagLU with the reference's [row * ns + sys] layout: one thread per
// system, serial Thomas (tridiagLU.c:133-153, 242-262).  Operator-level entry
// point for parity tests; the fused CRWENO path does not use it.
__global__ void k_tridiag_serial(double* a, double* b, double* c, double* x, int n, int ns, int* err) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= ns) return;
  int bad = 0;
  for (int i = 1; i < n; i++) {
    double bm = b[(long long)(i - 1) * ns + d];
    if (bm == 0.0) { bad = 1; break; }
    double f = a[(long long)i * ns + d] / bm;
    b[(long long)i * ns + d] -= f * c[(long long)(i - 1) * ns + d];
    a[(long long)i * ns + d] = -f * a[(long long)(i - 1) * ns + d];
    x[(long long)i * ns + d] -= f * x[(long long)(i - 1) * ns + d];
  }
  if (!bad) {
    const double x0 = x[d];
    long long e = (long long)(n - 1) * ns + d;
    if (b[e] == 0.0) bad = 1;
    else x[e] = (x[e] - a[e] * x0) / b[e];
    for (int i = n - 2; i >= 0 && !bad; i--) {
      long long r = (long long)i * ns + d;
      if (b[r] == 0.0) { bad = 1; break; }
      x[r] = (x[r] - c[r] * x[r + ns] - a[r] * (i == 0 ? x[r] : x0)) / b[r];
    }
  }
  if (bad) atomicOr(err, 1);
}


// ======================================================= operator-level only
// Upwind at every interface of direction DIR into an interface array (SoA);
// the fused path uses k_upwind_div instead.
template <int MODEL, int UPW, int DIR>
__global__ void k_upwind_iface(DevParams P, const double* __restrict__ U, const double* __restrict__ uL,
                               const double* __restrict__ uR, const double* __restrict__ fL,
                               const double* __restrict__ fR, double* __restrict__ fI) {
  constexpr int NF = Flow<MODEL>::NF;
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= P.nint[DIR]) return;
  int i, l;
  iface_decode<DIR>(P, q, i, l);
  const long long pL = cell_of<DIR>(P, i - 1, l), pR = cell_of<DIR>(P, i, l);
  double a[4], b[4], c[4], d[4], ucl[4], ucr[4], fi[4], spa;
  int spm;
  for (int m = 0; m < NF; m++) {
    a[m] = uL[m * P.pis + q]; b[m] = uR[m * P.pis + q]; c[m] = fL[m * P.pis + q]; d[m] = fR[m * P.pis + q];
    ucl[m] = U[m * P.ps + pL]; ucr[m] = U[m * P.ps + pR];
  }
  upwind_flow<MODEL, UPW, double>(a, b, c, d, ucl, ucr, P.gamma, DIR, fi, &spa, &spm);
  for (int m = 0; m < NF; m++) fI[m * P.pis + q] = fi[m];
  for (int m = NF; m < P.nvars; m++)
    fI[m * P.pis + q] = upwind_species(spm, spa, uL[m * P.pis + q], uR[m * P.pis + q], fL[m * P.pis + q], fR[m * P.pis + q]);
}

// FirstDerivativeFirstOrder (FirstDerivativeFirstOrder.c:40-100), or with
// P.par4 FirstDerivativeFourthOrderCentral (d4), on an AoS array with nv
// values per point: lines along dir that are interior in the other
// dimension, one-sided at the extreme ghost points.
__global__ void k_first_deriv(DevParams P, double* __restrict__ Df, const double* __restrict__ f, int dir,
                              int bias, int nv) {
  const int N = dir == 0 ? P.N0 : P.N1, nl = P.ndims == 1 ? 1 : (dir == 0 ? P.N1 : P.N0);
  const int len = N + 2 * P.ghosts;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)len * nl) return;
  int ii = (int)(idx % len) - P.ghosts, l = (int)(idx / len);
  auto at = [&](int i) -> long long { return dir == 0 ? pidx(P, i, l) : pidx(P, l, i); };
  const int mx = bias > 0 ? bias : 0, mn = bias < 0 ? bias : 0;
  if (P.par4) {
    for (int v = 0; v < nv; v++)
      Df[at(ii) * nv + v] = d4<double>(ii, N, P.ghosts, [&](int k) { return f[at(ii + k) * nv + v]; });
    return;
  }
  for (int v = 0; v < nv; v++) {
    double r;
    if (ii == -P.ghosts) r = f[at(ii + 1) * nv + v] - f[at(ii) * nv + v];
    else if (ii == N + P.ghosts - 1) r = f[at(ii) * nv + v] - f[at(ii - 1) * nv + v];
    else r = mx * f[at(ii + 1) * nv + v] - bias * f[at(ii) * nv + v] + mn * f[at(ii - 1) * nv + v];
    Df[at(ii) * nv + v] = r;
  }
}

// ================================================================ launchers
static inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

__global__ void k_reciprocal(const double* __restrict__ x, double* __restrict__ y, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = rcp_nr(x[i]);
}
void launch_reciprocal(const double* x, double* y, long long n, cudaStream_t s) {
  k_reciprocal<<<nblk(n, 256), 256, 0, s>>>(x, y, n);
}

void launch_aos_to_soa(const double* aos, double* soa, long long npg, int nv, long long ps, cudaStream_t s) {
  k_aos_to_soa<<<nblk(npg * nv, 256), 256, 0, s>>>(aos, soa, npg, nv, ps);
}
void launch_soa_to_aos(const double* soa, double* aos, long long npg, int nv, long long ps, cudaStream_t s) {
  k_soa_to_aos<<<nblk(npg * nv, 256), 256, 0, s>>>(soa, aos, npg, nv, ps);
}
void launch_soa_to_interior(const DevParams& P, const double* soa, double* out, cudaStream_t s) {
  k_soa_to_interior<<<nblk((long long)P.N0 * P.N1 * P.nvars, 256), 256, 0, s>>>(P, soa, out);
}
void launch_interior_to_soa(const DevParams& P, const double* in, double* soa, cudaStream_t s) {
  k_interior_to_soa<<<nblk((long long)P.N0 * P.N1 * P.nvars, 256), 256, 0, s>>>(P, in, soa);
}
void launch_iface_aos_to_soa(const double* aos, double* soa, long long ni, int nv, long long pis, cudaStream_t s) {
  k_iface_aos_to_soa<<<nblk(ni * nv, 256), 256, 0, s>>>(aos, soa, ni, nv, pis);
}
void launch_iface_soa_to_aos(const double* soa, double* aos, long long ni, int nv, long long pis, cudaStream_t s) {
  k_iface_soa_to_aos<<<nblk(ni * nv, 256), 256, 0, s>>>(soa, aos, ni, nv, pis);
}
void launch_transpose_flux_y(const DevParams& P, const double* U, double* UT, double* FT, cudaStream_t s) {
  dim3 grid(nblk(P.W0, 32), nblk(P.W1, 32)), blk(32, 8);
  k_transpose_flux_y<<<grid, blk, 0, s>>>(P, U, UT, FT);
}
void launch_transpose(const DevParams& P, const double* in, double* out, cudaStream_t s) {
  dim3 grid(nblk(P.W0, 32), nblk(P.W1, 32), P.nvars), blk(32, 8);
  k_transpose_planes<<<grid, blk, 0, s>>>(in, out, P.W0, P.W1, P.ps);
}
DevParams transposed_params(const DevParams& P) {
  DevParams T = P;
  T.N0 = P.N1; T.N1 = P.N0;
  T.W0 = P.W1; T.W1 = P.W0;
  T.nint[0] = P.nint[1]; T.nint[1] = P.nint[0];
  return T;
}
void launch_bc(const DevParams& P, double* u, const Zone& z, cudaStream_t s) {
  long long n = (long long)(z.ie[0] - z.is[0]) * (z.ie[1] - z.is[1]);
  if (n <= 0) return;
  k_bc_zone<<<nblk(n, 128), 128, 0, s>>>(P, u, z);
}
void launch_stage(long long n, double* Us, const double* u, const double* const* d, const double* a, int nterms,
                  cudaStream_t s) {
  k_stage<<<nblk(n, 256), 256, 0, s>>>(n, Us, u, nterms > 0 ? d[0] : nullptr, nterms > 0 ? a[0] : 0.0,
                                        nterms > 1 ? d[1] : nullptr, nterms > 1 ? a[1] : 0.0,
                                        nterms > 2 ? d[2] : nullptr, nterms > 2 ? a[2] : 0.0, nterms);
}
void launch_update(const DevParams& P, double* u, const double* const* d, const double* b, int ns, double* norm_acc,
                   cudaStream_t s) {
  long long n = (long long)P.nvars * P.ps;
  if (ns >= 1 && ns <= 4) {   // plane strides are multiples of 32: whole double2 pairs within a plane
    const long long n2 = n / 2;
    const double* dd[4] = {d[0], ns > 1 ? d[1] : nullptr, ns > 2 ? d[2] : nullptr, ns > 3 ? d[3] : nullptr};
    const double bb[4] = {b[0], ns > 1 ? b[1] : 0.0, ns > 2 ? b[2] : 0.0, ns > 3 ? b[3] : 0.0};
#define PIAFS_UPD(NS) k_update2<NS><<<nblk(n2, 256), 256, 0, s>>>(P, u, dd[0], bb[0], dd[1], bb[1], dd[2], bb[2], \
                                                                 dd[3], bb[3], norm_acc)
    switch (ns) {
      case 1: PIAFS_UPD(1); break;
      case 2: PIAFS_UPD(2); break;
      case 3: PIAFS_UPD(3); break;
      default: PIAFS_UPD(4); break;
    }
#undef PIAFS_UPD
    return;
  }
  k_update<<<nblk(n, 256), 256, 0, s>>>(P, u, d[0], b[0], ns > 1 ? d[1] : nullptr, ns > 1 ? b[1] : 0.0,
                                         ns > 2 ? d[2] : nullptr, ns > 2 ? b[2] : 0.0, ns > 3 ? d[3] : nullptr,
                                         ns > 3 ? b[3] : 0.0, ns, norm_acc);
}
void launch_cfl(const DevParams& P, const double* u, const double* dxinv, unsigned long long* out, cudaStream_t s) {
  k_cfl<<<nblk((long long)P.N0 * P.N1, 256), 256, 0, s>>>(P, u, dxinv, out);
}
void launch_flux(const DevParams& P, const double* U, double* F, int dir, cudaStream_t s) {
  unsigned nb = nblk(P.npg, 256);
  if (P.model == NS2D) {
    if (dir == 0) k_flux<NS2D, 0><<<nb, 256, 0, s>>>(P, U, F);
    else k_flux<NS2D, 1><<<nb, 256, 0, s>>>(P, U, F);
  } else {
    k_flux<EULER1D, 0><<<nb, 256, 0, s>>>(P, U, F);
  }
}
void launch_weno5(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                  int dir, cudaStream_t s) {
  long long n = P.nint[dir] * P.nvars;
  if (P.mixed) {
    if (dir == 0) k_weno5<0, true><<<nblk(n, 256), 256, 0, s>>>(P, U, F, uL, uR, fL, fR);
    else k_weno5<1, true><<<nblk(n, 256), 256, 0, s>>>(P, U, F, uL, uR, fL, fR);
  } else {
    if (dir == 0) k_weno5<0, false><<<nblk(n, 256), 256, 0, s>>>(P, U, F, uL, uR, fL, fR);
    else k_weno5<1, false><<<nblk(n, 256), 256, 0, s>>>(P, U, F, uL, uR, fL, fR);
  }
}

void launch_weno5_char(const DevParams& P, const double* U, const double* F, double* uL, double* uR, double* fL,
                       double* fR, int dir, cudaStream_t s) {
  const unsigned nb = nblk(P.nint[dir], 128);
  if (P.model == NS2D) {
    if (dir == 0) k_weno5_char<NS2D, 0><<<nb, 128, 0, s>>>(P, U, F, uL, uR, fL, fR);
    else k_weno5_char<NS2D, 1><<<nb, 128, 0, s>>>(P, U, F, uL, uR, fL, fR);
  } else {
    k_weno5_char<EULER1D, 0><<<nb, 128, 0, s>>>(P, U, F, uL, uR, fL, fR);
  }
}

template <int MODEL, int UPW>
static void upwind_div_dir(const DevParams& P, const double* U, const void* uL, const void* uR, const void* fL,
                           const void* fR, const double* dxinv, double* rhs, int dir, int mode, cudaStream_t s) {
  // the interface-flux tile holds nvars x (tile + 1) values: allow more than
  // the 48 KB default for many-species decks
  if (dir == 0) {
    dim3 grid(nblk(P.N0, 128), P.N1), blk(128, 1);
    if constexpr (MODEL == EULER1D) {
      if (P.mixed) {
        raise_smem_limit<k_upwind_div<MODEL, UPW, 0, true>>(200 * 1024);
        k_upwind_div<MODEL, UPW, 0, true><<<grid, blk, (size_t)P.nvars * 129 * sizeof(float), s>>>(
            P, U, uL, uR, fL, fR, dxinv, rhs, mode);
        return;
      }
    }
    {
      raise_smem_limit<k_upwind_div<MODEL, UPW, 0, false>>(200 * 1024);
      k_upwind_div<MODEL, UPW, 0, false><<<grid, blk, (size_t)P.nvars * 129 * sizeof(double), s>>>(
          P, U, uL, uR, fL, fR, dxinv, rhs, mode);
    }
  } else {
    dim3 grid(nblk(P.N0, 32), nblk(P.N1, 8)), blk(32, 8);
    raise_smem_limit<k_upwind_div<MODEL, UPW, 1, false>>(200 * 1024);
    k_upwind_div<MODEL, UPW, 1, false><<<grid, blk, (size_t)P.nvars * 9 * 32 * sizeof(double), s>>>(
        P, U, uL, uR, fL, fR, dxinv, rhs, mode);
  }
}
template <int MODEL>
static void upwind_div_model(const DevParams& P, const double* U, const void* uL, const void* uR, const void* fL,
                             const void* fR, const double* dxinv, double* rhs, int dir, int mode, cudaStream_t s) {
  switch (P.upwind) {
    case UPW_ROE: upwind_div_dir<MODEL, UPW_ROE>(P, U, uL, uR, fL, fR, dxinv, rhs, dir, mode, s); break;
    case UPW_RF: upwind_div_dir<MODEL, UPW_RF>(P, U, uL, uR, fL, fR, dxinv, rhs, dir, mode, s); break;
    case UPW_LLF: upwind_div_dir<MODEL, UPW_LLF>(P, U, uL, uR, fL, fR, dxinv, rhs, dir, mode, s); break;
    default: upwind_div_dir<MODEL, UPW_RUSANOV>(P, U, uL, uR, fL, fR, dxinv, rhs, dir, mode, s); break;
  }
}

void launch_upwind_div(const DevParams& P, const double* U, const void* uL, const void* uR, const void* fL,
                       const void* fR, const double* dxinv, double* rhs, int dir, int mode, cudaStream_t s) {
  if (P.model == NS2D) upwind_div_model<NS2D>(P, U, uL, uR, fL, fR, dxinv, rhs, dir, mode, s);
  else upwind_div_model<EULER1D>(P, U, uL, uR, fL, fR, dxinv, rhs, dir, mode, s);
}

template <int UPW, bool YT, bool MX, bool HYIN>
static void upwind_div2d_u(const DevParams& P, const double* U, const double* UT, const void* const* xi,
                           const void* const* yi, const double* dxinv, double* rhs, int neg, const void* hyin,
                           int n0, cudaStream_t s) {
  raise_smem_limit<k_upwind_div2d<UPW, YT, MX, HYIN>>(200 * 1024);
  dim3 grid(nblk(P.N0, 16), nblk(P.N1, 15));
  size_t smem = (size_t)P.nvars * (17 * 15 + (HYIN ? 0 : 16 * 17)) * (MX ? sizeof(float) : sizeof(double));
  const void* none = nullptr;
  k_upwind_div2d<UPW, YT, MX, HYIN><<<grid, 256, smem, s>>>(P, U, UT, xi[0], xi[1], xi[2], xi[3],
                                                             HYIN ? none : yi[0], HYIN ? none : yi[1],
                                                             HYIN ? none : yi[2], HYIN ? none : yi[3], dxinv, rhs,
                                                             neg, hyin, n0);
}
template <bool YT, bool MX, bool HYIN>
static void upwind_div2d_yt(const DevParams& P, const double* U, const double* UT, const void* const* xi,
                            const void* const* yi, const double* dxinv, double* rhs, int neg, const void* hyin,
                            int n0, cudaStream_t s) {
  switch (P.upwind) {
    case UPW_ROE: upwind_div2d_u<UPW_ROE, YT, MX, HYIN>(P, U, UT, xi, yi, dxinv, rhs, neg, hyin, n0, s); break;
    case UPW_RF: upwind_div2d_u<UPW_RF, YT, MX, HYIN>(P, U, UT, xi, yi, dxinv, rhs, neg, hyin, n0, s); break;
    case UPW_RUSANOV: upwind_div2d_u<UPW_RUSANOV, YT, MX, HYIN>(P, U, UT, xi, yi, dxinv, rhs, neg, hyin, n0, s); break;
    default: upwind_div2d_u<UPW_LLF, YT, MX, HYIN>(P, U, UT, xi, yi, dxinv, rhs, neg, hyin, n0, s); break;
  }
}
void launch_upwind_div2d(const DevParams& P, const double* U, const double* UT, const void* const* xi,
                         const void* const* yi, const double* dxinv, double* rhs, int neg, cudaStream_t s) {
  if (P.mixed) {
    if (UT) upwind_div2d_yt<true, true, false>(P, U, UT, xi, yi, dxinv, rhs, neg, nullptr, 0, s);
    else upwind_div2d_yt<false, true, false>(P, U, UT, xi, yi, dxinv, rhs, neg, nullptr, 0, s);
  } else {
    if (UT) upwind_div2d_yt<true, false, false>(P, U, UT, xi, yi, dxinv, rhs, neg, nullptr, 0, s);
    else upwind_div2d_yt<false, false, false>(P, U, UT, xi, yi, dxinv, rhs, neg, nullptr, 0, s);
  }
}
void launch_upwind_div2d_hy(const DevParams& P, const double* U, const void* const* xi, const double* dxinv,
                            const void* hy, int n0, double* rhs, int neg, cudaStream_t s) {
  const void* const* none = xi;   // y interface arrays are not read
  if (P.mixed) upwind_div2d_yt<false, true, true>(P, U, nullptr, xi, none, dxinv, rhs, neg, hy, n0, s);
  else upwind_div2d_yt<false, false, true>(P, U, nullptr, xi, none, dxinv, rhs, neg, hy, n0, s);
}
template <int UPW, bool MX>
static void slab_upwind_y_u(const DevParams& P, const double* UT, const void* const* yi, const double* dyinv,
                            void* hy, int n1, cudaStream_t s) {
  raise_smem_limit<k_slab_upwind_y<UPW, MX>>(200 * 1024);
  dim3 grid(nblk(P.N0, 16), nblk(P.N1, 15));
  size_t smem = (size_t)P.nvars * (16 * 17) * (MX ? sizeof(float) : sizeof(double));
  k_slab_upwind_y<UPW, MX><<<grid, 256, smem, s>>>(P, UT, yi[0], yi[1], yi[2], yi[3], dyinv, hy, n1);
}
template <bool MX>
static void slab_upwind_y_m(const DevParams& P, const double* UT, const void* const* yi, const double* dyinv,
                            void* hy, int n1, cudaStream_t s) {
  switch (P.upwind) {
    case UPW_ROE: slab_upwind_y_u<UPW_ROE, MX>(P, UT, yi, dyinv, hy, n1, s); break;
    case UPW_RF: slab_upwind_y_u<UPW_RF, MX>(P, UT, yi, dyinv, hy, n1, s); break;
    case UPW_RUSANOV: slab_upwind_y_u<UPW_RUSANOV, MX>(P, UT, yi, dyinv, hy, n1, s); break;
    default: slab_upwind_y_u<UPW_LLF, MX>(P, UT, yi, dyinv, hy, n1, s); break;
  }
}
void launch_slab_upwind_y(const DevParams& P, const double* UT, const void* const* yi, const double* dyinv, void* hy,
                          int n1, cudaStream_t s) {
  if (P.mixed) slab_upwind_y_m<true>(P, UT, yi, dyinv, hy, n1, s);
  else slab_upwind_y_m<false>(P, UT, yi, dyinv, hy, n1, s);
}

void launch_visc_source(const DevParams& P, const double* U, const double* dxinv, const double* imap,
                        const double* tdev, double cstage, double* rhs, int do_visc, int do_chem, cudaStream_t s,
                        double* hnu) {
  do_visc = do_visc && P.ndims == 2 && P.viscous;
  do_chem = do_chem && P.chem;
  if (do_visc) {
    dim3 grid(nblk(P.N0, 32), nblk(P.N1, 8)), blk(32, 8);
    if (P.par4) {
      if (P.mixed) k_visc4_source<true><<<grid, blk, 0, s>>>(P, U, dxinv, imap, tdev, cstage, rhs, do_chem, hnu);
      else k_visc4_source<false><<<grid, blk, 0, s>>>(P, U, dxinv, imap, tdev, cstage, rhs, do_chem, hnu);
    } else if (P.mixed) k_visc_source<true><<<grid, blk, 0, s>>>(P, U, dxinv, imap, tdev, cstage, rhs, do_chem, hnu);
    else k_visc_source<false><<<grid, blk, 0, s>>>(P, U, dxinv, imap, tdev, cstage, rhs, do_chem, hnu);
  } else if (do_chem) {
    const unsigned nb = nblk((long long)P.N0 * P.N1, 256);
    if (P.mixed) k_source<true><<<nb, 256, 0, s>>>(P, U, imap, tdev, cstage, rhs, hnu);
    else k_source<false><<<nb, 256, 0, s>>>(P, U, imap, tdev, cstage, rhs, hnu);
  }
}

void launch_sponge(const DevParams& P, const double* U, double* rhs, int dim, const int* is, const int* ie,
                   const double* sigma, const double* uref, cudaStream_t s) {
  const long long n = (long long)(ie[0] - is[0]) * (ie[1] - is[1]);
  if (n <= 0) return;
  k_sponge<<<nblk(n, 256), 256, 0, s>>>(P, U, rhs, dim, is[0], ie[0], is[1], ie[1], sigma, uref);
}

void launch_advance_time(double* tdev, double dt, cudaStream_t s) { k_advance_time<<<1, 1, 0, s>>>(tdev, dt); }

template <int MODEL, int UPW>
static void upwind_iface_m(const DevParams& P, const double* U, const double* uL, const double* uR, const double* fL,
                           const double* fR, double* fI, int dir, cudaStream_t s) {
  unsigned nb = nblk(P.nint[dir], 128);
  if (dir == 0) k_upwind_iface<MODEL, UPW, 0><<<nb, 128, 0, s>>>(P, U, uL, uR, fL, fR, fI);
  else k_upwind_iface<MODEL, UPW, 1><<<nb, 128, 0, s>>>(P, U, uL, uR, fL, fR, fI);
}
template <int MODEL>
static void upwind_iface_u(const DevParams& P, const double* U, const double* uL, const double* uR, const double* fL,
                           const double* fR, double* fI, int dir, cudaStream_t s) {
  switch (P.upwind) {
    case UPW_ROE: upwind_iface_m<MODEL, UPW_ROE>(P, U, uL, uR, fL, fR, fI, dir, s); break;
    case UPW_RF: upwind_iface_m<MODEL, UPW_RF>(P, U, uL, uR, fL, fR, fI, dir, s); break;
    case UPW_LLF: upwind_iface_m<MODEL, UPW_LLF>(P, U, uL, uR, fL, fR, fI, dir, s); break;
    default: upwind_iface_m<MODEL, UPW_RUSANOV>(P, U, uL, uR, fL, fR, fI, dir, s); break;
  }
}
void launch_upwind_iface(const DevParams& P, const double* U, const double* uL, const double* uR, const double* fL,
                         const double* fR, double* fI, int dir, cudaStream_t s) {
  if (P.model == NS2D) upwind_iface_u<NS2D>(P, U, uL, uR, fL, fR, fI, dir, s);
  else upwind_iface_u<EULER1D>(P, U, uL, uR, fL, fR, fI, dir, s);
}
void launch_first_deriv(const DevParams& P, double* Df, const double* f, int dir, int bias, int nv, cudaStream_t s) {
  const int N = dir == 0 ? P.N0 : P.N1, nl = P.ndims == 1 ? 1 : (dir == 0 ? P.N1 : P.N0);
  long long n = (long long)(N + 2 * P.ghosts) * nl;
  k_first_deriv<<<nblk(n, 128), 128, 0, s>>>(P, Df, f, dir, bias, nv);
}

void launch_tridiag(double* a, double* b, double* c, double* x, int n, int ns, int* err, cudaStream_t s) {
  k_tridiag_serial<<<nblk(ns, 128), 128, 0, s>>>(a, b, c, x, n, ns, err);
}

}  // namespace piafs
