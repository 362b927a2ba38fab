// Launcher interface of the device kernels (kernels.cu).
#pragma once
#include <atomic>
#include <cuda_runtime.h>
#include "common.cuh"

namespace piafs {

// Raise a kernel's dynamic shared-memory limit, once per device.
template <auto Kernel>
inline void raise_smem_limit(int bytes) {
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load() & bit) return;
  cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  done.fetch_or(bit);
}

// One boundary zone with its index extents resolved (single rank):
// [is[d], ie[d]) per dimension, ghost slab along `dim`
// (InitializeBoundaries.c:296-378), and its data
// (InitializeBoundaries.c:106-168): wall or inflow velocity, inflow density,
// outflow / inflow pressure, and in device memory the Dirichlet state (one
// value per variable) or the inflow passive scalars (variables 4..nvars-1).
struct Zone {
  int type, dim, face;
  int is[2], ie[2];
  double vel[2];
  double rho, pres;
  const double* val;
};

#ifdef __CUDACC__
// Boundary values at ghost point (g0, g1) of zone z (BCPeriodic.c,
// BCExtrapolate.c, BCSlipWall.c and the boundaries below): reads the zone's
// source point of u (SoA planes) and writes the ghost's variables to
// out[v * ostride] -- all of them, or for the flow boundaries of the
// Euler / Navier-Stokes models the flow variables (and the passive scalars
// of an inflow) only; the others stay untouched.  The periodic source keeps the zone-relative index in
// the other dimension, as the reference does.
__device__ __forceinline__ void bc_point(const DevParams& P, const Zone& z, const double* u, int g0, int g1,
                                         double* out, long long ostride) {
  const int gi[2] = {g0, g1};
  const int d = z.dim, b = gi[d] - z.is[d];
  int src[2] = {g0, g1};
  const int Nd = d == 0 ? P.N0 : P.N1;
  if (z.type == BC_PERIODIC) {
    if (P.ndims == 2) src[1 - d] = gi[1 - d] - z.is[1 - d];
    src[d] = z.face == 1 ? b + Nd - P.ghosts : b;
  } else {
    src[d] = z.face == 1 ? P.ghosts - 1 - b : Nd - b - 1;
  }
  const long long p2 = pidx(P, src[0], src[1]);
  if (z.type == BC_DIRICHLET) {        // BCDirichlet.c:26-39
    for (int v = 0; v < P.nvars; v++) out[v * ostride] = z.val[v];
    return;
  }
  if (z.type == BC_REFLECT) {          // BCReflect.c:27-50
    for (int v = 0; v < P.nvars; v++) out[v * ostride] = -1.0 * u[v * P.ps + p2];
    return;
  }
  if (z.type >= BC_NOSLIP) {
    // BCNoslipWall.c:41-78, BCSubsonicInflow.c:41-88, BCSubsonicOutflow.c:41-80,
    // BCSubsonicAmbivalent.c:46-132, BCSupersonicInflow.c:38-68,
    // BCSupersonicOutflow.c:41-82: the ghost's density, velocity and pressure
    // from the mirrored interior point and the zone's data; energy from them
    // with the boundary gamma; inflows also set the passive scalars, the
    // others leave them.  The reference has these for 2D only and leaves the
    // ghosts of other dimensionalities as they are.
    if (P.ndims != 2) return;
    const double g = P.bc_gamma, igm1 = 1.0 / (g - 1.0);
    double rho = 0.0, uv = 0.0, vv = 0.0, e, pr = 0.0;
    if (z.type != BC_SUP_INFLOW)
      ns_flowvar(u[p2], u[P.ps + p2], u[2 * P.ps + p2], u[3 * P.ps + p2], g, rho, uv, vv, e, pr);
    int type = z.type;
    if (type == BC_SUB_AMBIVALENT) {
      // inflow or outflow by the sign of the normal velocity at the face,
      // extrapolated from the first two interior points (BCSubsonicAmbivalent.c:70-86)
      int a[2] = {g0, g1}, b2[2] = {g0, g1};
      a[d] = z.face == 1 ? 0 : Nd - 1;
      b2[d] = z.face == 1 ? 1 : Nd - 2;
      const long long q1 = pidx(P, a[0], a[1]), q2 = pidx(P, b2[0], b2[1]);
      double r1, u1, v1, e1, p1, r2, u2, v2, e2, pq2;
      ns_flowvar(u[q1], u[P.ps + q1], u[2 * P.ps + q1], u[3 * P.ps + q1], g, r1, u1, v1, e1, p1);
      ns_flowvar(u[q2], u[P.ps + q2], u[2 * P.ps + q2], u[3 * P.ps + q2], g, r2, u2, v2, e2, pq2);
      const double ub = 1.5 * u1 - 0.5 * u2, vb = 1.5 * v1 - 0.5 * v2;
      const double nx = (d == 0 ? 1.0 : 0.0) * (double)z.face, ny = (d == 1 ? 1.0 : 0.0) * (double)z.face;
      type = (ub * nx + vb * ny > 0) ? BC_SUB_INFLOW : BC_SUB_OUTFLOW;
    }
    double rg, ug, vg, pg;
    switch (type) {
      case BC_NOSLIP: rg = rho; pg = pr; ug = 2.0 * z.vel[0] - uv; vg = 2.0 * z.vel[1] - vv; break;
      case BC_SUB_INFLOW: rg = z.rho; pg = pr; ug = z.vel[0]; vg = z.vel[1]; break;
      case BC_SUB_OUTFLOW: rg = rho; pg = z.pres; ug = uv; vg = vv; break;
      case BC_SUP_INFLOW: rg = z.rho; pg = z.pres; ug = z.vel[0]; vg = z.vel[1]; break;
      default: rg = rho; pg = pr; ug = uv; vg = vv; break;   // supersonic outflow
    }
    out[0] = rg;
    out[ostride] = rg * ug;
    out[2 * ostride] = rg * vg;
    out[3 * ostride] = igm1 * pg + 0.5 * rg * (ug * ug + vg * vg);
    // the ambivalent zone reads no scalars (BCSubsonicAmbivalent.c:118-127)
    if ((z.type == BC_SUB_INFLOW || z.type == BC_SUP_INFLOW) && z.val)
      for (int v = 4; v < P.nvars; v++) out[v * ostride] = z.val[v - 4];
    return;
  }
  if (z.type == BC_SLIPWALL) {
    const double g = P.bc_gamma, igm1 = 1.0 / (g - 1.0);
    if (P.ndims == 1) {
      double rho, uv, e, pr;
      eu_flowvar(u[p2], u[P.ps + p2], u[2 * P.ps + p2], g, rho, uv, e, pr);
      const double ug = 2.0 * z.vel[0] - uv;
      out[0] = rho;
      out[ostride] = rho * ug;
      out[2 * ostride] = igm1 * pr + 0.5 * rho * ug * ug;
    } else {
      double rho, uv, vv, e, pr, ug, vg;
      ns_flowvar(u[p2], u[P.ps + p2], u[2 * P.ps + p2], u[3 * P.ps + p2], g, rho, uv, vv, e, pr);
      if (d == 0) { ug = 2.0 * z.vel[0] - uv; vg = vv; }
      else        { ug = uv; vg = 2.0 * z.vel[1] - vv; }
      out[0] = rho;
      out[ostride] = rho * ug;
      out[2 * ostride] = rho * vg;
      out[3 * ostride] = igm1 * pr + 0.5 * rho * (ug * ug + vg * vg);
    }
  } else {
    for (int v = 0; v < P.nvars; v++) out[v * ostride] = u[v * P.ps + p2];
  }
}
#endif

void launch_aos_to_soa(const double* aos, double* soa, long long npg, int nv, long long ps, cudaStream_t s);
void launch_soa_to_aos(const double* soa, double* aos, long long npg, int nv, long long ps, cudaStream_t s);
void launch_soa_to_interior(const DevParams& P, const double* soa, double* out, cudaStream_t s);
void launch_interior_to_soa(const DevParams& P, const double* in, double* soa, cudaStream_t s);
void launch_iface_aos_to_soa(const double* aos, double* soa, long long ni, int nv, long long pis, cudaStream_t s);
void launch_iface_soa_to_aos(const double* soa, double* aos, long long ni, int nv, long long pis, cudaStream_t s);
void launch_bc(const DevParams& P, double* u, const Zone& z, cudaStream_t s);
// 2D only: plane-wise transpose of a ghosted state (j fastest in `out`) and
// the parameters that describe the transposed grid (dimensions swapped)
void launch_transpose(const DevParams& P, const double* in, double* out, cudaStream_t s);
// the transposed state of a 2D Navier-Stokes grid and its y flux, both in
// the transposed layout, in one pass
void launch_transpose_flux_y(const DevParams& P, const double* U, double* UT, double* FT, cudaStream_t s);
DevParams transposed_params(const DevParams& P);
void launch_stage(long long n, double* Us, const double* u, const double* const* d, const double* a, int nterms,
                  cudaStream_t s);
void launch_update(const DevParams& P, double* u, const double* const* d, const double* b, int ns, double* norm_acc,
                   cudaStream_t s);
void launch_cfl(const DevParams& P, const double* u, const double* dxinv, unsigned long long* out, cudaStream_t s);
void launch_flux(const DevParams& P, const double* U, double* F, int dir, cudaStream_t s);
// WENO5 interface values; doubles, or floats relative to each line's first
// value when P.mixed
// WENO5 on characteristic variables (FP64; all four interface arrays)
void launch_weno5_char(const DevParams& P, const double* U, const double* F, double* uL, double* uR, double* fL,
                       double* fR, int dir, cudaStream_t s);
void launch_weno5(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                  int dir, cudaStream_t s);
// CRWENO5 interface values (crweno.cu); -1 if a line is too long.  The
// interface arrays hold doubles, or floats relative to each line's first
// value when P.mixed (x-direction lines only).
int crweno_rows_per_thread(int N);
// CTAs per line (a thread-block cluster beyond one CTA's 4097 interfaces);
// -1 if a line is too long
int crweno_cluster_size(int N);
int launch_crweno(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL, void* fR,
                  int dir, int* err, cudaStream_t s);
// the same for lines of up to 4097 interfaces, one CTA per line
// (crweno_line.cu): true if it serves lines of N points; -1 from the
// launcher otherwise
bool crweno_line_fits(int N);
int launch_crweno_line(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL,
                       void* fR, int dir, int* err, cudaStream_t s);
// longer lines (up to 32769 interfaces) by clusters of CTAs that solve their
// segments' separator systems locally and couple them through one small
// system (crweno_line.cu); -1 if the line is not one of those
int launch_crweno_seg(const DevParams& P, const double* U, const double* F, void* uL, void* uR, void* fL,
                      void* fR, int dir, int* err, cudaStream_t s);
// CRWENO5 on characteristic variables (crweno_char.cu; 1D Euler and 2D
// Navier-Stokes without chemistry, FP64): all four interface arrays of
// direction dir; scratch holds crweno_char_scratch(P) doubles; *err is set on
// a zero pivot of a block inverse
long long crweno_char_scratch(const DevParams& P);
void launch_crweno_char(const DevParams& P, const double* U, const double* F, double* uL, double* uR, double* fL,
                        double* fR, int dir, double* scratch, int* err, cudaStream_t s);
// mode 0: rhs = -hyp_x; 1: rhs = -((-rhs) + hyp_y); 2: out = hyp_x; 3: out += hyp_y
// (interface arrays as written by launch_weno5 / launch_crweno; the mixed
// variant covers the 1D x direction, 2D goes through launch_upwind_div2d)
void launch_upwind_div(const DevParams& P, const double* U, const void* uL, const void* uR, const void* fL,
                       const void* fR, const double* dxinv, double* rhs, int dir, int mode, cudaStream_t s);
// both directions of a 2D hyperbolic term in one pass: xi / yi are the
// (uL, uR, fL, fR) interface arrays of x and y; y in the transposed layout
// with cell values from UT when UT is given.  rhs = -hyp (neg) or hyp.
void launch_upwind_div2d(const DevParams& P, const double* U, const double* UT, const void* const* xi,
                         const void* const* yi, const double* dxinv, double* rhs, int neg, cudaStream_t s);
// the same with the y term given: hy from the column slabs of a grid
// decomposed along y (launch_slab_upwind_y's layout, n0 columns per slab)
void launch_upwind_div2d_hy(const DevParams& P, const double* U, const void* const* xi, const double* dxinv,
                            const void* hy, int n0, double* rhs, int neg, cudaStream_t s);
// the y term of the hyperbolic divergence on a column slab (P: its N0
// columns, all N1 rows; UT and yi in the transposed layout; dyinv the whole
// grid's ghosted 1/dy), laid out for the row slabs of n1 rows
void launch_slab_upwind_y(const DevParams& P, const double* UT, const void* const* yi, const double* dyinv, void* hy,
                          int n1, cudaStream_t s);
// rhs += par (if do_visc) then rhs += source (if do_chem)
// sponge zone source on the RHS (box [is, ie) per dimension, sigma per index
// along dim, uref per variable; sigma and uref in device memory)
void launch_sponge(const DevParams& P, const double* U, double* rhs, int dim, const int* is, const int* ie,
                   const double* sigma, const double* uref, cudaStream_t s);
// hnu (optional): photon density planes [nz][ps] of this evaluation
void launch_visc_source(const DevParams& P, const double* U, const double* dxinv, const double* imap,
                        const double* tdev, double cstage, double* rhs, int do_visc, int do_chem, cudaStream_t s,
                        double* hnu = nullptr);
void launch_upwind_iface(const DevParams& P, const double* U, const double* uL, const double* uR, const double* fL,
                         const double* fR, double* fI, int dir, cudaStream_t s);
void launch_first_deriv(const DevParams& P, double* Df, const double* f, int dir, int bias, int nv, cudaStream_t s);
void launch_advance_time(double* tdev, double dt, cudaStream_t s);
void launch_reciprocal(const double* x, double* y, long long n, cudaStream_t s);
void launch_tridiag(double* a, double* b, double* c, double* x, int n, int ns, int* err, cudaStream_t s);

}  // namespace piafs
