// C ABI of the PIAFS GPU path (include/piafs_gpu.h): simulation object,
// time stepping with CUDA-graph replay, Solve() loop with reference-format
// output, and the operator-level entry points.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/piafs_gpu.h"
#include "deck.h"
#include "kernels.h"
#include "sim.h"

using namespace piafs;

namespace {
thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace

namespace piafs {
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return fail(e_ == cudaErrorMemoryAllocation ? PIAFS_ERR_MEMORY : PIAFS_ERR_CUDA,             \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                             \
  } while (0)


static void free_sim(piafs_gpu_sim* s) {
  if (!s) return;
  for (auto& g : s->graph) if (g) cudaGraphExecDestroy(g);
  cudaFree(s->u);
  for (int k = 1; k < MAX_STAGES; k++) cudaFree(s->U[k]);
  for (auto p : s->Ud) cudaFree(p);
  cudaFree(s->fC);
  for (auto p : s->iface) cudaFree(p);
  for (auto p : s->iface_y) cudaFree(p);
  cudaFree(s->scratch);
  cudaFree(s->ut);
  cudaFree(s->dxinv);
  cudaFree(s->imap);
  cudaFree(s->tdev);
  cudaFree(s->top_t);
  cudaFree(s->norm_acc);
  cudaFree(s->cfl_acc);
  cudaFree(s->err);
  cudaFree(s->aos);
  cudaFree(s->hnu);
  cudaFree(s->sponge_buf);
  cudaFree(s->zone_buf);
  cudaFree(s->crwchar);
  cudaFree(s->fCy);
  if (s->yfork) cudaEventDestroy(s->yfork);
  if (s->yjoin) cudaEventDestroy(s->yjoin);
  if (s->ystream) cudaStreamDestroy(s->ystream);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

// -------------------------------------------------------------- the RHS
// Cell-centred flux and interface values (uL, uR, fL, fR into I) of
// direction d.  The y pass of a 2D CRWENO5 run works on a transposed copy of
// U so that its lines, the tridiagonal systems, are contiguous in memory; its
// interface arrays are then in the transposed layout.  If `ev` is given, an
// event is recorded after the flux and after the reconstruction.
void piafs::enqueue_recon(piafs_gpu_sim* s, const double* U, int d, double* const* I, cudaEvent_t* ev, int* k) {
  const DevParams& P = s->P;
  auto mark = [&]() { if (ev) cudaEventRecord(ev[++*k], s->stream); };
  if (P.scheme == CRWENO5 && P.char_interp) {
    launch_flux(P, U, s->fC, d, s->stream);
    mark();
    launch_crweno_char(P, U, s->fC, I[0], I[1], I[2], I[3], d, s->crwchar, s->err, s->stream);
    mark();
    return;
  }
  if (d == 1 && s->ut) {
    if (P.model == NS2D) {
      launch_transpose_flux_y(P, U, s->ut, s->fC, s->stream);
    } else {
      launch_transpose(P, U, s->ut, s->stream);
      launch_flux(P, s->ut, s->fC, 1, s->stream);
    }
    mark();
    launch_crweno(s->PT, s->ut, s->fC, I[0], I[1], I[2], I[3], 0, s->err, s->stream);
    mark();
    return;
  }
  launch_flux(P, U, s->fC, d, s->stream);
  mark();
  if (P.scheme != CRWENO5 && P.char_interp) launch_weno5_char(P, U, s->fC, I[0], I[1], I[2], I[3], d, s->stream);
  else if (P.scheme != CRWENO5) launch_weno5(P, U, s->fC, I[0], I[1], I[2], I[3], d, s->stream);
  else launch_crweno(P, U, s->fC, I[0], I[1], I[2], I[3], d, s->err, s->stream);
  mark();
}

// HyperbolicFunction (HyperbolicFunction.c:35-119) over all directions into
// out: -hyp (neg, the stage derivative's first term) or hyp.  In 2D both
// directions' interfaces are reconstructed first and one kernel upwinds them
// and forms the divergence.
static void enqueue_hyp(piafs_gpu_sim* s, const double* U, double* out, bool neg, cudaEvent_t* ev = nullptr,
                        int* k = nullptr) {
  const DevParams& P = s->P;
  if (s->concurrent_y && !ev && P.ndims == 2) cudaEventRecord(s->yfork, s->stream);
  enqueue_recon(s, U, 0, s->iface, ev, k);
  if (P.ndims == 1) {
    launch_upwind_div(P, U, s->iface[0], s->iface[1], s->iface[2], s->iface[3], s->dxinv, out, 0, neg ? 0 : 2,
                      s->stream);
  } else {
    if (s->concurrent_y && !ev) {
      // the y pass joins the x pass's stream before the upwind kernel
      cudaStreamWaitEvent(s->ystream, s->yfork, 0);
      double* const* Iy = s->iface_y;
      launch_transpose_flux_y(P, U, s->ut, s->fCy, s->ystream);
      launch_crweno(s->PT, s->ut, s->fCy, Iy[0], Iy[1], Iy[2], Iy[3], 0, s->err, s->ystream);
      cudaEventRecord(s->yjoin, s->ystream);
      cudaStreamWaitEvent(s->stream, s->yjoin, 0);
    } else {
      enqueue_recon(s, U, 1, s->iface_y, ev, k);
    }
    const void* xi[4] = {s->iface[0], s->iface[1], s->iface[2], s->iface[3]};
    const void* yi[4] = {s->iface_y[0], s->iface_y[1], s->iface_y[2], s->iface_y[3]};
    launch_upwind_div2d(P, U, s->ut, xi, yi, s->dxinv, out, neg ? 1 : 0, s->stream);
  }
  if (ev) cudaEventRecord(ev[++*k], s->stream);
}

// TimeRHSFunctionExplicit (TimeRHSFunctionExplicit.c:29-77) on SoA arrays:
// rhs = -hyp + par + source; U must have its ghosts filled.
// hnu: where the source stores the photon density of this evaluation (the
// reference's Chemistry::nv_hnu), or nullptr
// the sponge zones' source (SourceFunction.c:42-57) added to rhs
static void enqueue_sponge(piafs_gpu_sim* s, const double* U, double* rhs) {
  for (const auto& z : s->sponges)
    launch_sponge(s->P, U, rhs, z.dim, z.is, z.ie, s->sponge_buf + z.sig_off, s->sponge_buf + z.ref_off, s->stream);
}

static void enqueue_rhs(piafs_gpu_sim* s, double* rhs, const double* U, const double* tdev, double cstage,
                        double* hnu = nullptr) {
  enqueue_hyp(s, U, rhs, true);
  launch_visc_source(s->P, U, s->dxinv, s->imap, tdev, cstage, rhs, 1, 1, s->stream, hnu);
  enqueue_sponge(s, U, rhs);
}

void piafs::enqueue_bc(piafs_gpu_sim* s, double* u) {
  for (const Zone& z : s->deck.zones) launch_bc(s->P, u, z, s->stream);
}

// One time step: TimePreStep's boundary conditions on u, TimeRK's stages and
// step completion, t += dt.  U[0] aliases u: the reference copies u into
// U[0] and re-applies the (idempotent) boundary conditions to it.
static void enqueue_step(piafs_gpu_sim* s, bool with_norm) {
  const DevParams& P = s->P;
  const Deck& d = s->deck;
  const int ns = d.nstages;
  const long long n = (long long)P.nvars * P.ps;
  enqueue_bc(s, s->u);
  for (int st = 0; st < ns; st++) {
    double* Us = st == 0 ? s->u : s->U[st];
    if (st > 0) {
      const double* dd[MAX_STAGES];
      double a[MAX_STAGES];
      for (int j = 0; j < st; j++) { dd[j] = s->Ud[j]; a[j] = d.dt * d.A[st * MAX_STAGES + j]; }
      launch_stage(n, Us, s->u, dd, a, st, s->stream);
      enqueue_bc(s, Us);
    }
    enqueue_rhs(s, s->Ud[st], Us, s->tdev, d.c[st], st == ns - 1 ? s->hnu : nullptr);
  }
  const double* dd[MAX_STAGES];
  double b[MAX_STAGES];
  for (int j = 0; j < ns; j++) { dd[j] = s->Ud[j]; b[j] = d.dt * d.b[j]; }
  if (with_norm) cudaMemsetAsync(s->norm_acc, 0, sizeof(double), s->stream);
  launch_update(P, s->u, dd, b, ns, with_norm ? s->norm_acc : nullptr, s->stream);
  launch_advance_time(s->tdev, d.dt, s->stream);
}

static int run_steps(piafs_gpu_sim* s, int nsteps, bool norm_last) {
  for (int k = 0; k < nsteps; k++) {
    const bool with_norm = norm_last && (k == nsteps - 1);
    const int gi = with_norm ? 1 : 0;
    if (s->use_graph) {
      if (!s->graph[gi]) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(s, with_norm);
        CK(cudaStreamEndCapture(s->stream, &g));
        CK(cudaGraphInstantiate(&s->graph[gi], g, 0));
        cudaGraphDestroy(g);
      }
      CK(cudaGraphLaunch(s->graph[gi], s->stream));
    } else {
      enqueue_step(s, with_norm);
    }
    s->t += s->deck.dt;   // same accumulation as the device clock (TimePostStep.c:31)
    s->iter++;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->stream));
  int e = 0;
  CK(cudaMemcpy(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    s->singular++;
    cudaMemset(s->err, 0, sizeof(int));
  }
  if (norm_last) {
    double sum = 0.0;
    CK(cudaMemcpy(&sum, s->norm_acc, sizeof(double), cudaMemcpyDeviceToHost));
    double npts = (double)s->P.N0 * (double)s->P.N1;
    s->last_norm = std::sqrt(sum / npts);
  }
  return PIAFS_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* piafs_gpu_last_error(void) { return g_err.c_str(); }

int piafs_gpu_create(const char* deck_dir, int precision, piafs_gpu_sim** out) {
  if (!deck_dir || !out) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  Deck d;
  std::string err;
  if (int r = read_deck(deck_dir, d, err)) return fail(r, err);
  return piafs::create_sim(std::move(d), precision, out);
}

}  // extern "C"

// A simulation from a parsed (or otherwise filled) deck: device arrays,
// initial state, simulation time restart_iter x dt.
int piafs::create_sim(Deck&& deck, int precision, piafs_gpu_sim** out) {
  if (!out) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  if (precision != PIAFS_PRECISION_FP64 && precision != PIAFS_PRECISION_MIXED)
    return fail(PIAFS_ERR_ARGUMENT, "precision must be PIAFS_PRECISION_FP64 or PIAFS_PRECISION_MIXED");
  auto* s = new piafs_gpu_sim();
  s->deck = std::move(deck);
  std::string err;
  int r = make_params(s->deck, s->P, err);
  if (r) { delete s; return fail(r, err); }
  s->precision = precision;
  s->P.mixed = precision == PIAFS_PRECISION_MIXED ? 1 : 0;
  {
    // PIAFS_GPU_NO_PACKED_SPECIES=1 keeps the passive variables' four
    // interface arrays (the same values; for checking the packed form)
    const DevParams& Q = s->P;
    const char* npk = std::getenv("PIAFS_GPU_NO_PACKED_SPECIES");
    s->P.pack_sp = (Q.model == NS2D && Q.ndims == 2 && Q.nvars > Q.nflow && Q.scheme == CRWENO5 &&
                    !Q.char_interp && Q.upwind != UPW_RF && crweno_line_fits(Q.N0) && crweno_line_fits(Q.N1) &&
                    !(npk && npk[0] == '1'))
                       ? 1 : 0;
  }
  if (s->P.mixed && s->P.char_interp) {
    delete s;
    return fail(PIAFS_ERR_UNSUPPORTED, "mixed precision runs hyp_interp_type components");
  }
  const char* ng = std::getenv("PIAFS_GPU_NO_GRAPH");
  s->use_graph = !(ng && ng[0] == '1');
  const DevParams& P = s->P;
  const Deck& d = s->deck;
  auto alloc = [&](double** p, size_t n) -> cudaError_t {
    cudaError_t e = cudaMalloc(p, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(*p, 0, n * sizeof(double));
    return e;
  };
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  const size_t planes = (size_t)P.nvars * P.ps, iplanes = (size_t)P.nvars * P.pis;
  if (e == cudaSuccess) e = alloc(&s->u, planes);
  for (int k = 1; k < d.nstages && e == cudaSuccess; k++) e = alloc(&s->U[k], planes);
  for (int k = 0; k < d.nstages && e == cudaSuccess; k++) e = alloc(&s->Ud[k], planes);
  if (e == cudaSuccess) e = alloc(&s->fC, planes);
  for (int k = 0; k < 5 && e == cudaSuccess; k++) e = alloc(&s->iface[k], iplanes);
  for (int k = 0; k < 4 && e == cudaSuccess && P.ndims == 2; k++) e = alloc(&s->iface_y[k], iplanes);
  if (e == cudaSuccess) e = alloc(&s->scratch, planes);
  // transposed y pass: 2D CRWENO5 (PIAFS_GPU_NO_YTRANSPOSE=1 keeps the
  // column-strided kernels instead in the FP64 path; the mixed path has only
  // the transposed one)
  const char* noyt = std::getenv("PIAFS_GPU_NO_YTRANSPOSE");
  if (e == cudaSuccess && P.scheme == CRWENO5 && P.char_interp) e = alloc(&s->crwchar, crweno_char_scratch(P));
  if (e == cudaSuccess && P.ndims == 2 && P.scheme == CRWENO5 && !P.char_interp &&
      (P.mixed || !(noyt && noyt[0] == '1'))) {
    e = alloc(&s->ut, planes);
    s->PT = transposed_params(P);
    // PIAFS_GPU_NO_CONCURRENT_Y=1 runs the y pass after the x pass on one
    // stream (the same values)
    const char* ncy = std::getenv("PIAFS_GPU_NO_CONCURRENT_Y");
    if (e == cudaSuccess && P.model == NS2D && !(ncy && ncy[0] == '1')) {
      e = alloc(&s->fCy, planes);
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->ystream, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->yfork, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->yjoin, cudaEventDisableTiming);
      s->concurrent_y = e == cudaSuccess;
    }
  }
  if (e == cudaSuccess) e = alloc(&s->dxinv, d.dxinv.size());
  if (e == cudaSuccess) e = alloc(&s->imap, d.imap.size());
  if (e == cudaSuccess) e = alloc(&s->tdev, 1);
  if (e == cudaSuccess) e = alloc(&s->top_t, 1);
  if (e == cudaSuccess) e = alloc(&s->norm_acc, 1);
  if (e == cudaSuccess) e = cudaMalloc(&s->cfl_acc, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&s->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(s->err, 0, sizeof(int));
  s->aos_bytes = (size_t)P.npg * P.nvars * sizeof(double);
  if (e == cudaSuccess) e = cudaMalloc(&s->aos, s->aos_bytes);
  // the species files carry the photon density of the last RK stage evaluated
  // (zero before the first step, as the reference's calloc'd nv_hnu)
  const bool binary_out = d.op_file_format == "binary" || d.op_file_format == "bin";
  if (e == cudaSuccess && d.write_species && binary_out) e = alloc(&s->hnu, (size_t)P.nz * P.ps);
  if (e == cudaSuccess && !d.sponges.empty()) {
    std::vector<double> hb;
    for (const auto& z : d.sponges) {
      piafs_gpu_sim::SpongeDev sd{};
      sd.dim = z.dim;
      for (int k = 0; k < 2; k++) { sd.is[k] = z.is[k]; sd.ie[k] = z.ie[k]; }
      sd.ref_off = hb.size();
      hb.insert(hb.end(), z.uref.begin(), z.uref.end());
      sd.sig_off = hb.size();
      hb.insert(hb.end(), z.sigma.begin(), z.sigma.end());
      s->sponges.push_back(sd);
    }
    e = alloc(&s->sponge_buf, hb.size());
    if (e == cudaSuccess) e = cudaMemcpy(s->sponge_buf, hb.data(), hb.size() * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) {
    std::vector<size_t> off;
    const std::vector<double> hv = pack_zone_values(d, off);
    if (!hv.empty()) {
      e = alloc(&s->zone_buf, hv.size());
      if (e == cudaSuccess) e = cudaMemcpy(s->zone_buf, hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) bind_zone_values(d, off, s->zone_buf, s->deck.zones.data());
    }
  }
  if (e == cudaSuccess) e = cudaMemcpy(s->dxinv, d.dxinv.data(), d.dxinv.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->imap, d.imap.data(), d.imap.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    int code = e == cudaErrorMemoryAllocation ? PIAFS_ERR_MEMORY : PIAFS_ERR_CUDA;
    std::string msg = std::string("device set-up failed: ") + cudaGetErrorString(e);
    free_sim(s);
    return fail(code, msg);
  }
  s->U[0] = s->u;
  // initial solution; restart time waqt = restart_iter * dt (TimeInitialize.c:51)
  int rr = piafs_gpu_set_state(s, d.u0.data(), d.restart_iter * d.dt);
  if (rr) { free_sim(s); return rr; }
  s->iter = d.restart_iter;
  *out = s;
  return PIAFS_OK;
}

extern "C" {

void piafs_gpu_destroy(piafs_gpu_sim* s) { free_sim(s); }

int piafs_gpu_get_photon_density(piafs_gpu_sim* s, double* nv_hnu) {
  if (!s || !nv_hnu) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  if (!s->hnu) return fail(PIAFS_ERR_ARGUMENT, "this simulation keeps no photon density (no species output)");
  const DevParams& P = s->P;
  std::vector<double> h((size_t)P.nz * P.ps);
  CK(cudaMemcpyAsync(h.data(), s->hnu, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  for (long long p = 0; p < P.npg; p++)
    for (int iz = 0; iz < P.nz; iz++) nv_hnu[(size_t)P.nz * p + iz] = h[(size_t)iz * P.ps + p];
  return PIAFS_OK;
}

int piafs_gpu_get_info(piafs_gpu_sim* s, piafs_gpu_info* info) {
  if (!s || !info) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  const Deck& d = s->deck;
  std::memset(info, 0, sizeof(*info));
  info->ndims = d.ndims; info->nvars = d.nvars; info->ghosts = d.ghosts;
  info->dim[0] = s->P.N0; info->dim[1] = s->P.N1;
  info->n_iter = d.n_iter; info->restart_iter = d.restart_iter;
  info->screen_op_iter = d.screen_op_iter; info->file_op_iter = d.file_op_iter;
  info->iter = s->iter; info->nstages = d.nstages;
  info->dt = d.dt; info->t = s->t;
  info->gamma = d.gamma; info->Re = d.Re; info->Pr = d.Pr;
  info->npoints_ghosted = s->P.npg;
  info->ninterfaces[0] = s->P.nint[0]; info->ninterfaces[1] = s->P.nint[1];
  info->cfl = s->last_cfl; info->norm = s->last_norm; info->singular = s->singular;
  // kernels per step: prestep BCs, per stage (combine + BCs for s > 0, flux
  // and reconstruction per direction plus the transpose of a transposed y
  // pass, one upwind/divergence kernel, viscous/source), update, clock
  const int nz = (int)d.zones.size();
  const int vs = ((s->P.ndims == 2 && s->P.viscous) || s->P.chem) ? 1 : 0;
  const int tr = (s->ut && s->P.model != NS2D) ? 1 : 0;   // NS2D: the transpose also forms the y flux
  info->launches_per_step = nz + d.nstages * (2 * s->P.ndims + 1 + tr + vs) + (d.nstages - 1) * (1 + nz) + 2;
  return PIAFS_OK;
}

int piafs_gpu_set_state(piafs_gpu_sim* s, const double* u_host, double t) {
  if (!s || !u_host) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  CK(cudaMemcpyAsync(s->aos, u_host, s->aos_bytes, cudaMemcpyHostToDevice, s->stream));
  launch_aos_to_soa(s->aos, s->u, s->P.npg, s->P.nvars, s->P.ps, s->stream);
  CK(cudaMemcpyAsync(s->tdev, &t, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->t = t;
  return PIAFS_OK;
}

int piafs_gpu_get_state(piafs_gpu_sim* s, double* u_host) {
  if (!s || !u_host) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  launch_soa_to_aos(s->u, s->aos, s->P.npg, s->P.nvars, s->P.ps, s->stream);
  CK(cudaMemcpyAsync(u_host, s->aos, s->aos_bytes, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return PIAFS_OK;
}

int piafs_gpu_get_solution(piafs_gpu_sim* s, double* out) {
  if (!s || !out) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  launch_soa_to_interior(s->P, s->u, s->aos, s->stream);
  CK(cudaMemcpyAsync(out, s->aos, (size_t)s->P.N0 * s->P.N1 * s->P.nvars * sizeof(double), cudaMemcpyDeviceToHost,
                     s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return PIAFS_OK;
}

int piafs_gpu_TimeRK(piafs_gpu_sim* s, int nsteps) {
  if (!s || nsteps < 0) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  return run_steps(s, nsteps, false);
}

int piafs_gpu_TimeRK_async(piafs_gpu_sim* s, int nsteps) {
  if (!s || nsteps < 0) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  for (int k = 0; k < nsteps; k++) {
    if (s->use_graph) {
      if (!s->graph[0]) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(s, false);
        CK(cudaStreamEndCapture(s->stream, &g));
        CK(cudaGraphInstantiate(&s->graph[0], g, 0));
        cudaGraphDestroy(g);
      }
      CK(cudaGraphLaunch(s->graph[0], s->stream));
    } else {
      enqueue_step(s, false);
    }
    s->t += s->deck.dt;
    s->iter++;
  }
  CK(cudaGetLastError());
  return PIAFS_OK;
}

int piafs_gpu_get_stream(piafs_gpu_sim* s, void** stream) {
  if (!s || !stream) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  *stream = (void*)s->stream;
  return PIAFS_OK;
}

int piafs_gpu_synchronize(piafs_gpu_sim* s) {
  if (!s) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  CK(cudaStreamSynchronize(s->stream));
  int e = 0;
  CK(cudaMemcpy(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) { s->singular++; cudaMemset(s->err, 0, sizeof(int)); }
  return PIAFS_OK;
}

int piafs_gpu_profile_rhs(piafs_gpu_sim* s, int reps, double* ms, int* nphases) {
  if (!s || !ms || !nphases || reps < 1) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  const DevParams& P = s->P;
  const int np = P.ndims == 1 ? 4 : 6;
  if (*nphases < np) return fail(PIAFS_ERR_ARGUMENT, "ms[] too small");
  *nphases = np;
  std::vector<cudaEvent_t> ev(np + 1);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  std::vector<double> acc(np, 0.0);
  double* U = s->u;
  double* R = s->Ud[0];
  // one untimed evaluation first: the first launches of a kernel outside the
  // step graphs carry one-time set-up
  for (int r = -1; r < reps; r++) {
    enqueue_bc(s, U);
    int k = 0;
    CK(cudaEventRecord(ev[0], s->stream));
    enqueue_hyp(s, U, R, true, ev.data(), &k);
    launch_visc_source(P, U, s->dxinv, s->imap, s->tdev, 0.0, R, 1, 1, s->stream);
    enqueue_sponge(s, U, R);
    CK(cudaEventRecord(ev[++k], s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (r < 0) continue;
    for (int i = 0; i < np; i++) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
      acc[i] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int i = 0; i < np; i++) ms[i] = acc[i] / reps;
  CK(cudaGetLastError());
  return PIAFS_OK;
}

int piafs_gpu_TimeRK_host(piafs_gpu_sim* s, double* u_host, double t) {
  if (int r = piafs_gpu_set_state(s, u_host, t)) return r;
  if (int r = run_steps(s, 1, false)) return r;
  return piafs_gpu_get_state(s, u_host);
}

int piafs_gpu_ComputeCFL(piafs_gpu_sim* s, double* cfl) {
  if (!s || !cfl) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  CK(cudaMemsetAsync(s->cfl_acc, 0, sizeof(unsigned long long), s->stream));
  launch_cfl(s->P, s->u, s->dxinv, s->cfl_acc, s->stream);
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, s->cfl_acc, sizeof(bits), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(cfl, &bits, sizeof(double));
  s->last_cfl = *cfl;
  return PIAFS_OK;
}

int piafs_gpu_Solve(piafs_gpu_sim* s, const char* output_dir) {
  if (!s || !output_dir) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  const Deck& d = s->deck;
  const bool write = d.op_file_format == "binary" || d.op_file_format == "bin";
  if (!write && d.op_file_format != "none")
    return fail(PIAFS_ERR_UNSUPPORTED, "op_file_format " + d.op_file_format + " is not supported (binary, none)");
  const bool overwrite = d.op_overwrite != "no";
  int index = 0;
  // a restart fast-forwards the output index (InitializeSolvers.c:240-245)
  if (!overwrite)
    for (int t = 0; t < d.restart_iter; t++)
      if ((t + 1) % d.file_op_iter == 0) index++;
  std::vector<double> host((size_t)s->P.N0 * s->P.N1 * d.nvars);
  std::vector<double> hnu_host;
  // ChemistryWriteSpecies (ChemistryWriteSpecies.c:19-90): per layer iz, the
  // seven species of the LAST layer (the reference copies layer z_i for every
  // iz) and the photon density of layer iz, as op_species_z<iz>[_NNNNN].bin,
  // written before the solution file of the same index (Solve.cpp:56-65)
  auto species = [&]() -> int {
    if (!d.write_species || !s->hnu) return PIAFS_OK;
    const DevParams& P = s->P;
    const int nz = P.nz, nsp = 8, z_i = nz - 1;
    hnu_host.resize((size_t)nz * P.ps);
    CK(cudaMemcpyAsync(hnu_host.data(), s->hnu, hnu_host.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const long long npts = (long long)P.N0 * P.N1;
    std::vector<double> sp((size_t)npts * nsp);
    int width = 1;
    for (int q = nz; q >= 10; q /= 10) width++;          // (int)log10(nz) + 1
    for (int iz = d.write_all_zlocs == "no" ? z_i : 0; iz < nz; iz++) {
      for (long long k = 0; k < npts; k++) {
        const int i = (int)(k % P.N0), j = (int)(k / P.N0);
        for (int m = 0; m < nsp - 1; m++) sp[k * nsp + m] = host[k * d.nvars + P.nflow + P.zstride * z_i + m];
        sp[k * nsp + nsp - 1] = hnu_host[(size_t)iz * P.ps + pidx(P, i, j)];
      }
      char name[96];
      if (overwrite) std::snprintf(name, sizeof(name), "op_species_z%0*d.bin", width, iz);
      else std::snprintf(name, sizeof(name), "op_species_z%0*d_%05d.bin", width, iz, index);
      std::string err;
      if (int r = write_binary(std::string(output_dir) + "/" + name, d, sp.data(), err, nsp)) return fail(r, err);
    }
    return PIAFS_OK;
  };
  auto output = [&]() -> int {
    if (!write) return PIAFS_OK;
    if (int r = piafs_gpu_get_solution(s, host.data())) return r;
    if (int r = species()) return r;
    char name[64];
    if (overwrite) std::snprintf(name, sizeof(name), "op.bin");
    else std::snprintf(name, sizeof(name), "op_%05d.bin", index);
    std::string err;
    if (int r = write_binary(std::string(output_dir) + "/" + name, d, host.data(), err)) return fail(r, err);
    if (!overwrite) index++;
    return PIAFS_OK;
  };
  // Solve.cpp:54-95; on screen steps the CFL before the step
  // (TimePreStep.c:54-65), the residual norm after it (TimePostStep.c:36-54)
  // and the TimePrintStep line (TimePrintStep.c:25-37)
  for (int it = s->iter; it < d.n_iter; it++) {
    if (it == 0) if (int r = output()) return r;
    const auto w0 = std::chrono::steady_clock::now();
    const bool screen = ((it + 1) % d.screen_op_iter) == 0;
    if (screen) {
      double c;
      if (int r = piafs_gpu_ComputeCFL(s, &c)) return r;
    }
    if (int r = run_steps(s, 1, screen)) return r;
    if (screen) {
      const double wct = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
      std::printf("iter=%7d  t=%1.3E  CFL=%1.3E  norm=%1.4E  wctime: %1.1E (s)  \n", it + 1, s->t, s->last_cfl,
                  s->last_norm, wct);
      std::fflush(stdout);
    }
    if (((it + 1) % d.file_op_iter == 0) && (it + 1 < d.n_iter))
      if (int r = output()) return r;
  }
  return output();
}

int piafs_gpu_TimeRK_norm(piafs_gpu_sim* s, int nsteps, double* norm) {
  if (!s || nsteps < 1 || !norm) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  if (int r = run_steps(s, nsteps, true)) return r;
  *norm = s->last_norm;
  return PIAFS_OK;
}

// SimWriteErrors (SimulationWriteErrors.c:65-80) for one simulation, after
// CalculateError (CalculateError.c:30-120) against exact.inp when the deck
// directory holds one
int piafs_gpu_WriteErrors(piafs_gpu_sim* s, const char* dir, double solver_runtime, double main_runtime) {
  if (!s || !dir) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  const Deck& d = s->deck;
  const DevParams& P = s->P;
  const long long npts = (long long)P.N0 * P.N1;
  std::vector<double> u((size_t)npts * d.nvars);
  if (int r = piafs_gpu_get_solution(s, u.data())) return r;
  double err3[3] = {-1.0, -1.0, -1.0};
  std::vector<double> ex;
  bool found = false;
  std::string msg;
  if (int r = read_exact(dir, d, ex, found, msg)) return fail(r, msg);
  if (found) {
    double nrm[3] = {0, 0, 0}, e[3] = {0, 0, 0};
    for (size_t k = 0; k < u.size(); k++) {
      const double x = ex[k], dd = u[k] - ex[k];
      nrm[0] += std::fabs(x); nrm[1] += x * x; nrm[2] = std::max(nrm[2], std::fabs(x));
      e[0] += std::fabs(dd); e[1] += dd * dd; e[2] = std::max(e[2], std::fabs(dd));
    }
    nrm[0] /= (double)npts; nrm[1] = std::sqrt(nrm[1] / (double)npts);
    e[0] /= (double)npts; e[1] = std::sqrt(e[1] / (double)npts);
    const double tol = 1e-15;
    const bool rel = nrm[0] > tol && nrm[1] > tol && nrm[2] > tol;
    for (int k = 0; k < 3; k++) err3[k] = rel ? e[k] / nrm[k] : e[k];
  }
  const std::string base(dir);
  FILE* f = std::fopen((base + "/errors.dat").c_str(), "w");
  if (!f) return fail(PIAFS_ERR_IO, "cannot write errors.dat");
  for (int k = 0; k < d.ndims; k++) std::fprintf(f, "%4d ", d.size[k]);
  for (int k = 0; k < d.ndims; k++) std::fprintf(f, "%4d ", 1);
  std::fprintf(f, "%1.16E  ", d.dt);
  std::fprintf(f, "%1.16E %1.16E %1.16E   ", err3[0], err3[1], err3[2]);
  std::fprintf(f, "%1.16E %1.16E\n", solver_runtime, main_runtime);
  std::fclose(f);
  // conservation errors: -1 per variable, as the reference leaves them
  // without conservation_check (Initialize.c:195-196)
  f = std::fopen((base + "/conservation.dat").c_str(), "w");
  if (!f) return fail(PIAFS_ERR_IO, "cannot write conservation.dat");
  for (int k = 0; k < d.ndims; k++) std::fprintf(f, "%4d ", d.size[k]);
  for (int k = 0; k < d.ndims; k++) std::fprintf(f, "%4d ", 1);
  std::fprintf(f, "%1.16E  ", d.dt);
  for (int v = 0; v < d.nvars; v++) std::fprintf(f, "%1.16E ", -1.0);
  std::fprintf(f, "\n");
  std::fclose(f);
  // calls of the hyperbolic, parabolic and source functions: one each per
  // RK stage, the parabolic one only for viscous Navier-Stokes
  // (NavierStokes2DParabolicFunction.c:64-65), the source one when the model
  // has a source (both models do, SourceFunction.c:37-39)
  const long long steps = (long long)s->iter - d.restart_iter;
  f = std::fopen((base + "/function_counts.dat").c_str(), "w");
  if (!f) return fail(PIAFS_ERR_IO, "cannot write function_counts.dat");
  std::fprintf(f, "%d\n", d.n_iter);
  std::fprintf(f, "%lld\n", steps * d.nstages);
  std::fprintf(f, "%lld\n", (P.ndims == 2 && P.viscous) ? steps * d.nstages : 0);
  std::fprintf(f, "%lld\n", steps * d.nstages);
  std::fclose(f);
  if (err3[0] >= 0) {
    std::printf("Computed errors for domain %d:\n", 0);
    std::printf("  L1         Error           : %1.16E\n", err3[0]);
    std::printf("  L2         Error           : %1.16E\n", err3[1]);
    std::printf("  Linfinity  Error           : %1.16E\n", err3[2]);
  }
  std::printf("Solver runtime (in seconds): %1.16E\n", solver_runtime);
  std::printf("Total  runtime (in seconds): %1.16E\n", main_runtime);
  return PIAFS_OK;
}

// ------------------------------------------------- operator-level calls
static int to_soa(piafs_gpu_sim* s, const double* aos, double* soa) {
  launch_aos_to_soa(aos, soa, s->P.npg, s->P.nvars, s->P.ps, s->stream);
  return PIAFS_OK;
}
static int set_top_t(piafs_gpu_sim* s, double t) {
  CK(cudaMemcpyAsync(s->top_t, &t, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  return PIAFS_OK;
}
static int finish(piafs_gpu_sim* s) {
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->stream));
  return PIAFS_OK;
}

int piafs_gpu_RHSFunction(piafs_gpu_sim* s, double* rhs, double* u, double t) {
  if (!s || !rhs || !u) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  const size_t planes = (size_t)s->P.nvars * s->P.ps * sizeof(double);
  double* U = s->scratch;
  double* R = s->Ud[0];
  to_soa(s, u, U);
  enqueue_bc(s, U);
  CK(cudaMemsetAsync(R, 0, planes, s->stream));
  if (int r = set_top_t(s, t)) return r;
  enqueue_rhs(s, R, U, s->top_t, 0.0);
  launch_soa_to_aos(U, u, s->P.npg, s->P.nvars, s->P.ps, s->stream);
  launch_soa_to_aos(R, rhs, s->P.npg, s->P.nvars, s->P.ps, s->stream);
  return finish(s);
}

int piafs_gpu_HyperbolicFunction(piafs_gpu_sim* s, double* hyp, const double* u, double t) {
  if (!s || !hyp || !u) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  const DevParams& P = s->P;
  double* U = s->scratch;
  double* H = s->Ud[0];
  to_soa(s, u, U);
  CK(cudaMemsetAsync(H, 0, (size_t)P.nvars * P.ps * sizeof(double), s->stream));
  enqueue_hyp(s, U, H, false);
  launch_soa_to_aos(H, hyp, P.npg, P.nvars, P.ps, s->stream);
  return finish(s);
}

static int visc_or_source(piafs_gpu_sim* s, double* out, const double* u, double t, int visc, int chem) {
  if (!s || !out || !u) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  const DevParams& P = s->P;
  double* U = s->scratch;
  double* R = s->Ud[0];
  to_soa(s, u, U);
  CK(cudaMemsetAsync(R, 0, (size_t)P.nvars * P.ps * sizeof(double), s->stream));
  if (int r = set_top_t(s, t)) return r;
  launch_visc_source(P, U, s->dxinv, s->imap, s->top_t, 0.0, R, visc, chem, s->stream);
  if (chem) enqueue_sponge(s, U, R);   // the sponge is part of SourceFunction
  launch_soa_to_aos(R, out, P.npg, P.nvars, P.ps, s->stream);
  return finish(s);
}
int piafs_gpu_ParabolicFunction(piafs_gpu_sim* s, double* par, const double* u, double t) {
  return visc_or_source(s, par, u, t, 1, 0);
}
int piafs_gpu_SourceFunction(piafs_gpu_sim* s, double* src, const double* u, double t) {
  return visc_or_source(s, src, u, t, 0, 1);
}

int piafs_gpu_ApplyBoundaryConditions(piafs_gpu_sim* s, double* u, double) {
  if (!s || !u) return fail(PIAFS_ERR_ARGUMENT, "null argument");
  to_soa(s, u, s->scratch);
  enqueue_bc(s, s->scratch);
  launch_soa_to_aos(s->scratch, u, s->P.npg, s->P.nvars, s->P.ps, s->stream);
  return finish(s);
}

int piafs_gpu_FFunction(piafs_gpu_sim* s, double* f, const double* u, int dir, double) {
  if (!s || !f || !u || dir < 0 || dir >= s->P.ndims) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  to_soa(s, u, s->scratch);
  launch_flux(s->P, s->scratch, s->fC, dir, s->stream);
  launch_soa_to_aos(s->fC, f, s->P.npg, s->P.nvars, s->P.ps, s->stream);
  return finish(s);
}

int piafs_gpu_InterpolateInterfacesHyp(piafs_gpu_sim* s, double* fI, const double* fC, const double* u, int upw,
                                       int dir, int uflag) {
  if (!s || !fI || !fC || !u || dir < 0 || dir >= s->P.ndims) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  DevParams P = s->P;
  P.mixed = 0;     // operator-level entry points are FP64
  P.pack_sp = 0;   // and return every interface array as the reference forms it
  to_soa(s, u, s->scratch);
  to_soa(s, fC, s->fC);
  if (P.scheme == CRWENO5 && P.char_interp)
    launch_crweno_char(P, s->scratch, s->fC, s->iface[0], s->iface[1], s->iface[2], s->iface[3], dir, s->crwchar,
                       s->err, s->stream);
  else if (P.scheme != CRWENO5 && P.char_interp)
    launch_weno5_char(P, s->scratch, s->fC, s->iface[0], s->iface[1], s->iface[2], s->iface[3], dir, s->stream);
  else if (P.scheme != CRWENO5)
    launch_weno5(P, s->scratch, s->fC, s->iface[0], s->iface[1], s->iface[2], s->iface[3], dir, s->stream);
  else
    launch_crweno(P, s->scratch, s->fC, s->iface[0], s->iface[1], s->iface[2], s->iface[3], dir, s->err, s->stream);
  const double* src = s->iface[(uflag ? 0 : 2) + (upw > 0 ? 0 : 1)];
  launch_iface_soa_to_aos(src, fI, P.nint[dir], P.nvars, P.pis, s->stream);
  return finish(s);
}

int piafs_gpu_Upwind(piafs_gpu_sim* s, double* fI, const double* fL, const double* fR, const double* uL,
                     const double* uR, const double* u, int dir, double) {
  if (!s || !fI || !fL || !fR || !uL || !uR || !u || dir < 0 || dir >= s->P.ndims)
    return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  const DevParams& P = s->P;
  const long long ni = P.nint[dir];
  to_soa(s, u, s->scratch);
  launch_iface_aos_to_soa(uL, s->iface[0], ni, P.nvars, P.pis, s->stream);
  launch_iface_aos_to_soa(uR, s->iface[1], ni, P.nvars, P.pis, s->stream);
  launch_iface_aos_to_soa(fL, s->iface[2], ni, P.nvars, P.pis, s->stream);
  launch_iface_aos_to_soa(fR, s->iface[3], ni, P.nvars, P.pis, s->stream);
  launch_upwind_iface(P, s->scratch, s->iface[0], s->iface[1], s->iface[2], s->iface[3], s->iface[4], dir, s->stream);
  launch_iface_soa_to_aos(s->iface[4], fI, ni, P.nvars, P.pis, s->stream);
  return finish(s);
}

int piafs_gpu_FirstDerivativePar(piafs_gpu_sim* s, double* Df, const double* f, int dir, int bias, int nv) {
  if (!s || !Df || !f || dir < 0 || dir >= s->P.ndims || nv < 1) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  launch_first_deriv(s->P, Df, f, dir, bias, nv, s->stream);
  return finish(s);
}

int piafs_gpu_tridiagLU(double* a, double* b, double* c, double* x, int n, int ns) {
  if (!a || !b || !c || !x || n < 0 || ns < 0) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  if (n == 0 || ns == 0) return PIAFS_OK;
  int* err = nullptr;
  CK(cudaMalloc(&err, sizeof(int)));
  CK(cudaMemset(err, 0, sizeof(int)));
  launch_tridiag(a, b, c, x, n, ns, err, 0);
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(err);
  CK(e);
  CK(cudaGetLastError());
  if (h) return fail(PIAFS_ERR_SINGULAR, "zero pivot in tridiagLU");
  return PIAFS_OK;
}

int piafs_gpu_reciprocal(const double* x, double* y, long long n) {
  if (!x || !y || n < 0) return fail(PIAFS_ERR_ARGUMENT, "bad argument");
  if (n == 0) return PIAFS_OK;
  launch_reciprocal(x, y, n, 0);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  return PIAFS_OK;
}

}  // extern "C"
