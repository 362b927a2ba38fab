// A 2D grid decomposed along y into row slabs, one per rank (one GPU each):
// the C ABI of include/piafs_gpu.h's piafs_gpu_slab_*.
//
// PIAFS decomposes its grid over MPI ranks and solves the CRWENO5 systems of
// lines that cross ranks with its MPI-parallel tridiagonal solver
// (tridiagLU.c:16-85 with the reduced system of :155-240), after exchanging
// ghost points (MPIExchangeBoundariesnD.c:45-177).  Here every rank owns the
// rows [rank n1, (rank + 1) n1) of the grid (its row slab, a simulation of its
// own whose x lines are whole) and, for the y direction, the columns
// [rank n0, (rank + 1) n0) over all rows (its column slab), so that every
// y line is whole on one rank and is solved by the same one-CTA line solve as
// on an undecomposed grid.  One RK stage:
//
//   stage_begin   U_s, the deck's boundary zones of this slab, x fluxes and
//                 x reconstruction                                  (device)
//   [halo]        ghost rows from the neighbouring slabs             (caller)
//   [columns]     the state's columns, ghost rows included, to their
//                 column slab, transposed                            (caller)
//   y_pass        y fluxes, reconstruction, upwinding and the y term of the
//                 divergence, laid out per destination row slab    (device)
//   [hy]          the y term back to the row slabs                   (caller)
//   stage_end     x upwinding, hyp = x term + y term, viscous terms and
//                 source into the stage derivative                  (device)
//
// The exchanges are the caller's (piafs_b200/slab.py: all-to-all over
// torch.distributed / NCCL, or copies between slabs held in one process);
// the library gives it the device buffers.  Every value is computed by the
// same arithmetic, in the same order, as on the undecomposed grid, so the
// decomposed solution equals the undecomposed one bit for bit.
#include <cstring>
#include <string>

#include "../../include/piafs_gpu.h"
#include "deck.h"
#include "kernels.h"
#include "sim.h"

using namespace piafs;

namespace piafs {
int set_last_error(int code, const std::string& msg);   // api.cu
}

namespace {
int sfail(int code, const std::string& m) { return piafs::set_last_error(code, m); }
long long round32(long long n) { return (n + 31) / 32 * 32; }
}  // namespace

#define SCK(call)                                                                                 \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return sfail(e_ == cudaErrorMemoryAllocation ? PIAFS_ERR_MEMORY : PIAFS_ERR_CUDA,            \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                            \
  } while (0)

struct piafs_gpu_slab {
  piafs_gpu_sim* row = nullptr;   // the row slab
  int rank = 0, nranks = 1, N0 = 0, N1 = 0, n0 = 0, n1 = 0, g = 0, nvars = 0;
  int periodic_y = 0;
  DevParams Pc{}, PTc{};          // the column slab and its transposed layout
  double* utc = nullptr;          // column slab state, transposed
  double* fcc = nullptr;          // its y fluxes, transposed
  void* ifc[4] = {nullptr, nullptr, nullptr, nullptr};   // its y interface arrays
  double* dyinv = nullptr;        // the whole grid's ghosted 1/dy
  void* hy_send = nullptr;        // y term of the column slab, per destination row slab
  void* hy_recv = nullptr;        // y term of the row slab, per source column slab
  size_t hy_bytes = 0;
};

static void free_slab(piafs_gpu_slab* sl) {
  if (!sl) return;
  if (sl->row) piafs_gpu_destroy(sl->row);
  cudaFree(sl->utc);
  cudaFree(sl->fcc);
  for (auto p : sl->ifc) cudaFree(p);
  cudaFree(sl->dyinv);
  cudaFree(sl->hy_send);
  cudaFree(sl->hy_recv);
  delete sl;
}

extern "C" {

int piafs_gpu_slab_create(const char* deck_dir, int precision, int rank, int nranks, piafs_gpu_slab** out) {
  if (!deck_dir || !out) return sfail(PIAFS_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  Deck whole;
  std::string err;
  if (int r = read_deck(deck_dir, whole, err)) return sfail(r, err);
  if (int r = check_deck(whole, err)) return sfail(r, err);
  if (precision == PIAFS_PRECISION_MIXED && whole.hyp_space_scheme != "crweno5")
    return sfail(PIAFS_ERR_UNSUPPORTED, "mixed precision on a decomposed grid runs CRWENO5 only");
  Deck part;
  bool periodic_y = false;
  if (int r = restrict_rows(whole, rank, nranks, part, periodic_y, err)) return sfail(r, err);
  const std::vector<double> dy(whole.dxinv.begin() + whole.size[0] + 2 * whole.ghosts, whole.dxinv.end());
  auto* sl = new piafs_gpu_slab();
  sl->rank = rank;
  sl->nranks = nranks;
  sl->N0 = whole.size[0];
  sl->N1 = whole.size[1];
  sl->n0 = sl->N0 / nranks;
  sl->n1 = sl->N1 / nranks;
  sl->g = whole.ghosts;
  sl->nvars = whole.nvars;
  sl->periodic_y = periodic_y ? 1 : 0;
  if (int r = piafs::create_sim(std::move(part), precision, &sl->row)) {
    free_slab(sl);
    return r;
  }
  piafs_gpu_sim* s = sl->row;
  // the row slab never runs a y pass of its own
  cudaFree(s->ut);
  s->ut = nullptr;
  s->concurrent_y = false;
  cudaFree(s->fCy);
  s->fCy = nullptr;
  for (auto& p : s->iface_y) { cudaFree(p); p = nullptr; }
  // the column slab: columns [rank n0, (rank + 1) n0), every row
  DevParams& C = sl->Pc;
  C = s->P;
  C.N0 = sl->n0;
  C.N1 = sl->N1;
  C.W0 = sl->n0 + 2 * sl->g;
  C.W1 = sl->N1 + 2 * sl->g;
  C.npg = (long long)C.W0 * C.W1;
  C.ps = round32(C.npg);
  C.nint[0] = (long long)(C.N0 + 1) * C.N1;
  C.nint[1] = (long long)C.N0 * (C.N1 + 1);
  C.pis = round32(C.nint[0] > C.nint[1] ? C.nint[0] : C.nint[1]);
  C.jg0 = 0;
  C.N1g = C.N1;
  // packed passive interface values need every line in one CTA, the column
  // slab's whole-grid y lines included
  if (!crweno_line_fits(sl->N1)) s->P.pack_sp = C.pack_sp = 0;
  sl->PTc = transposed_params(C);
  const size_t planes = (size_t)C.nvars * C.ps, iplanes = (size_t)C.nvars * C.pis;
  const size_t isz = s->P.mixed ? sizeof(float) : sizeof(double);
  sl->hy_bytes = (size_t)sl->nvars * sl->N1 * sl->n0 * isz;   // = nvars n1 N0 on the receiving side
  cudaError_t e = cudaSetDevice(s->device);
  if (e == cudaSuccess) e = cudaMalloc(&sl->utc, planes * sizeof(double));
  // ghost columns of the column slab are never read by the y pass; a
  // uniform state there keeps the pointwise y fluxes finite
  if (e == cudaSuccess) {
    std::vector<double> one(planes, 1.0);
    e = cudaMemcpy(sl->utc, one.data(), planes * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&sl->fcc, planes * sizeof(double));
  for (int k = 0; k < 4 && e == cudaSuccess; k++) e = cudaMalloc(&sl->ifc[k], iplanes * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&sl->dyinv, dy.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(sl->dyinv, dy.data(), dy.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&sl->hy_send, sl->hy_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&sl->hy_recv, sl->hy_bytes);
  if (e != cudaSuccess) {
    free_slab(sl);
    return sfail(e == cudaErrorMemoryAllocation ? PIAFS_ERR_MEMORY : PIAFS_ERR_CUDA,
                 std::string("slab set-up: ") + cudaGetErrorString(e));
  }
  *out = sl;
  return PIAFS_OK;
}

void piafs_gpu_slab_destroy(piafs_gpu_slab* sl) { free_slab(sl); }

int piafs_gpu_slab_get_info(piafs_gpu_slab* sl, piafs_gpu_slab_info* info) {
  if (!sl || !info) return sfail(PIAFS_ERR_ARGUMENT, "null argument");
  std::memset(info, 0, sizeof(*info));
  info->rank = sl->rank;
  info->nranks = sl->nranks;
  info->dim[0] = sl->N0;
  info->dim[1] = sl->N1;
  info->slab_rows = sl->n1;
  info->slab_cols = sl->n0;
  info->ghosts = sl->g;
  info->nvars = sl->nvars;
  info->nstages = sl->row->deck.nstages;
  info->periodic_y = sl->periodic_y;
  info->plane_stride = sl->row->P.ps;
  info->col_plane_stride = sl->Pc.ps;
  info->hy_bytes = (long long)sl->hy_bytes;
  info->hy_value_bytes = sl->row->P.mixed ? 4 : 8;
  return PIAFS_OK;
}

int piafs_gpu_slab_sim(piafs_gpu_slab* sl, piafs_gpu_sim** row) {
  if (!sl || !row) return sfail(PIAFS_ERR_ARGUMENT, "null argument");
  *row = sl->row;
  return PIAFS_OK;
}

int piafs_gpu_slab_state(piafs_gpu_slab* sl, int stage, double** U) {
  if (!sl || !U || stage < 0 || stage >= sl->row->deck.nstages) return sfail(PIAFS_ERR_ARGUMENT, "bad argument");
  *U = stage == 0 ? sl->row->u : sl->row->U[stage];
  return PIAFS_OK;
}

int piafs_gpu_slab_buffers(piafs_gpu_slab* sl, double** utc, void** hy_send, void** hy_recv) {
  if (!sl || !utc || !hy_send || !hy_recv) return sfail(PIAFS_ERR_ARGUMENT, "null argument");
  *utc = sl->utc;
  *hy_send = sl->hy_send;
  *hy_recv = sl->hy_recv;
  return PIAFS_OK;
}

// TimeRK's stage st (TimeRK.c:40-75) up to the x pass: U_st from u and the
// earlier stage derivatives (stage 0: u itself, after TimePreStep's boundary
// conditions), the slab's boundary zones, x fluxes and reconstruction.
int piafs_gpu_slab_stage_begin(piafs_gpu_slab* sl, int st) {
  if (!sl || st < 0 || st >= sl->row->deck.nstages) return sfail(PIAFS_ERR_ARGUMENT, "bad argument");
  piafs_gpu_sim* s = sl->row;
  const Deck& d = s->deck;
  double* Us = st == 0 ? s->u : s->U[st];
  if (st > 0) {
    const double* dd[MAX_STAGES];
    double a[MAX_STAGES];
    for (int j = 0; j < st; j++) { dd[j] = s->Ud[j]; a[j] = d.dt * d.A[st * MAX_STAGES + j]; }
    launch_stage((long long)s->P.nvars * s->P.ps, Us, s->u, dd, a, st, s->stream);
  }
  enqueue_bc(s, Us);
  enqueue_recon(s, Us, 0, s->iface);
  SCK(cudaGetLastError());
  return PIAFS_OK;
}

// The y pass on the column slab (its state filled by the caller): y fluxes,
// reconstruction along the whole y lines, upwinding at the y interfaces and
// the y term of the divergence into the send buffer of the y term.
int piafs_gpu_slab_y_pass(piafs_gpu_slab* sl, int st) {
  if (!sl || st < 0 || st >= sl->row->deck.nstages) return sfail(PIAFS_ERR_ARGUMENT, "bad argument");
  piafs_gpu_sim* s = sl->row;
  const DevParams& C = sl->Pc;
  launch_flux(C, sl->utc, sl->fcc, 1, s->stream);
  if (C.scheme == CRWENO5) {
    if (launch_crweno(sl->PTc, sl->utc, sl->fcc, sl->ifc[0], sl->ifc[1], sl->ifc[2], sl->ifc[3], 0, s->err,
                      s->stream))
      return sfail(PIAFS_ERR_UNSUPPORTED, "CRWENO5 y lines too long");
  } else {
    launch_weno5(sl->PTc, sl->utc, sl->fcc, sl->ifc[0], sl->ifc[1], sl->ifc[2], sl->ifc[3], 0, s->stream);
  }
  const void* yi[4] = {sl->ifc[0], sl->ifc[1], sl->ifc[2], sl->ifc[3]};
  launch_slab_upwind_y(C, sl->utc, yi, sl->dyinv, sl->hy_send, sl->n1, s->stream);
  SCK(cudaGetLastError());
  return PIAFS_OK;
}

// The rest of stage st's right-hand side (TimeRHSFunctionExplicit.c:29-77):
// x upwinding, hyp = x term + the received y term, rhs = -hyp, then the
// viscous terms and the source.
int piafs_gpu_slab_stage_end(piafs_gpu_slab* sl, int st) {
  if (!sl || st < 0 || st >= sl->row->deck.nstages) return sfail(PIAFS_ERR_ARGUMENT, "bad argument");
  piafs_gpu_sim* s = sl->row;
  const Deck& d = s->deck;
  double* Us = st == 0 ? s->u : s->U[st];
  const void* xi[4] = {s->iface[0], s->iface[1], s->iface[2], s->iface[3]};
  launch_upwind_div2d_hy(s->P, Us, xi, s->dxinv, sl->hy_recv, sl->n0, s->Ud[st], 1, s->stream);
  launch_visc_source(s->P, Us, s->dxinv, s->imap, s->tdev, d.c[st], s->Ud[st], 1, 1, s->stream);
  SCK(cudaGetLastError());
  return PIAFS_OK;
}

// TimeRK's step completion (TimeRK.c:83-99) and the clock; with_norm also
// sums the squared change of u over the slab (piafs_gpu_slab_norm_sum).
int piafs_gpu_slab_step_end(piafs_gpu_slab* sl, int with_norm) {
  if (!sl) return sfail(PIAFS_ERR_ARGUMENT, "null argument");
  piafs_gpu_sim* s = sl->row;
  const Deck& d = s->deck;
  const double* dd[MAX_STAGES];
  double b[MAX_STAGES];
  for (int j = 0; j < d.nstages; j++) { dd[j] = s->Ud[j]; b[j] = d.dt * d.b[j]; }
  if (with_norm) SCK(cudaMemsetAsync(s->norm_acc, 0, sizeof(double), s->stream));
  launch_update(s->P, s->u, dd, b, d.nstages, with_norm ? s->norm_acc : nullptr, s->stream);
  launch_advance_time(s->tdev, d.dt, s->stream);
  s->t += d.dt;
  s->iter++;
  SCK(cudaGetLastError());
  return PIAFS_OK;
}

int piafs_gpu_slab_norm_sum(piafs_gpu_slab* sl, double* sum) {
  if (!sl || !sum) return sfail(PIAFS_ERR_ARGUMENT, "null argument");
  piafs_gpu_sim* s = sl->row;
  SCK(cudaMemcpyAsync(sum, s->norm_acc, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  SCK(cudaStreamSynchronize(s->stream));
  return PIAFS_OK;
}

}  // extern "C"
