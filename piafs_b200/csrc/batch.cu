// Batched simulations: many independent PIAFS runs advanced together (sm_100a).
//
// The reference runs an ensemble one member after another (one deck each,
// OutputSolution.cpp).  Here every member lives on the device at once and one
// persistent kernel per Runge-Kutta stage advances all of them, a CTA per
// tile of a device-side tile list (batch_tile.cuh has the stage kernel; the
// FP64 and the mixed-precision instances are compiled in batch_stage_fp64.cu
// and batch_stage_mixed.cu).  A member's FP64 result agrees with its deck run
// alone to rounding (the compiler contracts multiply-adds differently in the
// fused kernel), and in either precision it is bit for bit the same whatever
// other members share the batch, since a tile's arithmetic depends only on
// its own member.
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
#include "batch_tile.cuh"

namespace piafs {
int set_last_error(int code, const std::string& msg);   // api.cu: piafs_gpu_last_error()
}

using namespace piafs;
using namespace piafs::batch;

namespace {

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

bool mixed(const piafs_gpu_batch* B) { return B->precision == PIAFS_PRECISION_MIXED; }

long long smem_bytes(const piafs_gpu_batch* B, int shape, int nv) {
  return mixed(B) ? StageTable<true>::smem(shape, nv) : StageTable<false>::smem(shape, nv);
}

int persistent_grid(piafs_gpu_batch* B) {
  // PIAFS_GPU_BATCH_GRID=n overrides the number of persistent CTAs
  if (const char* g = std::getenv("PIAFS_GPU_BATCH_GRID")) {
    const int n = std::atoi(g);
    if (n > 0) return n;
  }
  const long long sm = smem_bytes(B, B->shape, std::max(B->max_nv, 1));
  int per_sm = 0;
  per_sm = mixed(B) ? StageTable<true>::per_sm(B->shape, sm) : StageTable<false>::per_sm(B->shape, sm);
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
  const long long sm = smem_bytes(B, B->shape, B->max_nv);
  BCK(mixed(B) ? StageTable<true>::attr(B->shape, sm) : StageTable<false>::attr(B->shape, sm));
  cudaGraph_t g;
  BCK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < B->max_stages && e == cudaSuccess; s++) {
    if (mixed(B)) StageTable<true>::launch(B->shape, grid, sm, B->stream, B->dmem, B->dstate, B->dtiles, B->dntiles, s);
    else StageTable<false>::launch(B->shape, grid, sm, B->stream, B->dmem, B->dstate, B->dtiles, B->dntiles, s);
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
  if (P.scheme == CRWENO5) { err = "batched members use hyp_space_scheme weno5 or upw5"; return PIAFS_ERR_UNSUPPORTED; }
  if (P.viscous && P.par4) { err = "batched members use par_space_scheme 2"; return PIAFS_ERR_UNSUPPORTED; }
  if (P.char_interp) { err = "batched members use hyp_interp_type components"; return PIAFS_ERR_UNSUPPORTED; }
  if (!hm.deck.sponges.empty()) { err = "batched members have no sponge zones"; return PIAFS_ERR_UNSUPPORTED; }
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
    if (smem_bytes(B, B->shape, std::max(B->max_nv, P.nvars)) > optin)
      return nfail(PIAFS_ERR_UNSUPPORTED, "too many variables for the batched stage kernel's shared-memory tile");
  }
  P.mixed = mixed(B) ? 1 : 0;
  const int ns = d.nstages;
  const size_t planes = (size_t)P.nvars * P.ps;
  const size_t ndx = d.dxinv.size(), nim = req ? (P.chem ? (size_t)P.npg : 0) : d.imap.size();
  std::vector<size_t> zoff;
  const std::vector<double> zvals = pack_zone_values(d, zoff);
  const size_t bytes = ((3 + ns) * planes + ndx + nim + zvals.size()) * sizeof(double);
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
  double* zv = im + nim;
  bm.nzones = (int)d.zones.size();
  for (int z = 0; z < bm.nzones; z++) bm.zones[z] = d.zones[z];
  bind_zone_values(d, zoff, zv, bm.zones);
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
  if (e == cudaSuccess && !zvals.empty())
    e = cudaMemcpyAsync(zv, zvals.data(), zvals.size() * sizeof(double), cudaMemcpyHostToDevice, B->stream);
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
    if (k < 0) return nfail(PIAFS_ERR_ARGUMENT, "tile_x must be 8, 16 or 32");
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
    if (smem_bytes(B, c, B->max_nv) > optin) continue;
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
      if (smem_bytes(B, i, B->max_nv) > optin)
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
                          unsigned long long budget, unsigned long long max_points, int steps_per_round,
                          piafs_gpu_serve_result* out) {
  if (n < 0 || (n > 0 && (!reqs || !arrival_s || !out)) || steps_per_round < 1)
    return nfail(PIAFS_ERR_ARGUMENT, "bad argument");
  for (int k = 1; k < n; k++)
    if (arrival_s[k] < arrival_s[k - 1]) return nfail(PIAFS_ERR_ARGUMENT, "arrival times must be nondecreasing");
  piafs_gpu_batch* B = nullptr;
  if (int r = piafs_gpu_batch_create(precision, budget, &B)) return r;
  std::vector<int> slot_req;     // member id -> request index
  int next = 0, finished = 0, rc = PIAFS_OK;
  unsigned long long resident = 0;   // grid points of the resident requests
  auto points = [&](int k) -> unsigned long long {
    const unsigned long long n1 = (unsigned long long)std::max(reqs[k].n, 0);
    return reqs[k].kind == PIAFS_REQUEST_NS2D_BEAM ? n1 * n1 : n1;
  };
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
      if (max_points && resident > 0 && resident + points(next) > max_points) break;
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
      resident += points(next);
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
      resident -= points(k);
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
