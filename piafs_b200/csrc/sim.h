// The simulation object behind the C ABI's piafs_gpu_sim handle (private to
// the library: api.cu, slab.cu).
#pragma once
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/piafs_gpu.h"
#include "deck.h"
#include "kernels.h"

using namespace piafs;

struct piafs_gpu_sim {
  Deck deck;
  DevParams P;
  int precision = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  // 2D Navier-Stokes with a transposed y pass: the y pass (transpose, y
  // flux into fCy, y line solve) on ystream, concurrent with the x pass,
  // forked from and joined to `stream` by the two events
  bool concurrent_y = false;
  cudaStream_t ystream = nullptr;
  cudaEvent_t yfork = nullptr, yjoin = nullptr;
  double* fCy = nullptr;
  // device state (structure of arrays)
  double* u = nullptr;
  double* U[MAX_STAGES] = {nullptr};       // U[0] aliases u
  double* Ud[MAX_STAGES] = {nullptr};
  double* fC = nullptr;
  double* iface[5] = {nullptr};            // uL, uR, fL, fR, operator scratch
  double* iface_y[4] = {nullptr};          // uL, uR, fL, fR of the y direction (2D)
  double* scratch = nullptr;               // ghosted plane set for operator calls
  double* ut = nullptr;                    // transposed state of the y-direction CRWENO5 pass
  DevParams PT;                            // the transposed grid
  double* dxinv = nullptr;
  double* imap = nullptr;
  double* tdev = nullptr;                  // simulation time on the device
  double* top_t = nullptr;                 // time for operator calls
  double* norm_acc = nullptr;
  unsigned long long* cfl_acc = nullptr;
  int* err = nullptr;
  double* aos = nullptr;                   // ghosted AoS staging (host transfers)
  size_t aos_bytes = 0;
  double* hnu = nullptr;                   // photon density [nz][ps] of the last RK stage (species output)
  // sponge zones: extents on the host, ramp and reference state in sponge_buf
  struct SpongeDev { int dim; int is[2], ie[2]; size_t sig_off, ref_off; };
  std::vector<SpongeDev> sponges;
  double* sponge_buf = nullptr;
  double* zone_buf = nullptr;              // boundary zones' values (Zone::val)
  double* crwchar = nullptr;               // block rows of the characteristic CRWENO5 line solves
  // host mirror of the clock
  double t = 0.0;
  int iter = 0;
  double last_cfl = -1.0, last_norm = 0.0;
  int singular = 0;
  // CUDA graphs of one step: [0] plain, [1] with residual norm
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  bool use_graph = true;
};

namespace piafs {
// Cell-centred flux and interface values (uL, uR, fL, fR into I) of
// direction d of the simulation's grid; an event is recorded after the flux
// and after the reconstruction when ev is given.
void enqueue_recon(piafs_gpu_sim* s, const double* U, int d, double* const* I, cudaEvent_t* ev = nullptr,
                   int* k = nullptr);
// The deck's boundary zones applied to the ghost points of u.
void enqueue_bc(piafs_gpu_sim* s, double* u);
}  // namespace piafs
