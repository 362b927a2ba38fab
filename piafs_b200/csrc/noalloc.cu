// Hyperbolic term without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need the
// hyperbolic term: a plugin embedded in an application whose memory manager
// owns every byte of the device and forbids allocations behind its back, or
// a host loop that must not pay cudaMalloc's implicit device synchronisation
// or risk an out-of-memory failure in the middle of a run.
// piafs_gpu_HyperbolicFunction_noalloc serves them: it runs the same kernels
// as piafs_gpu_HyperbolicFunction (component-wise interpolation), but the
// working arrays those kernels need (the structure-of-arrays copy of the
// state, the cell-centred flux, the four reconstructed interface arrays and
// the result) live in one file-scope __device__ array of fixed size instead
// of buffers obtained from cudaMalloc.
//
// Rules of use
//   - The array is PIAFS_NOALLOC_SCRATCH_BYTES (64 MiB) on every GPU that
//     loads this library, held until the process exits.  Problems whose
//     working set does not fit are rejected with PIAFS_ERR_ARGUMENT.
//   - The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and caches it; make that
//     first call before any stream capture begins.
//   - Every call on a device shares the one array and leaves its contents
//     behind.  The call clears what must start at zero; calls whose work
//     overlaps on the GPU (other streams, other host threads) race on the
//     array and must be serialised by the caller.
//   - The call copies the zero-pivot flag to the host and synchronises its
//     stream before it returns.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/piafs_gpu.h"
#include "kernels.h"

using namespace piafs;

#define PIAFS_NOALLOC_SCRATCH_BYTES (64ull << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[PIAFS_NOALLOC_SCRATCH_BYTES];

namespace piafs {
int set_last_error(int code, const std::string& msg);   // api.cu: piafs_gpu_last_error()
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {nullptr};

int nfail(int code, const std::string& m) { return piafs::set_last_error(code, m); }

long long round32(long long n) { return (n + 31) / 32 * 32; }
}  // namespace

extern "C" int piafs_gpu_HyperbolicFunction_noalloc(const piafs_gpu_hyp_params* prm, double* hyp, const double* u,
                                                    const double* dxinv, void* stream) {
  if (!prm || !hyp || !u || !dxinv) return nfail(PIAFS_ERR_ARGUMENT, "null argument");
  const piafs_gpu_hyp_params& q = *prm;
  if (q.ndims < 1 || q.ndims > 2 || q.nvars < 1 || q.ghosts < 3 || q.dim[0] < 3 || (q.ndims == 2 && q.dim[1] < 3))
    return nfail(PIAFS_ERR_ARGUMENT, "bad grid description");
  if ((q.model == NS2D) != (q.ndims == 2) || (q.model != NS2D && q.model != EULER1D))
    return nfail(PIAFS_ERR_ARGUMENT, "model does not match ndims");
  if (q.model == NS2D ? q.nvars < 4 : q.nvars < 3) return nfail(PIAFS_ERR_ARGUMENT, "nvars too small for the model");
  if (q.scheme != WENO5 && q.scheme != CRWENO5 && q.scheme != UPW5)
    return nfail(PIAFS_ERR_ARGUMENT, "scheme must be WENO5, CRWENO5 or UPW5");
  if (q.upwind < UPW_ROE || q.upwind > UPW_RUSANOV) return nfail(PIAFS_ERR_ARGUMENT, "bad upwinding scheme");
  if (q.weno_type < W_JS || q.weno_type > W_YC) return nfail(PIAFS_ERR_ARGUMENT, "bad WENO weight type");

  DevParams P;
  std::memset(&P, 0, sizeof(P));
  P.ndims = q.ndims; P.nvars = q.nvars; P.ghosts = q.ghosts;
  P.N0 = q.dim[0]; P.N1 = q.ndims == 2 ? q.dim[1] : 1;
  P.W0 = P.N0 + 2 * P.ghosts; P.W1 = q.ndims == 2 ? P.N1 + 2 * P.ghosts : 1; P.g1 = q.ndims == 2 ? P.ghosts : 0;
  P.N1g = P.N1;
  P.npg = (long long)P.W0 * P.W1;
  P.ps = round32(P.npg);
  P.nint[0] = q.ndims == 1 ? P.N0 + 1 : (long long)(P.N0 + 1) * P.N1;
  P.nint[1] = q.ndims == 1 ? 0 : (long long)P.N0 * (P.N1 + 1);
  P.pis = round32(P.nint[0] > P.nint[1] ? P.nint[0] : P.nint[1]);
  P.model = q.model; P.scheme = q.scheme; P.upwind = q.upwind; P.weno_type = q.weno_type;
  P.no_limiting = q.no_limiting; P.eps = q.weno_eps; P.gamma = q.gamma; P.bc_gamma = q.gamma;
  if (P.scheme == CRWENO5)
    for (int d = 0; d < P.ndims; d++)
      if (crweno_cluster_size(d == 0 ? P.N0 : P.N1) < 0)
        return nfail(PIAFS_ERR_UNSUPPORTED, "crweno5 lines longer than 32769 points are outside the GPU path");

  // working set: state, flux and result planes, four interface plane sets,
  // the zero-pivot flag
  const unsigned long long planes = (unsigned long long)P.nvars * P.ps * sizeof(double);
  const unsigned long long iplanes = (unsigned long long)P.nvars * P.pis * sizeof(double);
  const unsigned long long need = 3 * planes + 4 * iplanes + 256;
  if (need > PIAFS_NOALLOC_SCRATCH_BYTES)
    return nfail(PIAFS_ERR_ARGUMENT, "problem needs " + std::to_string(need >> 20) + " MiB of working memory, " +
                                         "more than the " + std::to_string(PIAFS_NOALLOC_SCRATCH_BYTES >> 20) +
                                         " MiB allocation-free scratch");

  // device address of the scratch array, looked up once per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return nfail(PIAFS_ERR_UNSUPPORTED, "device index out of range");
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return nfail(PIAFS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addr[dev] = p;
    }
    base = (unsigned char*)g_addr[dev];
  }
  double* U = (double*)base;
  double* F = (double*)(base + planes);
  double* H = (double*)(base + 2 * planes);
  double* I[4];
  for (int k = 0; k < 4; k++) I[k] = (double*)(base + 3 * planes + k * iplanes);
  int* err = (int*)(base + 3 * planes + 4 * iplanes);

  cudaStream_t s = (cudaStream_t)stream;
  // the result accumulates over directions and the flag over lines: both
  // start at zero; the other arrays are fully overwritten before being read
  e = cudaMemsetAsync(H, 0, planes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  launch_aos_to_soa(u, U, P.npg, P.nvars, P.ps, s);
  for (int d = 0; d < P.ndims; d++) {
    launch_flux(P, U, F, d, s);
    if (P.scheme != CRWENO5) launch_weno5(P, U, F, I[0], I[1], I[2], I[3], d, s);
    else launch_crweno(P, U, F, I[0], I[1], I[2], I[3], d, err, s);
    launch_upwind_div(P, U, I[0], I[1], I[2], I[3], dxinv, H, d, d == 0 ? 2 : 3, s);
  }
  launch_soa_to_aos(H, hyp, P.npg, P.nvars, P.ps, s);
  int flag = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return nfail(PIAFS_ERR_CUDA, std::string("hyperbolic term: ") + cudaGetErrorString(e));
  if (flag) return nfail(PIAFS_ERR_SINGULAR, "zero pivot in a CRWENO5 line solve");
  return PIAFS_OK;
}
