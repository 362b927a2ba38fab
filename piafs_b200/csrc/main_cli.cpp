// piafs-gpu: command-line drop-in for the reference PIAFS binary on the
// B200 path.  Like src/main.cpp it runs the input deck of the current
// directory (or of the directory given as the first argument) and writes the
// op_NNNNN.bin files there.
#include <chrono>
#include <cstdio>
#include <string>

#include "../../include/piafs_gpu.h"

int main(int argc, char** argv) {
  const auto start = std::chrono::steady_clock::now();
  std::string dir = argc > 1 ? argv[1] : ".";
  piafs_gpu_sim* sim = nullptr;
  int r = piafs_gpu_create(dir.c_str(), PIAFS_PRECISION_FP64, &sim);
  if (r) {
    std::fprintf(stderr, "piafs-gpu: set-up failed (%d): %s\n", r, piafs_gpu_last_error());
    return 1;
  }
  piafs_gpu_info info;
  piafs_gpu_get_info(sim, &info);
  std::printf("piafs-gpu: %dD, nvars %d, grid %d x %d, %d steps of dt %g (gamma %.4e, Re %.4e, Pr %.4e)\n",
              info.ndims, info.nvars, info.dim[0], info.dim[1], info.n_iter, info.dt, info.gamma, info.Re, info.Pr);
  const auto t0 = std::chrono::steady_clock::now();
  r = piafs_gpu_Solve(sim, dir.c_str());
  const double solver_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (r) {
    std::fprintf(stderr, "piafs-gpu: solve failed (%d): %s\n", r, piafs_gpu_last_error());
    piafs_gpu_destroy(sim);
    return 1;
  }
  piafs_gpu_get_info(sim, &info);
  std::printf("piafs-gpu: completed %d steps, final time %f, CFL %.4e, norm %.4e\n", info.iter, info.t, info.cfl,
              info.norm);
  if (info.singular) std::printf("piafs-gpu: warning: %d steps met a zero pivot\n", info.singular);
  // errors.dat, conservation.dat, function_counts.dat (main.cpp:223-240)
  const double main_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
  if (piafs_gpu_WriteErrors(sim, dir.c_str(), solver_s, main_s))
    std::fprintf(stderr, "piafs-gpu: %s\n", piafs_gpu_last_error());
  piafs_gpu_destroy(sim);
  return 0;
}
