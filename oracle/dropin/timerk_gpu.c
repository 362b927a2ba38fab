/* The reference-side binding of the GPU time integrator (test harness).
 *
 * The reference selects its integrator by storing TimeRK
 * (src/TimeIntegration/TimeRK.c:34) in solver->TimeIntegrate
 * (src/Simulation/InitializeSolvers.c:204), which TimeStep calls
 * (src/TimeIntegration/TimeStep.c:16-24).  This file supplies a TimeRK of the
 * same signature that hands the step to the GPU library
 * (piafs_gpu_TimeRK_ts, include/piafs_hypar.h).  oracle/Makefile links it
 * ahead of the reference's own objects -- its unmodified main, initialisation,
 * output and diagnostics -- so the archive member holding the CPU TimeRK is
 * never pulled in: the reference binary runs with the GPU path as its time
 * integrator and nothing else changed.
 *
 * Built with -DPIAFS_CHECK_OPERATORS, the last step also holds the GPU
 * operators, called through the HyPar-signature entry points on the
 * reference's host arrays, to the reference's own operators (the CPU
 * functions its pointers still hold) on the same state -- the developed
 * state before the last step, where every operator carries signal (on a
 * quiescent or uniform initial state the hyperbolic term is round-off) --
 * and prints one line per operator: "check <operator> <worst per-variable
 * relative L2>" over the interior points (ghost points included for the
 * boundary conditions).
 */
#include <stdio.h>
#include <stdlib.h>

#include "piafs_hypar.h"

/* The reference ignores TimeIntegrate's status outside -Ddebug builds
 * (TimeStep.c:22); a step the GPU could not take ends the run here rather
 * than let the reference write an unadvanced solution. */
static int gpu_step(void* ts) {
  const int r = piafs_gpu_TimeRK_ts(ts);
  if (r) {
    fprintf(stderr, "TimeRK (GPU): step failed with status %d\n", r);
    exit(EXIT_FAILURE);
  }
  return 0;
}

#ifdef PIAFS_CHECK_OPERATORS
#include <math.h>
#include <string.h>

#include <hypar.h>
#include <mpivars_struct.h>
#include <simulation_object.h>
#include <timeintegration_struct.h>

#include "piafs_gpu.h"

/* worst per-variable relative L2 of got against want; interior points only
 * unless all is set; absolute where the reference norm is below 1e-15 */
static double worst_rel_l2(const HyPar* h, const double* got, const double* want, int all) {
  const int g = h->ghosts, nv = h->nvars;
  const int W0 = h->dim_local[0] + 2 * g;
  const int W1 = h->ndims > 1 ? h->dim_local[1] + 2 * g : 1;
  const int g1 = h->ndims > 1 ? g : 0;
  double worst = 0.0;
  for (int v = 0; v < nv; v++) {
    double num = 0.0, den = 0.0;
    for (int j = all ? 0 : g1; j < (all ? W1 : W1 - g1); j++)
      for (int i = all ? 0 : g; i < (all ? W0 : W0 - g); i++) {
        const long p = (long)i + (long)W0 * j;
        const double d = got[p * nv + v] - want[p * nv + v];
        num += d * d;
        den += want[p * nv + v] * want[p * nv + v];
      }
    const double e = den > 1e-30 ? sqrt(num / den) : sqrt(num);
    if (e > worst || e != e) worst = e;
  }
  return worst;
}

static void check_operators(TimeIntegration* TS) {
  SimulationObject* sim = (SimulationObject*)TS->simulation;
  HyPar* h = &sim[0].solver;
  MPIVariables* m = &sim[0].mpi;
  const double t = TS->waqt;
  const size_t n = (size_t)h->npoints_local_wghosts * h->nvars;
  double *u = malloc(n * sizeof(double)), *a = calloc(n, sizeof(double)), *b = calloc(n, sizeof(double));
  double *ua = malloc(n * sizeof(double)), *ub = malloc(n * sizeof(double));
  /* the device state of the steps taken so far, into the host array */
  if (piafs_gpu_hypar_sync(sim, TS->nsims)) {
    printf("check sync failed: %s\n", piafs_gpu_last_error());
    return;
  }
  memcpy(u, h->u, n * sizeof(double));
  /* ghost fill of the stage input (ApplyBoundaryConditions.c:31) */
  memcpy(ua, u, n * sizeof(double));
  memcpy(ub, u, n * sizeof(double));
  h->ApplyBoundaryConditions(h, m, ua, NULL, t);
  piafs_gpu_hypar_ApplyBoundaryConditions(h, m, ub, NULL, t);
  printf("check ApplyBoundaryConditions %.3e\n", worst_rel_l2(h, ub, ua, 1));
  memcpy(u, ua, n * sizeof(double));
  /* the right-hand side and its terms on the filled state */
  memset(a, 0, n * sizeof(double)); memset(b, 0, n * sizeof(double));
  h->HyperbolicFunction(a, u, h, m, t, 1, h->FFunction, h->Upwind);
  piafs_gpu_hypar_HyperbolicFunction(b, u, h, m, t, 1, h->FFunction, h->Upwind);
  printf("check HyperbolicFunction %.3e\n", worst_rel_l2(h, b, a, 0));
  if (h->ParabolicFunction) {
    memset(a, 0, n * sizeof(double)); memset(b, 0, n * sizeof(double));
    h->ParabolicFunction(a, u, h, m, t);
    piafs_gpu_hypar_ParabolicFunction(b, u, h, m, t);
    printf("check ParabolicFunction %.3e\n", worst_rel_l2(h, b, a, 0));
  }
  memset(a, 0, n * sizeof(double)); memset(b, 0, n * sizeof(double));
  h->SourceFunction(a, u, h, m, t);
  piafs_gpu_hypar_SourceFunction(b, u, h, m, t);
  printf("check SourceFunction %.3e\n", worst_rel_l2(h, b, a, 0));
  memcpy(ua, u, n * sizeof(double));
  memcpy(ub, u, n * sizeof(double));
  memset(a, 0, n * sizeof(double)); memset(b, 0, n * sizeof(double));
  TS->RHSFunction(a, ua, h, m, t);
  piafs_gpu_hypar_RHSFunction(b, ub, h, m, t);
  printf("check RHSFunction %.3e\n", worst_rel_l2(h, b, a, 0));
  for (int d = 0; d < h->ndims; d++) {
    memset(a, 0, n * sizeof(double)); memset(b, 0, n * sizeof(double));
    h->FFunction(a, u, d, h, t);
    piafs_gpu_hypar_FFunction(b, u, d, h, t);
    printf("check FFunction_%d %.3e\n", d, worst_rel_l2(h, b, a, 1));
  }
  fflush(stdout);
  free(u); free(a); free(b); free(ua); free(ub);
}

int TimeRK(void* ts) {
  TimeIntegration* TS = (TimeIntegration*)ts;
  if (TS->iter == TS->n_iter - 1) {
    /* attached by the earlier steps, or here when the run has one step */
    if (TS->iter == TS->restart_iter &&
        piafs_gpu_attach(TS->simulation, TS->nsims, PIAFS_PRECISION_FP64, TS->waqt)) {
      printf("check attach failed: %s\n", piafs_gpu_last_error());
      exit(EXIT_FAILURE);
    }
    check_operators(TS);
  }
  return gpu_step(ts);
}

#else

int TimeRK(void* ts) { return gpu_step(ts); }

#endif
