/* piafs_hypar.h -- the GPU path attached to the reference's own simulation
 * objects (libpiafs_hypar.so, built against llnl/piafs's include/ with
 * -Dserial, the single-rank layout).
 *
 * Where piafs_gpu.h starts from an input deck, these entry points start
 * from what the reference has already built in memory: its
 * SimulationObject array (include/simulation_object.h:26-33) after
 * InitializeSolvers -- the HyPar object (include/hypar.h:25-333) with its
 * grid, ghosted solution, boundary objects (DomainBoundary,
 * include/boundaryconditions.h:55-85), WENO parameters (WENOParameters,
 * include/interpolation.h:184-209), physics object (NavierStokes2D / Euler1D
 * with their Chemistry, include/physicalmodels/chemistry.h:139-260) and RK
 * tableau (ExplicitRKParameters, include/timeintegration_struct.h:168-174).
 * Nothing is read from files: restart state, working directory and any
 * change the caller made in memory are what the GPU sees.
 *
 * The signatures are the reference's function-pointer signatures, so the
 * entry points can be stored in the reference's own pointers:
 *   solver->TimeIntegrate = piafs_gpu_TimeRK_ts          (InitializeSolvers.c:204)
 *   TS->RHSFunction       = piafs_gpu_hypar_RHSFunction  (TimeInitialize.c:114)
 *   solver->HyperbolicFunction, ParabolicFunction, SourceFunction,
 *   ApplyBoundaryConditions, FFunction, Upwind, InterpolateInterfacesHyp,
 *   FirstDerivativePar = piafs_gpu_hypar_*                (include/hypar.h:204-290)
 * Return values are 0 or a PIAFS_ERR_* code of piafs_gpu.h (message in
 * piafs_gpu_last_error()); the reference ignores them outside -Ddebug
 * builds, so failures are also printed to stderr.
 */
#ifndef PIAFS_HYPAR_H
#define PIAFS_HYPAR_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mirror the reference's initialised simulations simobjs[0 .. nsims-1]
 * (SimulationObject*) on the current CUDA device, in PIAFS_PRECISION_FP64 or
 * _MIXED; one MPI rank per simulation.  The device state starts from each
 * solver->u at time `t` (TS->waqt; restart_iter x dt after TimeInitialize).
 * Attaching a simulation that is attached already re-uploads its solver->u. */
int piafs_gpu_attach(void* simobjs, int nsims, int precision, double t);
/* Release the device copies of simobjs[0 .. nsims-1]. */
int piafs_gpu_detach(void* simobjs, int nsims);

/* Bring solver->u of simobjs[0 .. nsims-1] up to date with the device state
 * (piafs_gpu_TimeRK_ts refreshes it only after the steps the reference
 * reads; callers that read the host state at other steps call this). */
int piafs_gpu_hypar_sync(void* simobjs, int nsims);

/* TimeIntegrate (TimeRK.c:34, called as TS->TimeIntegrate(TS) from
 * TimeStep.c:16-24): one time step of every simulation of the
 * TimeIntegration object `ts`, on the device.  Simulations that are not
 * attached yet are attached (FP64) on their first step.  The state stays on
 * the device between steps; solver->u is brought up to date after the steps
 * whose result the reference reads on the host -- the residual norm and CFL
 * of every screen_op_iter-th step (TimePreStep.c:54-65, TimePostStep.c:36-54),
 * the output of every file_op_iter-th step and the last step (Solve.cpp:
 * 54-95) -- together with the photon density (Chemistry::nv_hnu) the species
 * output writes.  The reference's physics pre-step hooks of these models
 * (NavierStokes2DPreStep.c, Euler1DPreStep.c) leave u unchanged, and its
 * pre-step boundary conditions only rewrite ghosts that every GPU step
 * rewrites the same way, so the device copy never goes stale.  The call
 * counters count_hyp / count_par / count_sou advance as the reference's RK
 * stages would advance them (function_counts.dat). */
int piafs_gpu_TimeRK_ts(void* ts);

/* The operators on the reference's HOST arrays (ghosted, array of
 * structures, as HyPar holds them), with the reference's signatures; `s` is
 * the attached HyPar*, `m` its MPIVariables* (unused on one rank).  Each
 * call copies its inputs to the device, runs the GPU operator and copies the
 * outputs back; they exist so that the reference can call each operator
 * through its own pointer, and for checking operators one by one. */
/* TimeRHSFunctionExplicit (TimeRHSFunctionExplicit.c:29): fills the ghosts
 * of u (boundary conditions) and rhs = -hyp + par + source */
int piafs_gpu_hypar_RHSFunction(double* rhs, double* u, void* s, void* m, double t);
/* HyperbolicFunction (HyperbolicFunction.c:34); FFunction == NULL gives a
 * zero hyperbolic term as in the reference, the physics is otherwise the
 * attached model's own */
int piafs_gpu_hypar_HyperbolicFunction(double* hyp, double* u, void* s, void* m, double t, int LimFlag,
                                       int (*FFunction)(double*, double*, int, void*, double),
                                       int (*Upwind)(double*, double*, double*, double*, double*, double*, int,
                                                     void*, double));
/* NavierStokes2DParabolicFunction (NavierStokes2DParabolicFunction.c:41) */
int piafs_gpu_hypar_ParabolicFunction(double* par, double* u, void* s, void* m, double t);
/* SourceFunction (SourceFunction.c:21) */
int piafs_gpu_hypar_SourceFunction(double* source, double* u, void* s, void* m, double t);
/* ApplyBoundaryConditions (ApplyBoundaryConditions.c:31) on u */
int piafs_gpu_hypar_ApplyBoundaryConditions(void* s, void* m, double* u, double* uref, double t);
/* FFunction (NavierStokes2DFlux.c:24 / Euler1DFlux.c:19) */
int piafs_gpu_hypar_FFunction(double* f, double* u, int dir, void* s, double t);
/* Upwind (NavierStokes2DUpwind.c / Euler1DUpwind.c): interface arrays of
 * direction dir, u ghosted */
int piafs_gpu_hypar_Upwind(double* fI, double* fL, double* fR, double* uL, double* uR, double* u, int dir,
                           void* s, double t);
/* InterpolateInterfacesHyp with its weights (SetInterpLimiterVar +
 * Interp1PrimFifthOrderWENO.c:77 / Interp1PrimFifthOrderCRWENO.c:81) */
int piafs_gpu_hypar_InterpolateInterfacesHyp(double* fI, double* fC, double* u, double* x, int upw, int dir,
                                             void* s, void* m, int uflag);
/* FirstDerivativePar = FirstDerivativeFirstOrder (FirstDerivativeFirstOrder.c:40)
 * on arrays of nvars values per ghosted point */
int piafs_gpu_hypar_FirstDerivativePar(double* Df, double* f, int dir, int bias, void* s, void* m);

#ifdef __cplusplus
}
#endif
#endif /* PIAFS_HYPAR_H */
