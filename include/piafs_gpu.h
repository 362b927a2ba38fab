/* piafs_gpu.h -- C ABI of the B200 (sm_100a) implementation of PIAFS's
 * per-stage right-hand side and explicit Runge-Kutta time step.
 *
 * The library replaces the hot path behind the reference's function-pointer
 * interface on HyPar (include/hypar.h:204-290 in llnl/piafs): TimeIntegrate,
 * HyperbolicFunction, InterpolateInterfacesHyp, Upwind, FFunction,
 * ParabolicFunction, FirstDerivativePar, SourceFunction and
 * ApplyBoundaryConditions.  It reads the reference's input deck (solver.inp,
 * boundary.inp, physics.inp, chemistry.inp, weno.inp, initial.inp, imap.inp)
 * and writes the reference's binary output files, so a deck runs unchanged on
 * either implementation.
 *
 * Conventions
 *   - Every function returns PIAFS_OK (0) or a PIAFS_ERR_* code; the message
 *     of the last failure on the calling thread is piafs_gpu_last_error().
 *     No function aborts the process.
 *   - Host arrays use the reference layout: array of structures, variable
 *     index fastest, then dim0, then dim1, ghost points included
 *     (include/arrayfunctions.h:43-50).  Interface arrays have no ghosts and
 *     dim_d + 1 entries along the reconstruction direction
 *     (src/Simulation/Initialize.c:165-174).
 *   - "Device" arguments are CUDA device pointers in that same layout.
 *   - A simulation object is used by one host thread at a time; every call is
 *     complete (synchronised) when it returns.
 */
#ifndef PIAFS_GPU_H
#define PIAFS_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PIAFS_OK = 0,
  PIAFS_ERR_ARGUMENT = 1,     /* bad argument or call sequence            */
  PIAFS_ERR_INPUT = 2,        /* missing or malformed input deck          */
  PIAFS_ERR_UNSUPPORTED = 3,  /* option outside the GPU path              */
  PIAFS_ERR_CUDA = 4,         /* CUDA runtime failure                     */
  PIAFS_ERR_SINGULAR = 5,     /* zero pivot in a tridiagonal solve        */
  PIAFS_ERR_IO = 6,           /* output file could not be written         */
  PIAFS_ERR_MEMORY = 7        /* device allocation failed                 */
};

enum { PIAFS_PRECISION_FP64 = 0, PIAFS_PRECISION_MIXED = 1 };

typedef struct piafs_gpu_sim piafs_gpu_sim;

typedef struct {
  int ndims, nvars, ghosts;
  int dim[2];                 /* interior points per dimension (dim[1] = 1 in 1D) */
  int n_iter, restart_iter, screen_op_iter, file_op_iter;
  int iter;                   /* completed time steps                     */
  int nstages;
  double dt, t;               /* time step, current simulation time        */
  double gamma, Re, Pr;       /* values in effect (chemistry may override) */
  long long npoints_ghosted;  /* points of a ghosted array                 */
  long long ninterfaces[2];   /* points of an interface array per dir      */
  double cfl, norm;           /* last diagnostics (TimePreStep/PostStep)   */
  int singular;               /* zero pivots seen since creation           */
  int launches_per_step;      /* kernels one time step launches            */
} piafs_gpu_info;

/* Message of the last failure on this thread ("" if none). */
const char* piafs_gpu_last_error(void);

/* Set up a simulation from the input deck in `deck_dir` and upload it to the
 * current CUDA device.  Replaces the reference's ReadInputs, Initialize,
 * InitialSolution, InitializeBoundaries, InitializeSolvers and
 * InitializePhysics (src/main.cpp:126-212).  `precision` is one of
 * PIAFS_PRECISION_*: FP64 throughout, or MIXED -- FP32 reconstruction
 * weights and rows, upwind fluxes, viscous stencils and chemistry source on
 * the FP64 conserved state, FP64 RK stage accumulation and FP64 tridiagonal
 * solves.  In the mixed path the time step, RHSFunction, HyperbolicFunction,
 * ParabolicFunction and SourceFunction use the mixed kernels; the lower-level
 * operator entry points (FFunction, InterpolateInterfacesHyp, Upwind,
 * FirstDerivativePar) stay FP64. */
int piafs_gpu_create(const char* deck_dir, int precision, piafs_gpu_sim** sim);
void piafs_gpu_destroy(piafs_gpu_sim* sim);
int piafs_gpu_get_info(piafs_gpu_sim* sim, piafs_gpu_info* info);

/* State transfer with host arrays in the reference layout (ghosts included).
 * set_state also sets the simulation time. */
int piafs_gpu_set_state(piafs_gpu_sim* sim, const double* u_host, double t);
int piafs_gpu_get_state(piafs_gpu_sim* sim, double* u_host);
/* Interior points only, in output-file order (npoints x nvars). */
int piafs_gpu_get_solution(piafs_gpu_sim* sim, double* u_interior_host);

/* Advance the device-resident state by `nsteps` time steps: per step the
 * boundary conditions on u (TimePreStep.c:36-41), the explicit RK stages
 * (TimeRK.c:34-102) and t += dt (TimePostStep.c:31).  Replaces
 * TS->TimeIntegrate = TimeRK (src/TimeIntegration/TimeRK.c:34). */
int piafs_gpu_TimeRK(piafs_gpu_sim* sim, int nsteps);

/* One time step on a host array, the drop-in form of TimeIntegrate when the
 * caller owns solver->u: copies u_host (ghosted, reference layout) to the
 * device, advances one step from time t and copies the result back. */
int piafs_gpu_TimeRK_host(piafs_gpu_sim* sim, double* u_host, double t);

/* The reference's Solve() loop (src/Simulation/Solve.cpp:29-123): n_iter
 * steps from the initial solution with op_NNNNN.bin written to `output_dir`
 * at iteration 0, every file_op_iter steps and at the end (binary output
 * format only); every screen_op_iter-th step prints the reference's
 * TimePrintStep line (iteration, time, CFL before the step, residual norm,
 * wall time; TimePrintStep.c:25-37) on stdout. */
int piafs_gpu_Solve(piafs_gpu_sim* sim, const char* output_dir);

/* piafs_gpu_TimeRK that also returns the residual norm of the last step,
 * sqrt(sum over interior points and variables of (u_new - u_old)^2 / points)
 * (TimePostStep.c:36-54). */
int piafs_gpu_TimeRK_norm(piafs_gpu_sim* sim, int nsteps, double* norm);

/* After a Solve: the reference's end-of-run files in `dir`, as SimWriteErrors
 * writes them for one simulation (SimulationWriteErrors.c:65-80) --
 * errors.dat (grid, processes, dt, the L1 / L2 / Linf errors against
 * exact.inp when `dir` holds one (CalculateError.c:30-120), else -1, and the
 * two runtimes), conservation.dat (-1 per variable: conservation_check is
 * not on the GPU path) and function_counts.dat -- and the runtime lines it
 * prints. */
int piafs_gpu_WriteErrors(piafs_gpu_sim* sim, const char* dir, double solver_runtime, double main_runtime);

/* Asynchronous form of piafs_gpu_TimeRK: enqueues nsteps steps on the
 * simulation's CUDA stream and returns without waiting (diagnostics and the
 * singular-pivot count are updated at the next synchronising call). */
int piafs_gpu_TimeRK_async(piafs_gpu_sim* sim, int nsteps);
/* The simulation's CUDA stream (a cudaStream_t), for callers that order
 * their own work or timing events after it. */
int piafs_gpu_get_stream(piafs_gpu_sim* sim, void** stream);
int piafs_gpu_synchronize(piafs_gpu_sim* sim);

/* Time each kernel phase of one right-hand-side evaluation on the current
 * state with CUDA events on the simulation's stream, averaged over `reps`
 * evaluations.  ms[k] receives the mean duration of phase k; phases are, per
 * direction d = 0..ndims-1, [2d] flux (with the transpose of a transposed
 * y pass), [2d+1] interface reconstruction (WENO5 or the CRWENO5 line
 * solve), then [2 ndims] upwinding + divergence of all directions and
 * [2 ndims + 1] viscous + source.  nphases (in/out) is the capacity / count. */
int piafs_gpu_profile_rhs(piafs_gpu_sim* sim, int reps, double* ms, int* nphases);

/* Photon density of the last RK stage evaluated (the reference's
 * Chemistry::nv_hnu, ChemistrySolve.c:46-58, as the species output writes it):
 * into nv_hnu[nz * p + iz] for every ghosted point p and simulated layer iz.
 * Only simulations that write species files keep it. */
int piafs_gpu_get_photon_density(piafs_gpu_sim* sim, double* nv_hnu);

/* max CFL of the current state (NavierStokes2DComputeCFL.c /
 * Euler1DComputeCFL.c). */
int piafs_gpu_ComputeCFL(piafs_gpu_sim* sim, double* cfl);

/* ---- operator-level entry points (device pointers, reference layout) ----
 * These mirror the HyPar function pointers one to one and exist so that each
 * operator can be checked on its own.  Time-dependent operators take t. */

/* TS->RHSFunction = TimeRHSFunctionExplicit (TimeRHSFunctionExplicit.c:29);
 * fills the ghosts of u (boundary conditions) like the reference does. */
int piafs_gpu_RHSFunction(piafs_gpu_sim* sim, double* rhs, double* u, double t);
/* solver->HyperbolicFunction (HyperbolicFunction.c:34) */
int piafs_gpu_HyperbolicFunction(piafs_gpu_sim* sim, double* hyp, const double* u, double t);
/* solver->ParabolicFunction = NavierStokes2DParabolicFunction (:41) */
int piafs_gpu_ParabolicFunction(piafs_gpu_sim* sim, double* par, const double* u, double t);
/* solver->SourceFunction (SourceFunction.c:21) */
int piafs_gpu_SourceFunction(piafs_gpu_sim* sim, double* source, const double* u, double t);
/* solver->ApplyBoundaryConditions (ApplyBoundaryConditions.c:31) */
int piafs_gpu_ApplyBoundaryConditions(piafs_gpu_sim* sim, double* u, double t);
/* solver->FFunction (NavierStokes2DFlux.c:24 / Euler1DFlux.c:19) */
int piafs_gpu_FFunction(piafs_gpu_sim* sim, double* f, const double* u, int dir, double t);
/* solver->SetInterpLimiterVar + solver->InterpolateInterfacesHyp
 * (WENOFifthOrderCalculateWeights.c:41 + Interp1PrimFifthOrderWENO.c:77 /
 * Interp1PrimFifthOrderCRWENO.c:81): the interface values of fC (uflag = 0)
 * or of u (uflag = 1), left-biased for upw > 0, right-biased for upw < 0. */
int piafs_gpu_InterpolateInterfacesHyp(piafs_gpu_sim* sim, double* fI, const double* fC, const double* u,
                                       int upw, int dir, int uflag);
/* solver->Upwind (NavierStokes2DUpwind.c / Euler1DUpwind.c) */
int piafs_gpu_Upwind(piafs_gpu_sim* sim, double* fI, const double* fL, const double* fR, const double* uL,
                     const double* uR, const double* u, int dir, double t);
/* solver->FirstDerivativePar = FirstDerivativeFirstOrder
 * (FirstDerivativeFirstOrder.c:40) on an array with `nv` values per point */
int piafs_gpu_FirstDerivativePar(piafs_gpu_sim* sim, double* Df, const double* f, int dir, int bias, int nv);
/* tridiagLU (tridiagLU.c:86), serial semantics: ns independent systems of n
 * rows, layout [row * ns + system], solved in place into x.  Returns
 * PIAFS_ERR_SINGULAR on a zero pivot like the reference's -1. */
int piafs_gpu_tridiagLU(double* a, double* b, double* c, double* x, int n, int ns);

/* ---- batched simulations (ensembles and request serving) ----
 * No counterpart in the reference, whose ensemble mode (OutputSolution.cpp,
 * one deck per member) runs members one after another.  A batch holds many
 * independent simulations ("members") resident on the device at once, each
 * from its own input deck and of its own size, physics and step count, and
 * advances all of them together: one persistent kernel per Runge-Kutta
 * stage walks a device-side list of tiles that covers every member, and a
 * step (the stage kernels plus a small per-step epilogue) is replayed from a
 * CUDA graph whatever the mix of members.  Members join and leave between
 * steps (continuous batching).  Supported members: 2D navierstokes2d with or
 * without photochemistry and viscosity, and 1D euler1d without chemistry,
 * WENO5 (any weight variant), any upwinding, any explicit RK tableau,
 * periodic / extrapolate / slip-wall boundaries.  In FP64 a member's result
 * agrees with the same deck run alone through piafs_gpu_TimeRK to rounding
 * (relative L2 within 1e-12), and is bit for bit the same whatever other
 * members share the batch and whenever they join or leave. */
typedef struct piafs_gpu_batch piafs_gpu_batch;
typedef struct {
  int members;                      /* admitted and not yet removed       */
  int active;                       /* still stepping                     */
  int tiles;                        /* tiles in the current launch list   */
  int tile_x, tile_y;               /* tile shape of the 2D stage kernel  */
  long long steps;                  /* batch steps taken                  */
  unsigned long long bytes_in_use;  /* member state held on the device    */
  unsigned long long budget_bytes;  /* 0: no limit                        */
  int launches_per_step;            /* kernels one batch step launches    */
  int min_ctas_per_sm;              /* occupancy the stage kernel is built for */
} piafs_gpu_batch_info;
/* hbm_budget_bytes bounds the device memory the members' state may take
 * (0: no bound); precision is PIAFS_PRECISION_*. */
int piafs_gpu_batch_create(int precision, unsigned long long hbm_budget_bytes, piafs_gpu_batch** batch);
void piafs_gpu_batch_destroy(piafs_gpu_batch* batch);
/* Admit the simulation of the input deck in deck_dir, to run nsteps time
 * steps (<= 0: the deck's n_iter).  On success *id names the member.  Returns
 * PIAFS_ERR_MEMORY, with nothing changed, when the budget cannot hold it now,
 * and PIAFS_ERR_UNSUPPORTED for decks outside the batched path. */
int piafs_gpu_batch_add(piafs_gpu_batch* batch, const char* deck_dir, int nsteps, int* id);
/* piafs_gpu_batch_add for n decks, parsed in parallel by host threads and
 * admitted in order; nsteps may be NULL (every deck's n_iter).  Stops at the
 * first failure; *n_added members were admitted, their ids in ids[]. */
int piafs_gpu_batch_add_many(piafs_gpu_batch* batch, const char* const* deck_dirs, int n, const int* nsteps,
                             int* ids, int* n_added);
/* Advance every active member by up to nsteps steps; a member stops after
 * its own step count.  Waits for the device. */
int piafs_gpu_batch_step(piafs_gpu_batch* batch, int nsteps);
/* Up to cap ids of members that finished since the last call, count in *n. */
int piafs_gpu_batch_poll(piafs_gpu_batch* batch, int* done, int cap, int* n);
/* A member's solution (interior points, the layout of the op files) and its
 * time and step count. */
int piafs_gpu_batch_get_solution(piafs_gpu_batch* batch, int id, double* u_interior);
int piafs_gpu_batch_member(piafs_gpu_batch* batch, int id, double* t, int* iter, int* done);
/* The stage derivative k_stage (TimeRHSFunctionExplicit's rhs) of the
 * member's last step, interior points in the layout of the op files. */
int piafs_gpu_batch_get_stage_derivative(piafs_gpu_batch* batch, int id, int stage, double* k_interior);
/* A member's state buffers with ghosts, reference layout: which = 0 the
 * solution, 1 and 2 the two stage-state buffers of its last step. */
int piafs_gpu_batch_get_buffer(piafs_gpu_batch* batch, int id, int which, double* u_ghosted);
/* Release a member's device memory (finished or not). */
int piafs_gpu_batch_remove(piafs_gpu_batch* batch, int id);
int piafs_gpu_batch_get_info(piafs_gpu_batch* batch, piafs_gpu_batch_info* info);
/* Autotuner: with force_tile_x = 0, time every launch configuration of the
 * stage kernel (2D tile 32x8, 16x16 or 64x4, each compiled for one or two
 * CTAs per SM) on the current members -- one warm-up and two timed steps
 * each, the members' state saved before and restored after every trial --
 * and keep the fastest; info.tile_x / tile_y / min_ctas_per_sm report it.
 * A nonzero force_tile_x selects that tile width (one CTA per SM) instead. */
int piafs_gpu_batch_tune(piafs_gpu_batch* batch, int force_tile_x);
/* Select a launch configuration directly, e.g. one an earlier tune chose for
 * the same class of members (tile_x x tile_y = 32x8, 16x16 or 64x4;
 * min_ctas_per_sm 1 or 2). */
int piafs_gpu_batch_set_launch(piafs_gpu_batch* batch, int tile_x, int tile_y, int min_ctas_per_sm);

/* ---- request serving ----
 * No counterpart in the reference.  A request is a solve described by its
 * parameters instead of an input deck on disk: the library writes the deck
 * in memory (the decks of the package's case generators, cases.py) and
 * generates the initial fields on the device, so a stream of requests needs
 * no file traffic.  Kinds: the 1D Euler density wave (rho = 1 + amp
 * sin(2 pi x), u = 1, p = 1, gamma 1.4, periodic, WENO5, Roe, SSPRK3) and the
 * 2D photochemical beam (quiescent O2/O3 gas, density noise of amplitude
 * `noise` from `seed`, Gaussian beam map of amplitude `amp` and 1/e radius
 * `beam_radius`, Re through the beam half-angle, periodic x, slip walls y,
 * WENO5, LLF, SSPRK3). */
enum { PIAFS_REQUEST_EULER1D_WAVE = 1, PIAFS_REQUEST_NS2D_BEAM = 2 };
typedef struct {
  int kind;                 /* PIAFS_REQUEST_*                                */
  int n;                    /* grid points (1D) or grid side (2D, square)     */
  int nsteps;               /* time steps                                     */
  double dt;                /* time step                                      */
  double amp;               /* density-wave (1D) or beam (2D) amplitude       */
  double beam_radius;       /* 2D                                             */
  double Re;                /* 2D                                             */
  double noise;             /* 2D                                             */
  unsigned long long seed;  /* 2D                                             */
} piafs_gpu_request;
int piafs_gpu_batch_add_request(piafs_gpu_batch* batch, const piafs_gpu_request* req, int* id);
/* Sum of a member's solution over interior points and variables, reduced on
 * the device in a fixed order (the same bits every time for the same state). */
int piafs_gpu_batch_checksum(piafs_gpu_batch* batch, int id, double* sum);
typedef struct {
  double arrival_s;         /* from the trace                                 */
  double admitted_s;        /* admission time, seconds from the trace start   */
  double finished_s;        /* result ready (retired), seconds from the start */
  int steps;
  double checksum;          /* piafs_gpu_batch_checksum of the final state    */
} piafs_gpu_serve_result;
/* Replay a request trace in real time with continuous batching: request k
 * arrives at arrival_s[k] (seconds from the start, nondecreasing); arrived
 * requests are admitted in arrival order while the HBM budget holds them and
 * the resident grid points stay within max_resident_points (0: no bound; a
 * request is always admitted when nothing is resident); a request that does
 * not fit waits, and so do the ones behind it.  Between admission rounds all
 * resident requests advance steps_per_round steps together; a finished
 * request's checksum is taken and its memory released at once.  The points
 * bound trades concurrency for latency: every resident request shares the
 * device, so admitting fewer at a time lets each finish sooner once started.
 * Returns when every request has finished; latency of request k is
 * out[k].finished_s - out[k].arrival_s. */
int piafs_gpu_serve_trace(const piafs_gpu_request* reqs, const double* arrival_s, int n, int precision,
                          unsigned long long hbm_budget_bytes, unsigned long long max_resident_points,
                          int steps_per_round, piafs_gpu_serve_result* out);

/* ---- a 2D grid decomposed along y, one GPU per row slab ----
 * Replaces the reference's MPI decomposition of one grid
 * (MPIExchangeBoundariesnD.c:45-177, the MPI-parallel tridiagLU.c:16-85,
 * 155-240).  Rank r of nranks owns rows [r n1, (r+1) n1) of the grid (its row
 * slab: a piafs_gpu_sim of its own, whose x lines are whole) and, for the y
 * direction, columns [r n0, (r+1) n0) over every row (its column slab), so
 * that each y line is solved whole on one GPU; n1 = N1 / nranks and
 * n0 = N0 / nranks must be whole numbers.  The caller moves the data between
 * the slabs at three points of every RK stage (piafs_b200/slab.py does it
 * with all-to-all collectives):
 *   piafs_gpu_slab_stage_begin(st)      U_st, boundary zones, x pass
 *   halo: rows [0, g) and [n1-g, n1) of U_st to the neighbouring row slabs'
 *         ghost rows (wrapping around when periodic_y)
 *   columns: rows [-g, n1+g) of U_st, columns of slab c, to column slab c,
 *         transposed (the column state `utc`, [var][col + g][row + g],
 *         plane stride col_plane_stride; the first slab's lower and the last
 *         slab's upper ghost rows included)
 *   piafs_gpu_slab_y_pass(st)           y pass on the column slab -> hy_send
 *   hy: block r of hy_send ([var][n1][n0] values of hy_value_bytes) to row
 *         slab r, which stores block c (from column slab c) at block c of
 *         its hy_recv
 *   piafs_gpu_slab_stage_end(st)        x upwinding, divergence, viscous
 *                                       terms and source
 * and after the last stage piafs_gpu_slab_step_end.  The result equals the
 * undecomposed simulation's bit for bit.  2D decks without sponge zones,
 * characteristic interpolation or par_space_scheme 4, whose x-face boundary
 * zones span every row; FP64, or mixed precision with CRWENO5.  The row
 * slab's piafs_gpu_sim (piafs_gpu_slab_sim) gives its state, solution, CFL
 * and stream; every call runs on that stream. */
typedef struct piafs_gpu_slab piafs_gpu_slab;
typedef struct {
  int rank, nranks;
  int dim[2];                  /* the whole grid's interior points          */
  int slab_rows, slab_cols;    /* n1, n0                                    */
  int ghosts, nvars, nstages;
  int periodic_y;              /* ghost rows wrap around the last slab      */
  long long plane_stride;      /* row slab state: [var][row + g][col + g]   */
  long long col_plane_stride;  /* column slab state: [var][col + g][row + g] */
  long long hy_bytes;          /* size of hy_send and of hy_recv            */
  int hy_value_bytes;          /* 8 (FP64) or 4 (mixed precision)           */
} piafs_gpu_slab_info;
int piafs_gpu_slab_create(const char* deck_dir, int precision, int rank, int nranks, piafs_gpu_slab** slab);
void piafs_gpu_slab_destroy(piafs_gpu_slab* slab);
int piafs_gpu_slab_get_info(piafs_gpu_slab* slab, piafs_gpu_slab_info* info);
int piafs_gpu_slab_sim(piafs_gpu_slab* slab, piafs_gpu_sim** row_slab);
/* device pointers: U of stage st (row slab), the column state, the y-term buffers */
int piafs_gpu_slab_state(piafs_gpu_slab* slab, int stage, double** U);
int piafs_gpu_slab_buffers(piafs_gpu_slab* slab, double** utc, void** hy_send, void** hy_recv);
int piafs_gpu_slab_stage_begin(piafs_gpu_slab* slab, int stage);
int piafs_gpu_slab_y_pass(piafs_gpu_slab* slab, int stage);
int piafs_gpu_slab_stage_end(piafs_gpu_slab* slab, int stage);
/* TimeRK's completion of the step; with_norm: sum of the squared change of
 * u over the slab's points, read by piafs_gpu_slab_norm_sum (which
 * synchronises the stream) */
int piafs_gpu_slab_step_end(piafs_gpu_slab* slab, int with_norm);
int piafs_gpu_slab_norm_sum(piafs_gpu_slab* slab, double* sum);

/* ---- diagnostics ----
 * No counterpart in the reference.  y[i] = 1/x[i] (device arrays) computed
 * by the Newton-Raphson reciprocal that the reconstruction and line-solve
 * kernels use in place of a division, so that callers can check its
 * accuracy against 1/x; for finite x whose reciprocal is a normal number. */
int piafs_gpu_reciprocal(const double* x, double* y, long long n);

/* ---- allocation-free hyperbolic term ----
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they need the hyperbolic term: a plugin inside an application
 * whose memory manager owns the whole device and forbids allocations behind
 * its back, or a host loop that must not pay cudaMalloc's implicit device
 * synchronisation or risk an out-of-memory failure in the middle of a run.
 * It computes what piafs_gpu_HyperbolicFunction computes (component-wise
 * WENO5, CRWENO5 or upw5 interpolation; characteristic interpolation is not
 * available through piafs_gpu_hyp_params), from the caller's u (ghosted,
 * ghosts filled, reference layout) and dxinv (ghosted 1/dx of each
 * dimension, concatenated), into the caller's hyp, with no simulation object
 * and no device allocation.  Its working arrays live in one 64 MiB
 * __device__ array that every GPU loading this library holds until exit;
 * problems whose working set (about 7 x nvars x ghosted points x 8 bytes)
 * exceeds it are rejected with PIAFS_ERR_ARGUMENT.  The first call on a
 * device looks up that array's address with the device current (make it
 * before any stream capture begins); all calls on a device share the array,
 * so calls that overlap on the GPU race and must be serialised by the
 * caller.  The call runs on `stream` (a cudaStream_t, 0 for the default
 * stream), then copies the zero-pivot flag to the host and synchronises that
 * stream before it returns. */
enum { PIAFS_MODEL_EULER1D = 0, PIAFS_MODEL_NS2D = 1 };
enum { PIAFS_SCHEME_WENO5 = 0, PIAFS_SCHEME_CRWENO5 = 1, PIAFS_SCHEME_UPW5 = 2 };
enum { PIAFS_UPWIND_ROE = 0, PIAFS_UPWIND_RF = 1, PIAFS_UPWIND_LLF = 2, PIAFS_UPWIND_RUSANOV = 3 };
enum { PIAFS_WENO_JS = 0, PIAFS_WENO_MAPPED = 1, PIAFS_WENO_BORGES = 2, PIAFS_WENO_YC = 3 };
typedef struct {
  int ndims, nvars, ghosts;
  int dim[2];          /* interior points per dimension */
  int model;           /* PIAFS_MODEL_*   */
  int scheme;          /* PIAFS_SCHEME_*  */
  int upwind;          /* PIAFS_UPWIND_*  */
  int weno_type;       /* PIAFS_WENO_*    */
  int no_limiting;     /* weno.inp no_limiting */
  double weno_eps;     /* weno.inp epsilon     */
  double gamma;        /* ratio of specific heats in effect */
} piafs_gpu_hyp_params;
int piafs_gpu_HyperbolicFunction_noalloc(const piafs_gpu_hyp_params* p, double* hyp, const double* u,
                                         const double* dxinv, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PIAFS_GPU_H */
