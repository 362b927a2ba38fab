/* CPU restatement of the PIAFS per-stage RHS + explicit RK path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle: the test suite, the
 * smoke check and the CPU-baseline leg of the benchmark call it to check the
 * GPU path.  No product code links it.
 *
 * Layout is the reference's: array-of-structures, variable index fastest,
 * then dim0, dim1, ghost points included (include/arrayfunctions.h:43-50).
 * Interface arrays carry no ghosts and have dim_d+1 entries along the
 * reconstruction direction (src/Simulation/Initialize.c:165-174).
 */
#ifndef PIAFS_ORACLE_H
#define PIAFS_ORACLE_H

#define ORC_MAX_ZONES 16

enum { ORC_EULER1D = 0, ORC_NS2D = 1 };
enum { ORC_WENO5 = 0, ORC_CRWENO5 = 1 };
enum { ORC_ROE = 0, ORC_RF = 1, ORC_LLF = 2, ORC_RUSANOV = 3 };
enum { ORC_W_JS = 0, ORC_W_MAPPED = 1, ORC_W_BORGES = 2, ORC_W_YC = 3 };
enum { ORC_BC_PERIODIC = 0, ORC_BC_EXTRAPOLATE = 1, ORC_BC_SLIPWALL = 2 };

typedef struct {
  /* grid */
  int ndims, nvars, ghosts;
  int dim[2];
  /* schemes */
  int model, scheme, upwind, weno_type, no_limiting;
  double weno_eps;
  /* physics */
  double gamma, Re, Pr, Tref, T0, TS, TA, TB;
  /* gamma seen by the wall boundary conditions: the physics.inp value, set
   * before chemistry overrides the flow gamma (NavierStokes2DInitialize.c:172-174
   * precede :196-200) */
  double bc_gamma;
  int viscous;                 /* NS2D with Re > 0 */
  /* chemistry (normalised quantities, ChemistryInitialize.c:267-353) */
  int include_chem;
  int n_flow_vars, nz, z_stride, grid_stride;
  double k[11];                /* k0a k0b k1a k1b k2a k2b k3a k3b k4 k5 k6 (normalised) */
  double q[11];                /* q0a ... q6 (normalised) */
  double chem_gamma, I0, c, h, nu, n_O2, t_start_norm, t_pulse_norm, sO3, dz;
  /* time integration (Butcher tableau) */
  int nstages;
  double A[16], b[4], cst[4];
  double dt;
  /* boundary zones (single rank: is/ie already resolved) */
  int nb;
  int bc_type[ORC_MAX_ZONES], bc_dim[ORC_MAX_ZONES], bc_face[ORC_MAX_ZONES];
  int bc_is[ORC_MAX_ZONES][2], bc_ie[ORC_MAX_ZONES][2];
  double bc_vel[ORC_MAX_ZONES][2];
} orc_params;

#ifdef __cplusplus
extern "C" {
#endif

/* sizes */
long orc_npoints_ghosted(const orc_params* P);
long orc_ninterfaces(const orc_params* P, int dir);

/* ghost fills (ApplyBoundaryConditions) */
int orc_apply_bc(const orc_params* P, double* u);
/* cell-centred flux at every point including ghosts (FFunction) */
int orc_flux(const orc_params* P, double* f, const double* u, int dir);
/* interface reconstruction for one (upw, uflag) combination, weights included
 * (SetInterpLimiterVar + InterpolateInterfacesHyp) */
int orc_interp(const orc_params* P, double* fI, const double* fC, const double* u,
               int upw, int dir, int uflag);
/* upwinding (Upwind) */
int orc_upwind(const orc_params* P, double* fI, const double* fL, const double* fR,
               const double* uL, const double* uR, const double* u, int dir);
/* hyperbolic term (HyperbolicFunction) */
int orc_hyperbolic(const orc_params* P, double* hyp, const double* u, const double* dxinv);
/* viscous term (NavierStokes2DParabolicFunction) */
int orc_parabolic(const orc_params* P, double* par, const double* u, const double* dxinv);
/* first-order one-sided differences (FirstDerivativeFirstOrder) */
int orc_first_derivative(const orc_params* P, double* Df, const double* f, int dir, int bias, int nv);
/* source term (SourceFunction -> ChemistrySource) */
int orc_source(const orc_params* P, double* src, const double* u, const double* imap, double t);
/* full RHS (TimeRHSFunctionExplicit); u gets its ghosts filled */
int orc_rhs(const orc_params* P, double* rhs, double* u, const double* dxinv,
            const double* imap, double t);
/* batched serial Thomas solve, layout [row*ns + sys] (tridiagLU serial path) */
int orc_tridiag(double* a, double* b, double* c, double* x, int n, int ns);
/* nsteps explicit RK steps (TimePreStep BC + TimeRK), t advanced by dt each */
int orc_run(const orc_params* P, double* u, const double* dxinv, const double* imap,
            double t0, int nsteps);
/* max CFL over the interior (ComputeCFL) */
double orc_cfl(const orc_params* P, const double* u, const double* dxinv);

#ifdef __cplusplus
}
#endif
#endif
