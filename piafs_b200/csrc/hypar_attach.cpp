// The GPU path attached to the reference's own simulation objects
// (include/piafs_hypar.h).  Host code only, compiled against the reference's
// include/ with -Dserial so that HyPar, SimulationObject, TimeIntegration,
// DomainBoundary, WENOParameters, the physics objects and Chemistry have the
// layout of the single-rank reference build they come from.
//
// A simulation is mirrored by filling the same Deck that read_deck fills
// from the input files (deck.h), here from the reference's initialised
// objects: sizes and options from HyPar (include/hypar.h:25-333), the RK
// tableau from ExplicitRKParameters (TimeExplicitRKInitialize.c:72-82), the
// WENO options from WENOParameters (WENOInitialize.c), gamma / Re / Pr /
// upwinding / Sutherland constants from the physics object (after the
// chemistry overrides of NavierStokes2DInitialize.c:196-217), the normalised
// photochemical constants, beam map and layer index from Chemistry
// (ChemistryInitialize.c:267-476), the boundary zones with their index
// ranges and data from DomainBoundary (InitializeBoundaries.c:82-378), and
// the ghosted grid, 1/dx and solution from HyPar::x, dxinv and u.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/piafs_gpu.h"
#include "../../include/piafs_hypar.h"
#include "deck.h"

// The reference's structures.  Included after every header of this library:
// the reference's math_ops.h defines function-like min / max macros.
extern "C" {
#include <boundaryconditions.h>
#include <hypar.h>
#include <interpolation.h>
#include <mpivars_struct.h>
#include <physicalmodels/chemistry.h>
#include <physicalmodels/euler1d.h>
#include <physicalmodels/navierstokes2d.h>
#include <simulation_object.h>
#include <timeintegration_struct.h>
}

namespace piafs {
int set_last_error(int code, const std::string& msg);   // api.cu: piafs_gpu_last_error()
}

namespace {

using piafs::Deck;

// an attached simulation: the device simulation and device staging for the
// host-array operator calls (six arrays of the larger of a ghosted and an
// interface array)
struct Attached {
  piafs_gpu_sim* gpu = nullptr;
  double* stage[6] = {nullptr};
  size_t elems = 0;
  long long npg = 0, nint[2] = {0, 0};
  int nvars = 0;
  Chemistry* chem = nullptr;
  bool species = false;
  bool par_counted = false, sou_counted = false;   // which call counters a stage advances
};

std::mutex g_mu;
std::map<const void*, Attached> g_att;   // keyed by HyPar*

int fail(int code, const std::string& msg) {
  std::fprintf(stderr, "piafs_gpu (HyPar): %s\n", msg.c_str());
  return piafs::set_last_error(code, msg);
}

int report(int code) {
  if (code) std::fprintf(stderr, "piafs_gpu (HyPar): %s\n", piafs_gpu_last_error());
  return code;
}

int zone_type(const std::string& t, int& type) {
  static const std::map<std::string, int> types = {
      {"periodic", piafs::BC_PERIODIC}, {"extrapolate", piafs::BC_EXTRAPOLATE},
      {"dirichlet", piafs::BC_DIRICHLET}, {"reflect", piafs::BC_REFLECT},
      {"slip-wall", piafs::BC_SLIPWALL}, {"noslip-wall", piafs::BC_NOSLIP},
      {"subsonic-inflow", piafs::BC_SUB_INFLOW}, {"subsonic-outflow", piafs::BC_SUB_OUTFLOW},
      {"subsonic-ambivalent", piafs::BC_SUB_AMBIVALENT}, {"supersonic-inflow", piafs::BC_SUP_INFLOW},
      {"supersonic-outflow", piafs::BC_SUP_OUTFLOW}};
  auto it = types.find(t);
  if (it == types.end()) return -1;
  type = it->second;
  return 0;
}

// Deck from an initialised single-rank simulation object
int deck_from_hypar(SimulationObject* so, Deck& d, std::string& err) {
  HyPar* h = &so->solver;
  MPIVariables* mpi = &so->mpi;
  d = Deck();
  d.ndims = h->ndims;
  d.nvars = h->nvars;
  d.ghosts = h->ghosts;
  if (d.ndims < 1 || d.ndims > 2) { err = "ndims must be 1 or 2"; return PIAFS_ERR_UNSUPPORTED; }
  for (int k = 0; k < d.ndims; k++) {
    if (mpi->iproc && mpi->iproc[k] != 1) {
      err = "one MPI rank per simulation: the GPU holds the whole grid";
      return PIAFS_ERR_UNSUPPORTED;
    }
    d.size.push_back(h->dim_local[k]);
  }
  d.n_iter = h->n_iter;
  d.restart_iter = h->restart_iter;
  d.screen_op_iter = h->screen_op_iter;
  d.file_op_iter = h->file_op_iter;
  d.dt = h->dt;
  d.time_scheme = h->time_scheme;
  d.time_scheme_type = h->time_scheme_type;
  d.hyp_space_scheme = h->spatial_scheme_hyp;
  d.hyp_interp_type = h->interp_type;
  d.par_space_scheme = h->spatial_scheme_par;
  d.ip_file_type = h->ip_file_type;
  d.op_file_format = h->op_file_format;
  d.op_overwrite = h->op_overwrite;
  d.model = h->model;
  d.input_mode = h->input_mode;
  d.output_mode = h->output_mode;
  d.conservation_check = h->ConservationCheck;

  // the RK tableau the reference set up (row-major A of nstages x nstages)
  if (d.time_scheme == "rk") {
    const ExplicitRKParameters* p = (const ExplicitRKParameters*)h->msti;
    if (!p || p->nstages < 1 || p->nstages > piafs::MAX_STAGES) {
      err = "RK tableau missing or with more stages than the GPU path holds";
      return PIAFS_ERR_UNSUPPORTED;
    }
    d.nstages = p->nstages;
    for (int i = 0; i < p->nstages; i++) {
      for (int j = 0; j < p->nstages; j++) d.A[i * piafs::MAX_STAGES + j] = p->A[i * p->nstages + j];
      d.b[i] = p->b[i];
      d.c[i] = p->c[i];
    }
  } else if (d.time_scheme == "euler") {
    d.nstages = 1;
    d.b[0] = 1.0;
  } else {
    err = "time_scheme " + d.time_scheme + " is not supported";
    return PIAFS_ERR_UNSUPPORTED;
  }

  // WENO-family options (WENOInitialize.c; upw5 has none)
  if (const WENOParameters* w = (const WENOParameters*)h->interp) {
    if (d.hyp_space_scheme == "weno5" || d.hyp_space_scheme == "crweno5") {
      d.mapped = w->mapped;
      d.borges = w->borges;
      d.yc = w->yc;
      d.no_limiting = w->no_limiting;
      d.weno_eps = w->eps;
    }
  }

  // physics object (values in effect: chemistry has replaced gamma, Re, Pr)
  Chemistry* chem = nullptr;
  if (d.model == "navierstokes2d") {
    const NavierStokes2D* ph = (const NavierStokes2D*)h->physics;
    if (!ph) { err = "navierstokes2d physics object missing"; return PIAFS_ERR_INPUT; }
    d.gamma = ph->gamma;
    d.upwinding = ph->upw_choice;
    d.Re = ph->Re;
    d.Pr = ph->Pr;
    d.Tref = ph->Tref; d.T0 = ph->T0; d.TS = ph->TS; d.TA = ph->TA; d.TB = ph->TB;
    d.write_output = ph->write_op;
    d.include_chem = ph->include_chem ? "yes" : "no";
    if (ph->include_chem) chem = (Chemistry*)ph->chem;
  } else if (d.model == "euler1d") {
    const Euler1D* ph = (const Euler1D*)h->physics;
    if (!ph) { err = "euler1d physics object missing"; return PIAFS_ERR_INPUT; }
    d.gamma = ph->gamma;
    d.upwinding = ph->upw_choice;
    d.include_chem = ph->include_chem ? "yes" : "no";
    if (ph->include_chem) chem = (Chemistry*)ph->chem;
  } else {
    err = "model " + d.model + " is not on the GPU path (euler1d, navierstokes2d)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  // the boundary objects carry the gamma the walls use (the physics.inp
  // value for NS2D, zero for Euler1D, which never sets it)
  const DomainBoundary* B = (const DomainBoundary*)h->boundary;
  d.bc_gamma = (B && h->nBoundaryZones > 0) ? B[0].gamma : (d.model == "navierstokes2d" ? d.gamma : 0.0);

  if (chem) {
    d.chem = true;
    const double kn[11] = {chem->k0a_norm, chem->k0b_norm, chem->k1a_norm, chem->k1b_norm, chem->k2a_norm,
                           chem->k2b_norm, chem->k3a_norm, chem->k3b_norm, chem->k4_norm, chem->k5_norm,
                           chem->k6_norm};
    const double qn[11] = {chem->q0a_norm, chem->q0b_norm, chem->q1a_norm, chem->q1b_norm, chem->q2a_norm,
                           chem->q2b_norm, chem->q3a_norm, chem->q3b_norm, chem->q4_norm, chem->q5_norm,
                           chem->q6_norm};
    for (int i = 0; i < 11; i++) { d.kn[i] = kn[i]; d.qn[i] = qn[i]; }
    d.chem_gamma = chem->gamma;
    d.I0 = chem->I0;
    d.ch_c = chem->c;
    d.ch_h = chem->h;
    d.ch_nu = chem->nu;
    d.n_O2 = chem->n_O2;
    d.t_start_norm = chem->t_start_norm;
    d.t_pulse_norm = chem->t_pulse_norm;
    d.sO3 = chem->sO3;
    d.dz = chem->dz;
    d.nz = chem->z_i + 1;                  // simulated layers
    d.L_ref = chem->L_ref; d.kg = chem->kg; d.IA = chem->IA; d.IB = chem->IB; d.IC = chem->IC;
    d.write_all_zlocs = chem->write_all_zlocs;
    d.write_species = d.model == "euler1d" || d.write_output == "yes";
  }

  // grid, 1/dx (ghosted, dimensions concatenated) and the ghosted solution
  const int g = d.ghosts;
  size_t off = 0, npg = 1;
  for (int k = 0; k < d.ndims; k++) {
    const int W = d.size[k] + 2 * g;
    d.x.insert(d.x.end(), h->x + off, h->x + off + W);
    d.dxinv.insert(d.dxinv.end(), h->dxinv + off, h->dxinv + off + W);
    d.grid.insert(d.grid.end(), h->x + off + g, h->x + off + g + d.size[k]);
    off += W;
    npg *= (size_t)W;
  }
  d.u0.assign(h->u, h->u + npg * (size_t)d.nvars);
  d.imap.assign(npg, 0.0);
  if (chem && chem->imap) d.imap.assign(chem->imap, chem->imap + npg);

  // boundary zones with the index ranges the reference computed
  if (h->nBoundaryZones > piafs::MAX_ZONES) { err = "too many boundary zones"; return PIAFS_ERR_UNSUPPORTED; }
  const int nscalars = d.nvars - (2 + d.ndims);
  size_t xoff[2] = {0, d.ndims > 1 ? (size_t)d.size[0] : 0};
  for (int n = 0; B && n < h->nBoundaryZones; n++) {
    const DomainBoundary& b = B[n];
    if (!b.on_this_proc) continue;
    const std::string type = b.bctype;
    if (type == "sponge") {
      // BCSponge.c:42-73: sigma from the coordinate along dim
      piafs::SpongeZone sz{};
      sz.dim = b.dim;
      sz.face = b.face;
      for (int k = 0; k < 2; k++) {
        sz.is[k] = k < d.ndims ? b.is[k] : 0;
        sz.ie[k] = k < d.ndims ? b.ie[k] : 1;
      }
      sz.uref.assign(b.SpongeValue, b.SpongeValue + d.nvars);
      const double xs = b.xmin[b.dim], xe = b.xmax[b.dim];
      for (int q = sz.is[b.dim]; q < sz.ie[b.dim]; q++) {
        const double xq = d.grid[xoff[b.dim] + q];
        sz.sigma.push_back(b.face > 0 ? (xq - xs) / (xe - xs) : (xq - xe) / (xs - xe));
      }
      if (sz.ie[0] > sz.is[0] && sz.ie[1] > sz.is[1]) d.sponges.push_back(sz);
      continue;
    }
    piafs::Zone z{};
    if (zone_type(type, z.type)) {
      err = "boundary type " + type + " is not on the GPU path";
      return PIAFS_ERR_UNSUPPORTED;
    }
    z.dim = b.dim;
    z.face = b.face;
    for (int k = 0; k < 2; k++) {
      z.is[k] = k < d.ndims ? b.is[k] : 0;
      z.ie[k] = k < d.ndims ? b.ie[k] : 1;
    }
    if (b.FlowVelocity) for (int k = 0; k < d.ndims; k++) z.vel[k] = b.FlowVelocity[k];
    z.rho = b.FlowDensity;
    z.pres = b.FlowPressure;
    std::vector<double> vals;
    if (z.type == piafs::BC_DIRICHLET && b.DirichletValue) vals.assign(b.DirichletValue, b.DirichletValue + d.nvars);
    if ((z.type == piafs::BC_SUB_INFLOW || z.type == piafs::BC_SUP_INFLOW) && b.scalars && nscalars > 0)
      vals.assign(b.scalars, b.scalars + nscalars);
    d.zones.push_back(z);
    d.zone_vals.push_back(vals);
  }
  return piafs::check_deck(d, err);
}

bool d_viscous(const HyPar* h) {
  return std::string(h->model) == "navierstokes2d" && ((const NavierStokes2D*)h->physics)->Re > 0;
}

Attached* find(const void* solver) {
  auto it = g_att.find(solver);
  return it == g_att.end() ? nullptr : &it->second;
}

void release(Attached& a) {
  for (auto& p : a.stage) if (p) cudaFree(p);
  if (a.gpu) piafs_gpu_destroy(a.gpu);
  a = Attached();
}

// attach (or re-upload) one simulation object; caller holds g_mu
int attach_one(SimulationObject* so, int precision, double t) {
  HyPar* h = &so->solver;
  if (Attached* a = find(h)) return report(piafs_gpu_set_state(a->gpu, h->u, t));
  Deck d;
  std::string err;
  if (int r = deck_from_hypar(so, d, err)) return fail(r, err);
  const bool species = d.write_species && (d.op_file_format == "binary" || d.op_file_format == "bin");
  Chemistry* chem = nullptr;
  if (d.chem) chem = d.model == "navierstokes2d" ? (Chemistry*)((NavierStokes2D*)h->physics)->chem
                                                : (Chemistry*)((Euler1D*)h->physics)->chem;
  Attached a;
  if (int r = piafs::create_sim(std::move(d), precision, &a.gpu)) return report(r);
  piafs_gpu_info info;
  piafs_gpu_get_info(a.gpu, &info);
  a.npg = info.npoints_ghosted;
  a.nint[0] = info.ninterfaces[0];
  a.nint[1] = info.ninterfaces[1];
  a.nvars = info.nvars;
  a.chem = chem;
  a.species = species;
  // NavierStokes2DParabolicFunction counts only viscous calls (:64-65);
  // SourceFunction counts calls of a model source (SourceFunction.c:37-39)
  a.par_counted = h->ParabolicFunction && d_viscous(h);
  a.sou_counted = h->SFunction != nullptr;
  long long big = a.npg > a.nint[0] ? a.npg : a.nint[0];
  if (a.nint[1] > big) big = a.nint[1];
  a.elems = (size_t)big * a.nvars;
  for (auto& p : a.stage) {
    if (cudaMalloc(&p, a.elems * sizeof(double)) != cudaSuccess) {
      release(a);
      return fail(PIAFS_ERR_MEMORY, "device staging for the operator calls");
    }
  }
  if (int r = piafs_gpu_set_state(a.gpu, h->u, t)) { release(a); return report(r); }
  g_att[h] = a;
  return PIAFS_OK;
}

// host <-> staging copies of the operator calls
int h2d(double* dst, const double* src, size_t n) {
  if (cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(PIAFS_ERR_CUDA, "host-to-device copy of an operator argument");
  return 0;
}
int d2h(double* dst, const double* src, size_t n) {
  if (cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(PIAFS_ERR_CUDA, "device-to-host copy of an operator result");
  return 0;
}

Attached* lookup(void* s) {
  std::lock_guard<std::mutex> lk(g_mu);
  Attached* a = find(s);
  if (!a) fail(PIAFS_ERR_ARGUMENT, "this HyPar object is not attached (piafs_gpu_attach)");
  return a;
}

}  // namespace

extern "C" {

int piafs_gpu_attach(void* simobjs, int nsims, int precision, double t) {
  if (!simobjs || nsims < 1) return fail(PIAFS_ERR_ARGUMENT, "no simulation objects");
  SimulationObject* sim = (SimulationObject*)simobjs;
  std::lock_guard<std::mutex> lk(g_mu);
  for (int n = 0; n < nsims; n++)
    if (int r = attach_one(&sim[n], precision, t)) return r;
  return PIAFS_OK;
}

int piafs_gpu_detach(void* simobjs, int nsims) {
  if (!simobjs || nsims < 1) return fail(PIAFS_ERR_ARGUMENT, "no simulation objects");
  SimulationObject* sim = (SimulationObject*)simobjs;
  std::lock_guard<std::mutex> lk(g_mu);
  for (int n = 0; n < nsims; n++) {
    auto it = g_att.find(&sim[n].solver);
    if (it == g_att.end()) continue;
    release(it->second);
    g_att.erase(it);
  }
  return PIAFS_OK;
}

int piafs_gpu_hypar_sync(void* simobjs, int nsims) {
  if (!simobjs || nsims < 1) return fail(PIAFS_ERR_ARGUMENT, "no simulation objects");
  SimulationObject* sim = (SimulationObject*)simobjs;
  std::lock_guard<std::mutex> lk(g_mu);
  for (int n = 0; n < nsims; n++) {
    Attached* a = find(&sim[n].solver);
    if (!a) return fail(PIAFS_ERR_ARGUMENT, "this HyPar object is not attached (piafs_gpu_attach)");
    if (int r = piafs_gpu_get_state(a->gpu, sim[n].solver.u)) return report(r);
  }
  return PIAFS_OK;
}

int piafs_gpu_TimeRK_ts(void* ts) {
  if (!ts) return fail(PIAFS_ERR_ARGUMENT, "null TimeIntegration");
  TimeIntegration* TS = (TimeIntegration*)ts;
  SimulationObject* sim = (SimulationObject*)TS->simulation;
  std::lock_guard<std::mutex> lk(g_mu);
  for (int n = 0; n < TS->nsims; n++) {
    HyPar* h = &sim[n].solver;
    if (!find(h))
      if (int r = attach_one(&sim[n], PIAFS_PRECISION_FP64, TS->waqt)) return r;
    Attached& a = *find(h);
    if (int r = piafs_gpu_TimeRK(a.gpu, 1)) return report(r);
    piafs_gpu_info info;
    piafs_gpu_get_info(a.gpu, &info);
    h->count_hyp += info.nstages;
    if (a.par_counted) h->count_par += info.nstages;
    if (a.sou_counted) h->count_sou += info.nstages;
    // the steps after which the reference reads solver->u on the host
    const int next = TS->iter + 1;
    const bool out = next % h->file_op_iter == 0 || next >= h->n_iter;
    const bool need = next % h->screen_op_iter == 0 || (next + 1) % h->screen_op_iter == 0 || out;
    if (need)
      if (int r = piafs_gpu_get_state(a.gpu, h->u)) return report(r);
    if (out && a.species && a.chem && a.chem->nv_hnu)
      if (int r = piafs_gpu_get_photon_density(a.gpu, a.chem->nv_hnu)) return report(r);
  }
  return PIAFS_OK;
}

int piafs_gpu_hypar_RHSFunction(double* rhs, double* u, void* s, void* m, double t) {
  (void)m;
  Attached* a = lookup(s);
  if (!a || !rhs || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  const size_t n = (size_t)a->npg * a->nvars;
  HyPar* h = (HyPar*)s;
  if (int r = h2d(a->stage[0], u, n)) return r;
  if (int r = piafs_gpu_RHSFunction(a->gpu, a->stage[1], a->stage[0], t)) return report(r);
  h->count_hyp++;
  if (a->par_counted) h->count_par++;
  if (a->sou_counted) h->count_sou++;
  if (int r = d2h(u, a->stage[0], n)) return r;
  return d2h(rhs, a->stage[1], n);
}

int piafs_gpu_hypar_HyperbolicFunction(double* hyp, double* u, void* s, void* m, double t, int LimFlag,
                                       int (*FFunction)(double*, double*, int, void*, double),
                                       int (*Upwind)(double*, double*, double*, double*, double*, double*, int,
                                                     void*, double)) {
  (void)m; (void)LimFlag; (void)Upwind;
  Attached* a = lookup(s);
  if (!a || !hyp || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  const size_t n = (size_t)a->npg * a->nvars;
  if (!FFunction) {   // HyperbolicFunction.c:67-69: zero hyperbolic term
    std::memset(hyp, 0, n * sizeof(double));
    return PIAFS_OK;
  }
  ((HyPar*)s)->count_hyp++;
  if (int r = h2d(a->stage[0], u, n)) return r;
  if (int r = piafs_gpu_HyperbolicFunction(a->gpu, a->stage[1], a->stage[0], t)) return report(r);
  return d2h(hyp, a->stage[1], n);
}

int piafs_gpu_hypar_ParabolicFunction(double* par, double* u, void* s, void* m, double t) {
  (void)m;
  Attached* a = lookup(s);
  if (!a || !par || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  const size_t n = (size_t)a->npg * a->nvars;
  if (a->par_counted) ((HyPar*)s)->count_par++;
  if (int r = h2d(a->stage[0], u, n)) return r;
  if (int r = piafs_gpu_ParabolicFunction(a->gpu, a->stage[1], a->stage[0], t)) return report(r);
  return d2h(par, a->stage[1], n);
}

int piafs_gpu_hypar_SourceFunction(double* source, double* u, void* s, void* m, double t) {
  (void)m;
  Attached* a = lookup(s);
  if (!a || !source || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  const size_t n = (size_t)a->npg * a->nvars;
  if (a->sou_counted) ((HyPar*)s)->count_sou++;
  if (int r = h2d(a->stage[0], u, n)) return r;
  if (int r = piafs_gpu_SourceFunction(a->gpu, a->stage[1], a->stage[0], t)) return report(r);
  return d2h(source, a->stage[1], n);
}

int piafs_gpu_hypar_ApplyBoundaryConditions(void* s, void* m, double* u, double* uref, double t) {
  (void)m; (void)uref;
  Attached* a = lookup(s);
  if (!a || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  const size_t n = (size_t)a->npg * a->nvars;
  if (int r = h2d(a->stage[0], u, n)) return r;
  if (int r = piafs_gpu_ApplyBoundaryConditions(a->gpu, a->stage[0], t)) return report(r);
  return d2h(u, a->stage[0], n);
}

int piafs_gpu_hypar_FFunction(double* f, double* u, int dir, void* s, double t) {
  Attached* a = lookup(s);
  if (!a || !f || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  const size_t n = (size_t)a->npg * a->nvars;
  if (int r = h2d(a->stage[0], u, n)) return r;
  if (int r = piafs_gpu_FFunction(a->gpu, a->stage[1], a->stage[0], dir, t)) return report(r);
  return d2h(f, a->stage[1], n);
}

int piafs_gpu_hypar_Upwind(double* fI, double* fL, double* fR, double* uL, double* uR, double* u, int dir,
                           void* s, double t) {
  Attached* a = lookup(s);
  if (!a || !fI || !fL || !fR || !uL || !uR || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  if (dir < 0 || dir > 1 || a->nint[dir] == 0) return fail(PIAFS_ERR_ARGUMENT, "bad direction");
  const size_t ni = (size_t)a->nint[dir] * a->nvars, n = (size_t)a->npg * a->nvars;
  if (int r = h2d(a->stage[0], fL, ni)) return r;
  if (int r = h2d(a->stage[1], fR, ni)) return r;
  if (int r = h2d(a->stage[2], uL, ni)) return r;
  if (int r = h2d(a->stage[3], uR, ni)) return r;
  if (int r = h2d(a->stage[4], u, n)) return r;
  if (int r = piafs_gpu_Upwind(a->gpu, a->stage[5], a->stage[0], a->stage[1], a->stage[2], a->stage[3], a->stage[4],
                               dir, t))
    return report(r);
  return d2h(fI, a->stage[5], ni);
}

int piafs_gpu_hypar_InterpolateInterfacesHyp(double* fI, double* fC, double* u, double* x, int upw, int dir,
                                             void* s, void* m, int uflag) {
  (void)x; (void)m;
  Attached* a = lookup(s);
  if (!a || !fI || !fC || !u) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  if (dir < 0 || dir > 1 || a->nint[dir] == 0) return fail(PIAFS_ERR_ARGUMENT, "bad direction");
  const size_t ni = (size_t)a->nint[dir] * a->nvars, n = (size_t)a->npg * a->nvars;
  if (int r = h2d(a->stage[0], fC, n)) return r;
  if (int r = h2d(a->stage[1], u, n)) return r;
  if (int r = piafs_gpu_InterpolateInterfacesHyp(a->gpu, a->stage[2], a->stage[0], a->stage[1], upw, dir, uflag))
    return report(r);
  return d2h(fI, a->stage[2], ni);
}

int piafs_gpu_hypar_FirstDerivativePar(double* Df, double* f, int dir, int bias, void* s, void* m) {
  (void)m;
  Attached* a = lookup(s);
  if (!a || !Df || !f) return a ? fail(PIAFS_ERR_ARGUMENT, "null argument") : PIAFS_ERR_ARGUMENT;
  const size_t n = (size_t)a->npg * a->nvars;
  if (int r = h2d(a->stage[0], f, n)) return r;
  if (int r = piafs_gpu_FirstDerivativePar(a->gpu, a->stage[1], a->stage[0], dir, bias, a->nvars)) return report(r);
  return d2h(Df, a->stage[1], n);
}

}  // extern "C"
