/* CPU restatement of the PIAFS per-stage RHS + explicit RK path.
 *
 * TEST INFRASTRUCTURE ONLY (see piafs_oracle.h).  Each function cites the
 * reference file:line it restates; arithmetic is written in the reference's
 * evaluation order so that, built with the same compiler flags as the
 * reference (-O2, no FMA contraction), results agree bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "piafs_oracle.h"

#define G (P->ghosts)
static inline int W0(const orc_params* P) { return P->dim[0] + 2 * P->ghosts; }
static inline int W1(const orc_params* P) { return P->ndims == 2 ? P->dim[1] + 2 * P->ghosts : 1; }
static inline int G1(const orc_params* P) { return P->ndims == 2 ? P->ghosts : 0; }
/* point index of cell (i,j) (arrayfunctions.h:43-50) */
static inline long PIX(const orc_params* P, int i, int j) {
  return (long)(i + P->ghosts) + (long)W0(P) * (long)(j + G1(P));
}
static inline int NO(const orc_params* P, int dir) { /* number of lines along dir */
  if (P->ndims == 1) return 1;
  return dir == 0 ? P->dim[1] : P->dim[0];
}
/* interface index (i along dir, l = line) in an interface array (bounds_inter) */
static inline long IIX(const orc_params* P, int dir, int i, int l) {
  if (P->ndims == 1) return i;
  if (dir == 0) return (long)i + (long)(P->dim[0] + 1) * l;
  return (long)l + (long)P->dim[0] * i;
}
/* cell (i along dir, line l) */
static inline long CIX(const orc_params* P, int dir, int i, int l) {
  if (P->ndims == 1) return PIX(P, i, 0);
  return dir == 0 ? PIX(P, i, l) : PIX(P, l, i);
}
static inline long STRIDE(const orc_params* P, int dir) { return dir == 0 ? 1 : W0(P); }

#define absolute(a) ((a) < 0 ? -(a) : (a))
#define maxd(a, b) ((a) > (b) ? (a) : (b))
#define max3(a, b, c) maxd(maxd((a), (b)), maxd((b), (c)))

long orc_npoints_ghosted(const orc_params* P) { return (long)W0(P) * W1(P); }
long orc_ninterfaces(const orc_params* P, int dir) {
  if (P->ndims == 1) return P->dim[0] + 1;
  return dir == 0 ? (long)(P->dim[0] + 1) * P->dim[1] : (long)P->dim[0] * (P->dim[1] + 1);
}

/* ---------------------------------------------------------------- flow vars */
/* _NavierStokes2DGetFlowVar_ (navierstokes2d.h:70-80) */
static inline void ns_flowvar(const double* u, double g, double* rho, double* vx, double* vy,
                              double* e, double* P) {
  double vsq;
  *rho = u[0];
  *vx = (*rho == 0) ? 0 : u[1] / *rho;
  *vy = (*rho == 0) ? 0 : u[2] / *rho;
  *e = u[3];
  vsq = (*vx * *vx) + (*vy * *vy);
  *P = (*e - 0.5 * *rho * vsq) * (g - 1.0);
}
/* _Euler1DGetFlowVar_ (euler1d.h:61-69) */
static inline void eu_flowvar(const double* u, double g, double* rho, double* v, double* e, double* P) {
  *rho = u[0];
  *v = u[1] / *rho;
  *e = u[2];
  *P = (*e - 0.5 * *rho * *v * *v) * (g - 1.0);
}

/* --------------------------------------------------------------- boundaries */
/* BCPeriodicU (BCPeriodic.c:22-62), BCExtrapolateU (BCExtrapolate.c:16-50),
 * BCSlipWallU (BCSlipWall.c:24-136); zones are applied in file order
 * (ApplyBoundaryConditions.c:48-51). */
int orc_apply_bc(const orc_params* P, double* u) {
  int nv = P->nvars, n;
  for (n = 0; n < P->nb; n++) {
    int d = P->bc_dim[n], face = P->bc_face[n];
    int is0 = P->bc_is[n][0], ie0 = P->bc_ie[n][0];
    int is1 = P->ndims == 2 ? P->bc_is[n][1] : 0, ie1 = P->ndims == 2 ? P->bc_ie[n][1] : 1;
    int i, j;
    for (j = is1; j < ie1; j++) {
      for (i = is0; i < ie0; i++) {
        int gi[2] = {i, j};
        long p1 = PIX(P, i, j), p2;
        int b = gi[d] - P->bc_is[n][d];                     /* 0..g-1 */
        int src[2] = {i, j};
        if (P->bc_type[n] == ORC_BC_PERIODIC) {
          /* the source index keeps the zone-relative index in the other
           * dimension (BCPeriodic.c:47-53 index without the is[] offset) */
          int o = 1 - d;
          if (P->ndims == 2) src[o] = gi[o] - P->bc_is[n][o];
          if (face == 1) src[d] = b + P->dim[d] - G;       /* index2 = index1 + size - ghosts */
          else src[d] = b;
        } else {
          if (face == 1) src[d] = G - 1 - b;
          else src[d] = P->dim[d] - b - 1;
        }
        p2 = PIX(P, src[0], src[1]);
        if (P->bc_type[n] == ORC_BC_SLIPWALL) {
          double g = P->bc_gamma;
          double inv_gamma_m1 = 1.0 / (g - 1.0);
          if (P->ndims == 1) {
            double rho, uvel, energy, pressure, rho_gpt, uvel_gpt, energy_gpt, pressure_gpt;
            eu_flowvar(u + (long)nv * p2, g, &rho, &uvel, &energy, &pressure);
            rho_gpt = rho;
            pressure_gpt = pressure;
            uvel_gpt = 2.0 * P->bc_vel[n][0] - uvel;
            energy_gpt = inv_gamma_m1 * pressure_gpt + 0.5 * rho_gpt * uvel_gpt * uvel_gpt;
            u[nv * p1 + 0] = rho_gpt;
            u[nv * p1 + 1] = rho_gpt * uvel_gpt;
            u[nv * p1 + 2] = energy_gpt;
          } else {
            double rho, uvel, vvel, energy, pressure, uvel_gpt, vvel_gpt, energy_gpt;
            ns_flowvar(u + (long)nv * p2, g, &rho, &uvel, &vvel, &energy, &pressure);
            if (d == 0) { uvel_gpt = 2.0 * P->bc_vel[n][0] - uvel; vvel_gpt = vvel; }
            else        { uvel_gpt = uvel; vvel_gpt = 2.0 * P->bc_vel[n][1] - vvel; }
            energy_gpt = inv_gamma_m1 * pressure + 0.5 * rho * (uvel_gpt * uvel_gpt + vvel_gpt * vvel_gpt);
            u[nv * p1 + 0] = rho;
            u[nv * p1 + 1] = rho * uvel_gpt;
            u[nv * p1 + 2] = rho * vvel_gpt;
            u[nv * p1 + 3] = energy_gpt;
          }
        } else {
          memcpy(u + nv * p1, u + nv * p2, sizeof(double) * nv);
        }
      }
    }
  }
  return 0;
}

/* --------------------------------------------------------------------- flux */
/* NavierStokes2DFlux (NavierStokes2DFlux.c:24-52, navierstokes2d.h:88-113),
 * Euler1DFlux (Euler1DFlux.c:19-45, euler1d.h:74-88): all points incl. ghosts */
int orc_flux(const orc_params* P, double* f, const double* u, int dir) {
  long np = orc_npoints_ghosted(P), p;
  int nv = P->nvars, m;
  for (p = 0; p < np; p++) {
    const double* up = u + nv * p;
    double* fp = f + nv * p;
    if (P->model == ORC_NS2D) {
      double rho, vx, vy, e, Pr;
      ns_flowvar(up, P->gamma, &rho, &vx, &vy, &e, &Pr);
      if (dir == 0) {
        fp[0] = rho * vx; fp[1] = rho * vx * vx + Pr; fp[2] = rho * vx * vy; fp[3] = (e + Pr) * vx;
        for (m = 4; m < nv; m++) fp[m] = vx * up[m];
      } else {
        fp[0] = rho * vy; fp[1] = rho * vy * vx; fp[2] = rho * vy * vy + Pr; fp[3] = (e + Pr) * vy;
        for (m = 4; m < nv; m++) fp[m] = vy * up[m];
      }
    } else {
      double rho, v, e, Pr;
      eu_flowvar(up, P->gamma, &rho, &v, &e, &Pr);
      fp[0] = (rho) * (v); fp[1] = (rho) * (v) * (v) + (Pr); fp[2] = ((e) + (Pr)) * (v);
      for (m = 3; m < nv; m++) fp[m] = v * up[m];
    }
  }
  return 0;
}

/* ------------------------------------------------------------ WENO weights */
static const double thirteen_by_twelve = 13.0 / 12.0;
static const double one_fourth = 1.0 / 4.0;
static const double one_sixth = 1.0 / 6.0;
static const double one_third = 1.0 / 3.0;

/* _WENOWeights_v_JS_/_M_/_Z_/_YC_ (interpolation.h:255-545), one value */
static inline void weno_weights(int type, double c1, double c2, double c3, double m3, double m2,
                                double m1, double p1, double p2, double eps, double* w1,
                                double* w2, double* w3) {
  double b1, b2, b3, a1, a2, a3, a_sum_inv, tau;
  b1 = thirteen_by_twelve * (m3 - 2 * m2 + m1) * (m3 - 2 * m2 + m1)
     + one_fourth * (m3 - 4 * m2 + 3 * m1) * (m3 - 4 * m2 + 3 * m1);
  b2 = thirteen_by_twelve * (m2 - 2 * m1 + p1) * (m2 - 2 * m1 + p1)
     + one_fourth * (m2 - p1) * (m2 - p1);
  b3 = thirteen_by_twelve * (m1 - 2 * p1 + p2) * (m1 - 2 * p1 + p2)
     + one_fourth * (3 * m1 - 4 * p1 + p2) * (3 * m1 - 4 * p1 + p2);
  if (type == ORC_W_JS || type == ORC_W_MAPPED) {
    a1 = c1 / ((b1 + eps) * (b1 + eps));
    a2 = c2 / ((b2 + eps) * (b2 + eps));
    a3 = c3 / ((b3 + eps) * (b3 + eps));
    a_sum_inv = 1.0 / (a1 + a2 + a3);
    *w1 = a1 * a_sum_inv; *w2 = a2 * a_sum_inv; *w3 = a3 * a_sum_inv;
    if (type == ORC_W_MAPPED) {
      double x1 = *w1, x2 = *w2, x3 = *w3;
      a1 = x1 * (c1 + c1 * c1 - 3 * c1 * x1 + x1 * x1) / (c1 * c1 + x1 * (1.0 - 2.0 * c1));
      a2 = x2 * (c2 + c2 * c2 - 3 * c2 * x2 + x2 * x2) / (c2 * c2 + x2 * (1.0 - 2.0 * c2));
      a3 = x3 * (c3 + c3 * c3 - 3 * c3 * x3 + x3 * x3) / (c3 * c3 + x3 * (1.0 - 2.0 * c3));
      a_sum_inv = 1.0 / (a1 + a2 + a3);
      *w1 = a1 * a_sum_inv; *w2 = a2 * a_sum_inv; *w3 = a3 * a_sum_inv;
    }
    return;
  }
  if (type == ORC_W_BORGES) tau = absolute(b3 - b1);
  else tau = (m3 - 4 * m2 + 6 * m1 - 4 * p1 + p2) * (m3 - 4 * m2 + 6 * m1 - 4 * p1 + p2);
  a1 = c1 * (1.0 + (tau / (b1 + eps)) * (tau / (b1 + eps)));
  a2 = c2 * (1.0 + (tau / (b2 + eps)) * (tau / (b2 + eps)));
  a3 = c3 * (1.0 + (tau / (b3 + eps)) * (tau / (b3 + eps)));
  a_sum_inv = 1.0 / (a1 + a2 + a3);
  *w1 = a1 * a_sum_inv; *w2 = a2 * a_sum_inv; *w3 = a3 * a_sum_inv;
}

/* stencil cells for interface i (Interp1PrimFifthOrderWENO.c:124-144):
 * upw>0: qm1 = i-1, (m3,m2,m1,p1,p2) = (i-3,i-2,i-1,i,i+1);
 * upw<0: qm1 = i,   (m3,m2,m1,p1,p2) = (i+2,i+1,i,i-1,i-2). */
static inline void stencil(const orc_params* P, int dir, int i, int l, int upw, long q[5]) {
  long s = STRIDE(P, dir);
  long qm1 = CIX(P, dir, upw > 0 ? i - 1 : i, l);
  if (upw > 0) { q[0] = qm1 - 2 * s; q[1] = qm1 - s; q[2] = qm1; q[3] = qm1 + s; q[4] = qm1 + 2 * s; }
  else         { q[0] = qm1 + 2 * s; q[1] = qm1 + s; q[2] = qm1; q[3] = qm1 - s; q[4] = qm1 - 2 * s; }
}

/* optimal weights (WENOFifthOrderCalculateWeights.c:208-226; single rank) */
static inline void optimal(const orc_params* P, int dir, int i, double* c1, double* c2, double* c3) {
  if (P->scheme == ORC_CRWENO5 && !(i == 0 || i == P->dim[dir])) {
    *c1 = 0.2; *c2 = 0.5; *c3 = 0.3;
  } else {
    *c1 = 0.1; *c2 = 0.6; *c3 = 0.3;
  }
}

/* ------------------------------------------------------------ tridiagonal */
/* tridiagLU serial path (tridiagLU.c:133-153 forward, :242-262 backward) */
int orc_tridiag(double* a, double* b, double* c, double* x, int n, int ns) {
  int i, d, bad = 0;
  if (ns == 0 || n == 0) return 0;
  for (i = 1; i < n; i++) {
    for (d = 0; d < ns; d++) {
      double factor;
      if (b[(long)(i - 1) * ns + d] == 0) { bad = 1; continue; }
      factor = a[(long)i * ns + d] / b[(long)(i - 1) * ns + d];
      b[(long)i * ns + d] -= factor * c[(long)(i - 1) * ns + d];
      a[(long)i * ns + d] = -factor * a[(long)(i - 1) * ns + d];
      x[(long)i * ns + d] -= factor * x[(long)(i - 1) * ns + d];
    }
  }
  {
    int istart = n - 1;
    for (d = 0; d < ns; d++) {
      double xp1 = 0;
      if (b[(long)istart * ns + d] == 0) { bad = 1; continue; }
      x[(long)istart * ns + d] = (x[(long)istart * ns + d] - a[(long)istart * ns + d] * x[d]
                                  - c[(long)istart * ns + d] * xp1) / b[(long)istart * ns + d];
    }
    for (i = istart - 1; i > -1; i--) {
      for (d = 0; d < ns; d++) {
        if (b[(long)i * ns + d] == 0) { bad = 1; continue; }
        x[(long)i * ns + d] = (x[(long)i * ns + d] - c[(long)i * ns + d] * x[(long)(i + 1) * ns + d]
                               - a[(long)i * ns + d] * x[d]) / b[(long)i * ns + d];
      }
    }
  }
  return bad ? -1 : 0;
}

/* ------------------------------------------------------------ interpolation */
/* WENOFifthOrderCalculateWeights + Interp1PrimFifthOrderWENO
 * (Interp1PrimFifthOrderWENO.c:77-171) or Interp1PrimFifthOrderCRWENO
 * (Interp1PrimFifthOrderCRWENO.c:81-240) for one (upw, uflag) */
int orc_interp(const orc_params* P, double* fI, const double* fC, const double* u, int upw,
               int dir, int uflag) {
  int nv = P->nvars, nl = NO(P, dir), N = P->dim[dir], l, i, v, ret = 0;
  const double* F = uflag ? u : fC;
  int crweno = (P->scheme == ORC_CRWENO5);
  int nsys = nl * nv;
  double *A = NULL, *B = NULL, *C = NULL, *R = NULL;
  if (crweno) {
    long tot = (long)(N + 1) * nsys;
    A = (double*)calloc(tot, sizeof(double)); B = (double*)calloc(tot, sizeof(double));
    C = (double*)calloc(tot, sizeof(double)); R = (double*)calloc(tot, sizeof(double));
  }
  for (l = 0; l < nl; l++) {
    for (i = 0; i < N + 1; i++) {
      long q[5], pI = IIX(P, dir, i, l);
      double c1, c2, c3;
      int bnd = (i == 0 || i == N);
      stencil(P, dir, i, l, upw, q);
      optimal(P, dir, i, &c1, &c2, &c3);
      for (v = 0; v < nv; v++) {
        double fm3 = F[nv * q[0] + v], fm2 = F[nv * q[1] + v], fm1 = F[nv * q[2] + v];
        double fp1 = F[nv * q[3] + v], fp2 = F[nv * q[4] + v];
        double w1, w2, w3, f1, f2, f3;
        if (P->no_limiting) { w1 = c1; w2 = c2; w3 = c3; }
        else weno_weights(P->weno_type, c1, c2, c3, fm3, fm2, fm1, fp1, fp2, P->weno_eps, &w1, &w2, &w3);
        if (!crweno || bnd) {
          f1 = (2 * one_sixth) * fm3 + (-7 * one_sixth) * fm2 + (11 * one_sixth) * fm1;
          f2 = (-one_sixth) * fm2 + (5 * one_sixth) * fm1 + (2 * one_sixth) * fp1;
          f3 = (2 * one_sixth) * fm1 + (5 * one_sixth) * fp1 + (-one_sixth) * fp2;
        } else {
          f1 = (one_sixth) * fm2 + (5 * one_sixth) * fm1;
          f2 = (5 * one_sixth) * fm1 + (one_sixth) * fp1;
          f3 = (one_sixth) * fm1 + (5 * one_sixth) * fp1;
        }
        if (!crweno) {
          fI[nv * pI + v] = w1 * f1 + w2 * f2 + w3 * f3;
        } else {
          long r = (long)nsys * i + (long)l * nv + v;
          if (bnd) { A[r] = 0.0; B[r] = 1.0; C[r] = 0.0; }
          else if (upw > 0) {
            A[r] = (2 * one_third) * w1 + (one_third) * w2;
            B[r] = (one_third) * w1 + (2 * one_third) * w2 + (2 * one_third) * w3;
            C[r] = (one_third) * w3;
          } else {
            C[r] = (2 * one_third) * w1 + (one_third) * w2;
            B[r] = (one_third) * w1 + (2 * one_third) * w2 + (2 * one_third) * w3;
            A[r] = (one_third) * w3;
          }
          R[r] = w1 * f1 + w2 * f2 + w3 * f3;
        }
      }
    }
  }
  if (crweno) {
    ret = orc_tridiag(A, B, C, R, N + 1, nsys);
    for (l = 0; l < nl; l++)
      for (i = 0; i < N + 1; i++)
        for (v = 0; v < nv; v++) fI[nv * IIX(P, dir, i, l) + v] = R[(long)nsys * i + (long)l * nv + v];
    free(A); free(B); free(C); free(R);
  }
  return ret;
}

/* --------------------------------------------------------------- upwinding */
/* eigen-structure of the flow block; species are the identity block
 * (navierstokes2d.h:115-313, euler1d.h:93-200) */
typedef struct { double L[4][4], R[4][4], D[4]; int nf; } eig_t;

static void ns_roeavg(const double* uL, const double* uR, double g, double* ua) {
  /* _NavierStokes2DRoeAverage_ (navierstokes2d.h:115-159), flow variables */
  double rho, vx, vy, e, Pp, H, csq, vsq;
  double rhoL, vxL, vyL, eL, PL, HL, cLsq, vsqL;
  double rhoR, vxR, vyR, eR, PR, HR, cRsq, vsqR;
  rhoL = uL[0]; vxL = uL[1] / rhoL; vyL = uL[2] / rhoL; eL = uL[3];
  vsqL = (vxL * vxL) + (vyL * vyL); PL = (eL - 0.5 * rhoL * vsqL) * (g - 1.0);
  cLsq = g * PL / rhoL; HL = 0.5 * (vxL * vxL + vyL * vyL) + cLsq / (g - 1.0);
  rhoR = uR[0]; vxR = uR[1] / rhoR; vyR = uR[2] / rhoR; eR = uR[3];
  vsqR = (vxR * vxR) + (vyR * vyR); PR = (eR - 0.5 * rhoR * vsqR) * (g - 1.0);
  cRsq = g * PR / rhoR; HR = 0.5 * (vxR * vxR + vyR * vyR) + cRsq / (g - 1.0);
  {
    double tL = sqrt(rhoL), tR = sqrt(rhoR);
    rho = tL * tR;
    vx = (tL * vxL + tR * vxR) / (tL + tR);
    vy = (tL * vyL + tR * vyR) / (tL + tR);
    H = (tL * HL + tR * HR) / (tL + tR);
    vsq = vx * vx + vy * vy;
    csq = (g - 1.0) * (H - 0.5 * vsq);
    Pp = csq * rho / g;
    e = Pp / (g - 1.0) + 0.5 * rho * vsq;
    ua[0] = rho; ua[1] = rho * vx; ua[2] = rho * vy; ua[3] = e;
  }
}
static void eu_roeavg(const double* uL, const double* uR, double g, double* ua) {
  /* _Euler1DRoeAverage_ (euler1d.h:93-125) */
  double rho, v, e, Pp, H, csq, rhoL, vL, eL, PL, HL, cLsq, rhoR, vR, eR, PR, HR, cRsq;
  rhoL = uL[0]; vL = uL[1] / rhoL; eL = uL[2]; PL = (eL - 0.5 * rhoL * vL * vL) * (g - 1.0);
  cLsq = g * PL / rhoL; HL = 0.5 * vL * vL + cLsq / (g - 1.0);
  rhoR = uR[0]; vR = uR[1] / rhoR; eR = uR[2]; PR = (eR - 0.5 * rhoR * vR * vR) * (g - 1.0);
  cRsq = g * PR / rhoR; HR = 0.5 * vR * vR + cRsq / (g - 1.0);
  {
    double tL = sqrt(rhoL), tR = sqrt(rhoR);
    rho = tL * tR;
    v = (tL * vL + tR * vR) / (tL + tR);
    H = (tL * HL + tR * HR) / (tL + tR);
    csq = (g - 1.0) * (H - 0.5 * v * v);
    Pp = csq * rho / g;
    e = Pp / (g - 1.0) + 0.5 * rho * v * v;
    ua[0] = rho; ua[1] = rho * v; ua[2] = e;
  }
}
/* eigenvalues of the flow block (navierstokes2d.h:161-190 / euler1d.h:131-147);
 * returns the species eigenvalue (normal velocity) */
static double ns_eigvals(const double* u, double g, int dir, double D[4]) {
  double rho, vx, vy, e, Pp, c, vn;
  ns_flowvar(u, g, &rho, &vx, &vy, &e, &Pp);
  c = sqrt(g * Pp / rho);
  vn = dir == 0 ? vx : vy;
  D[0] = vn - c;
  if (dir == 0) { D[1] = vn + c; D[2] = vn; } else { D[1] = vn; D[2] = vn + c; }
  D[3] = vn;
  return vn;
}
static double eu_eigvals(const double* u, double g, double D[3]) {
  double rho, v, e, Pp, c;
  eu_flowvar(u, g, &rho, &v, &e, &Pp);
  c = sqrt(g * Pp / rho);
  D[0] = v; D[1] = (v - c); D[2] = (v + c);
  return v;
}
static void ns_eigvec(const double* u, double ga, int dir, eig_t* E) {
  /* _NavierStokes2DLeftEigenvectors_ / _RightEigenvectors_ (navierstokes2d.h:194-313) */
  double gm1 = ga - 1.0, rho, vx, vy, e, Pp, a, un, ek, h0, nx = 0, ny = 0;
  double (*L)[4] = E->L, (*R)[4] = E->R;
  ns_flowvar(u, ga, &rho, &vx, &vy, &e, &Pp);
  ek = 0.5 * (vx * vx + vy * vy);
  a = sqrt(ga * Pp / rho);
  h0 = a * a / gm1 + ek;
  E->nf = 4;
  if (dir == 0) {
    un = vx; nx = 1.0;
    L[0][0] = (gm1 * ek + a * un) / (2 * a * a);
    L[0][1] = ((-gm1) * vx - a * nx) / (2 * a * a);
    L[0][2] = ((-gm1) * vy - a * ny) / (2 * a * a);
    L[0][3] = gm1 / (2 * a * a);
    L[3][0] = (a * a - gm1 * ek) / (a * a);
    L[3][1] = (gm1 * vx) / (a * a);
    L[3][2] = (gm1 * vy) / (a * a);
    L[3][3] = (-gm1) / (a * a);
    L[1][0] = (gm1 * ek - a * un) / (2 * a * a);
    L[1][1] = ((-gm1) * vx + a * nx) / (2 * a * a);
    L[1][2] = ((-gm1) * vy + a * ny) / (2 * a * a);
    L[1][3] = gm1 / (2 * a * a);
    L[2][0] = (vy - un * ny) / nx;
    L[2][1] = ny;
    L[2][2] = (ny * ny - 1.0) / nx;
    L[2][3] = 0.0;
    R[0][0] = 1.0; R[1][0] = vx - a * nx; R[2][0] = vy - a * ny; R[3][0] = h0 - a * un;
    R[0][3] = 1.0; R[1][3] = vx; R[2][3] = vy; R[3][3] = ek;
    R[0][1] = 1.0; R[1][1] = vx + a * nx; R[2][1] = vy + a * ny; R[3][1] = h0 + a * un;
    R[0][2] = 0.0; R[1][2] = ny; R[2][2] = -nx; R[3][2] = vx * ny - vy * nx;
  } else {
    un = vy; ny = 1.0;
    L[0][0] = (gm1 * ek + a * un) / (2 * a * a);
    L[0][1] = ((1.0 - ga) * vx - a * nx) / (2 * a * a);
    L[0][2] = ((1.0 - ga) * vy - a * ny) / (2 * a * a);
    L[0][3] = gm1 / (2 * a * a);
    L[3][0] = (a * a - gm1 * ek) / (a * a);
    L[3][1] = gm1 * vx / (a * a);
    L[3][2] = gm1 * vy / (a * a);
    L[3][3] = (1.0 - ga) / (a * a);
    L[2][0] = (gm1 * ek - a * un) / (2 * a * a);
    L[2][1] = ((1.0 - ga) * vx + a * nx) / (2 * a * a);
    L[2][2] = ((1.0 - ga) * vy + a * ny) / (2 * a * a);
    L[2][3] = gm1 / (2 * a * a);
    L[1][0] = (un * nx - vx) / ny;
    L[1][1] = (1.0 - nx * nx) / ny;
    L[1][2] = -nx;
    L[1][3] = 0;
    R[0][0] = 1.0; R[1][0] = vx - a * nx; R[2][0] = vy - a * ny; R[3][0] = h0 - a * un;
    R[0][3] = 1.0; R[1][3] = vx; R[2][3] = vy; R[3][3] = ek;
    R[0][2] = 1.0; R[1][2] = vx + a * nx; R[2][2] = vy + a * ny; R[3][2] = h0 + a * un;
    R[0][1] = 0; R[1][1] = ny; R[2][1] = -nx; R[3][1] = vx * ny - vy * nx;
  }
}
static void eu_eigvec(const double* u, double gamma, eig_t* E) {
  /* _Euler1DLeftEigenvectors_ / _RightEigenvectors_ (euler1d.h:153-200) */
  double rho, v, e, Pp, c;
  double (*L)[4] = E->L, (*R)[4] = E->R;
  eu_flowvar(u, gamma, &rho, &v, &e, &Pp);
  c = sqrt(gamma * Pp / rho);
  E->nf = 3;
  memset(E->L, 0, sizeof(E->L)); memset(E->R, 0, sizeof(E->R));
  L[1][0] = ((gamma - 1) / (rho * c)) * (-(v * v) / 2 - c * v / (gamma - 1));
  L[1][1] = ((gamma - 1) / (rho * c)) * (v + c / (gamma - 1));
  L[1][2] = ((gamma - 1) / (rho * c)) * (-1);
  L[0][0] = ((gamma - 1) / (rho * c)) * (rho * (-(v * v) / 2 + c * c / (gamma - 1)) / c);
  L[0][1] = ((gamma - 1) / (rho * c)) * (rho * v / c);
  L[0][2] = ((gamma - 1) / (rho * c)) * (-rho / c);
  L[2][0] = ((gamma - 1) / (rho * c)) * ((v * v) / 2 - c * v / (gamma - 1));
  L[2][1] = ((gamma - 1) / (rho * c)) * (-v + c / (gamma - 1));
  L[2][2] = ((gamma - 1) / (rho * c)) * (1);
  R[0][1] = -rho / (2 * c); R[1][1] = -rho * (v - c) / (2 * c);
  R[2][1] = -rho * ((v * v) / 2 + (c * c) / (gamma - 1) - c * v) / (2 * c);
  R[0][0] = 1; R[1][0] = v; R[2][0] = v * v / 2;
  R[0][2] = rho / (2 * c); R[1][2] = rho * (v + c) / (2 * c);
  R[2][2] = rho * ((v * v) / 2 + (c * c) / (gamma - 1) + c * v) / (2 * c);
}

/* y = M x on the flow block (MatVecMult, matmult_native.h:119-126; species
 * rows of the block-diagonal matrices are the identity) */
static inline void fmatvec(int nf, double M[4][4], const double* x, double* y) {
  int i, j;
  for (i = 0; i < nf; i++) { y[i] = 0; for (j = 0; j < nf; j++) y[i] += M[i][j] * x[j]; }
}

/* NavierStokes2DUpwind{Roe,RF,LLF,Rusanov} (NavierStokes2DUpwind.c:26-332)
 * and Euler1DUpwind{Roe,RF,LLF,Rusanov} (Euler1DUpwind.c:27-330) */
int orc_upwind(const orc_params* P, double* fI, const double* fL, const double* fR,
               const double* uL, const double* uR, const double* u, int dir) {
  int nv = P->nvars, nl = NO(P, dir), N = P->dim[dir], l, i, k;
  int ns2d = (P->model == ORC_NS2D), nf = ns2d ? 4 : 3;
  double g = P->gamma;
  for (l = 0; l < nl; l++) {
    for (i = 0; i < N + 1; i++) {
      long p = IIX(P, dir, i, l);
      long pL = CIX(P, dir, i - 1, l), pR = CIX(P, dir, i, l);
      const double *uLp = uL + nv * p, *uRp = uR + nv * p, *fLp = fL + nv * p, *fRp = fR + nv * p;
      double* fIp = fI + nv * p;
      double ua[4], D[4], vnC;
      eig_t E;
      if (P->upwind == ORC_ROE) {
        double udiff[64], DL[4][4], modA[4][4], udiss[4];
        int a, b, c;
        for (k = 0; k < nv; k++) udiff[k] = 0.5 * (uRp[k] - uLp[k]);
        if (ns2d) {
          ns_roeavg(u + nv * pL, u + nv * pR, g, ua);
          vnC = ns_eigvals(ua, g, dir, D);
          ns_eigvec(ua, g, dir, &E);
        } else {
          eu_roeavg(u + nv * pL, u + nv * pR, g, ua);
          vnC = eu_eigvals(ua, g, D);
          eu_eigvec(ua, g, &E);
        }
        {
          double Ds[4], dsp;
          if (ns2d) {
            double delta = 0.000001, delta2 = delta * delta;
            for (a = 0; a < nf; a++)
              Ds[a] = (absolute(D[a]) < delta ? (D[a] * D[a] + delta2) / (2 * delta) : absolute(D[a]));
            dsp = (absolute(vnC) < delta ? (vnC * vnC + delta2) / (2 * delta) : absolute(vnC));
          } else {
            for (a = 0; a < nf; a++) Ds[a] = absolute(D[a]);
            dsp = absolute(vnC);
          }
          for (a = 0; a < nf; a++) for (b = 0; b < nf; b++) DL[a][b] = Ds[a] * E.L[a][b];
          for (a = 0; a < nf; a++) for (b = 0; b < nf; b++) {
            modA[a][b] = 0.0;
            for (c = 0; c < nf; c++) modA[a][b] += E.R[a][c] * DL[c][b];
          }
          fmatvec(nf, modA, udiff, udiss);
          for (k = 0; k < nf; k++) fIp[k] = 0.5 * (fLp[k] + fRp[k]) - udiss[k];
          for (k = nf; k < nv; k++) fIp[k] = 0.5 * (fLp[k] + fRp[k]) - dsp * udiff[k];
        }
      } else if (P->upwind == ORC_RUSANOV) {
        double udiff[64], alphaL, alphaR, alphaavg, alpha, c;
        for (k = 0; k < nv; k++) udiff[k] = 0.5 * (uRp[k] - uLp[k]);
        if (ns2d) {
          double rho, vel[2], Ee, Pp;
          ns_roeavg(u + nv * pL, u + nv * pR, g, ua);
          ns_flowvar(u + nv * pL, g, &rho, &vel[0], &vel[1], &Ee, &Pp);
          c = sqrt(g * Pp / rho); alphaL = c + absolute(vel[dir]);
          ns_flowvar(u + nv * pR, g, &rho, &vel[0], &vel[1], &Ee, &Pp);
          c = sqrt(g * Pp / rho); alphaR = c + absolute(vel[dir]);
          ns_flowvar(ua, g, &rho, &vel[0], &vel[1], &Ee, &Pp);
          c = sqrt(g * Pp / rho); alphaavg = c + absolute(vel[dir]);
        } else {
          double rho, uvel, Ee, Pp;
          eu_roeavg(u + nv * pL, u + nv * pR, g, ua);
          eu_flowvar(u + nv * pL, g, &rho, &uvel, &Ee, &Pp);
          c = g * Pp / rho; alphaL = c + absolute(uvel);     /* no sqrt (Euler1DUpwind.c) */
          eu_flowvar(u + nv * pR, g, &rho, &uvel, &Ee, &Pp);
          c = g * Pp / rho; alphaR = c + absolute(uvel);
          eu_flowvar(ua, g, &rho, &uvel, &Ee, &Pp);
          c = g * Pp / rho; alphaavg = c + absolute(uvel);
        }
        alpha = max3(alphaL, alphaR, alphaavg);
        for (k = 0; k < nv; k++) fIp[k] = 0.5 * (fLp[k] + fRp[k]) - alpha * udiff[k];
      } else {
        /* characteristic-based LLF / RF */
        double ucL[4], ucR[4], fcL[4], fcR[4], fc[4], eigL[4], eigR[4], eigC[4], vnL, vnR;
        if (ns2d) {
          ns_roeavg(uLp, uRp, g, ua);
          ns_eigvec(ua, g, dir, &E);
          vnL = ns_eigvals(uLp, g, dir, eigL);
          vnR = ns_eigvals(uRp, g, dir, eigR);
          vnC = ns_eigvals(ua, g, dir, eigC);
        } else {
          /* Euler1D LLF/RF average the cell-centred states (Euler1DUpwind.c) */
          eu_roeavg(u + nv * pL, u + nv * pR, g, ua);
          eu_eigvec(ua, g, &E);
          vnL = eu_eigvals(u + nv * pL, g, eigL);
          vnR = eu_eigvals(u + nv * pR, g, eigR);
          vnC = eu_eigvals(ua, g, eigC);
        }
        fmatvec(nf, E.L, uLp, ucL); fmatvec(nf, E.L, uRp, ucR);
        fmatvec(nf, E.L, fLp, fcL); fmatvec(nf, E.L, fRp, fcR);
        for (k = 0; k < nf; k++) {
          if (P->upwind == ORC_RF && (eigL[k] > 0) && (eigC[k] > 0) && (eigR[k] > 0)) fc[k] = fcL[k];
          else if (P->upwind == ORC_RF && (eigL[k] < 0) && (eigC[k] < 0) && (eigR[k] < 0)) fc[k] = fcR[k];
          else {
            double alpha = max3(absolute(eigL[k]), absolute(eigC[k]), absolute(eigR[k]));
            fc[k] = 0.5 * (fcL[k] + fcR[k] + alpha * (ucL[k] - ucR[k]));
          }
        }
        fmatvec(nf, E.R, fc, fIp);
        for (k = nf; k < nv; k++) {
          if (P->upwind == ORC_RF && (vnL > 0) && (vnC > 0) && (vnR > 0)) fIp[k] = fLp[k];
          else if (P->upwind == ORC_RF && (vnL < 0) && (vnC < 0) && (vnR < 0)) fIp[k] = fRp[k];
          else {
            double alpha = max3(absolute(vnL), absolute(vnC), absolute(vnR));
            fIp[k] = 0.5 * (fLp[k] + fRp[k] + alpha * (uLp[k] - uRp[k]));
          }
        }
      }
    }
  }
  return 0;
}

/* ---------------------------------------------------------------- hyperbolic */
/* HyperbolicFunction (HyperbolicFunction.c:34-127) + ReconstructHyperbolic (:168-214) */
int orc_hyperbolic(const orc_params* P, double* hyp, const double* u, const double* dxinv) {
  int nv = P->nvars, d, ret = 0;
  long np = orc_npoints_ghosted(P);
  double* fC = (double*)calloc(np * nv, sizeof(double));
  long nimax = orc_ninterfaces(P, 0);
  if (P->ndims == 2 && orc_ninterfaces(P, 1) > nimax) nimax = orc_ninterfaces(P, 1);
  double* fI = (double*)calloc(nimax * nv, sizeof(double));
  double* uL = (double*)calloc(nimax * nv, sizeof(double));
  double* uR = (double*)calloc(nimax * nv, sizeof(double));
  double* fL = (double*)calloc(nimax * nv, sizeof(double));
  double* fR = (double*)calloc(nimax * nv, sizeof(double));
  int offset = 0;
  memset(hyp, 0, sizeof(double) * np * nv);
  for (d = 0; d < P->ndims; d++) {
    int nl = NO(P, d), N = P->dim[d], l, i, v;
    orc_flux(P, fC, u, d);
    ret |= orc_interp(P, uL, fC, u, 1, d, 1);
    ret |= orc_interp(P, uR, fC, u, -1, d, 1);
    ret |= orc_interp(P, fL, fC, u, 1, d, 0);
    ret |= orc_interp(P, fR, fC, u, -1, d, 0);
    orc_upwind(P, fI, fL, fR, uL, uR, u, d);
    for (l = 0; l < nl; l++) {
      for (i = 0; i < N; i++) {
        long p = CIX(P, d, i, l), p1 = IIX(P, d, i, l), p2 = IIX(P, d, i + 1, l);
        for (v = 0; v < nv; v++)
          hyp[nv * p + v] += dxinv[offset + G + i] * (fI[nv * p2 + v] - fI[nv * p1 + v]);
      }
    }
    offset += N + 2 * G;
  }
  free(fC); free(fI); free(uL); free(uR); free(fL); free(fR);
  return ret;
}

/* ------------------------------------------------------------------ viscous */
/* FirstDerivativeFirstOrder (FirstDerivativeFirstOrder.c:40-100): one-sided
 * differences on the lines along dir that are interior in the other dims */
int orc_first_derivative(const orc_params* P, double* Df, const double* f, int dir, int bias, int nv) {
  int nl = NO(P, dir), N = P->dim[dir], l, i, v;
  int mx = bias > 0 ? bias : 0, mn = bias < 0 ? bias : 0;
  for (l = 0; l < nl; l++) {
    {
      long qC = CIX(P, dir, -G, l), qR = CIX(P, dir, -G + 1, l);
      for (v = 0; v < nv; v++) Df[qC * nv + v] = f[qR * nv + v] - f[qC * nv + v];
    }
    for (i = -G + 1; i < N + G - 1; i++) {
      long qC = CIX(P, dir, i, l), qL = CIX(P, dir, i - 1, l), qR = CIX(P, dir, i + 1, l);
      for (v = 0; v < nv; v++)
        Df[qC * nv + v] = mx * f[qR * nv + v] - bias * f[qC * nv + v] + mn * f[qL * nv + v];
    }
    {
      long qL = CIX(P, dir, N + G - 2, l), qC = CIX(P, dir, N + G - 1, l);
      for (v = 0; v < nv; v++) Df[qC * nv + v] = f[qC * nv + v] - f[qL * nv + v];
    }
  }
  return 0;
}

/* NavierStokes2DParabolicFunction (NavierStokes2DParabolicFunction.c:41-204) */
int orc_parabolic(const orc_params* P, double* par, const double* u, const double* dxinv) {
  int nv = P->nvars, g = G, imax = P->dim[0], jmax = P->dim[1], i, j, v;
  long np = orc_npoints_ghosted(P), size = np * nv;
  static const double two_third = 2.0 / 3.0;
  double inv_gamma_m1, inv_Re, inv_Pr;
  double *Q, *QX, *QY, *FV, *FD;
  memset(par, 0, sizeof(double) * size);
  if (P->model != ORC_NS2D || !P->viscous) return 0;
  inv_gamma_m1 = 1.0 / (P->gamma - 1.0);
  inv_Re = 1.0 / P->Re;
  inv_Pr = 1.0 / P->Pr;
  Q = (double*)calloc(size, sizeof(double)); QX = (double*)calloc(size, sizeof(double));
  QY = (double*)calloc(size, sizeof(double)); FV = (double*)calloc(size, sizeof(double));
  FD = (double*)calloc(size, sizeof(double));
  for (i = -g; i < imax + g; i++)
    for (j = -g; j < jmax + g; j++) {
      long p = PIX(P, i, j) * nv;
      double energy, pressure;
      ns_flowvar(u + p, P->gamma, &Q[p + 0], &Q[p + 1], &Q[p + 2], &energy, &pressure);
      Q[p + 3] = P->gamma * pressure / Q[p + 0];
    }
  orc_first_derivative(P, QX, Q, 0, 1, nv);
  orc_first_derivative(P, QY, Q, 1, 1, nv);
  for (i = -g; i < imax + g; i++)
    for (j = -g; j < jmax + g; j++) {
      long p = PIX(P, i, j) * nv;
      double dxi = dxinv[g + i], dyi = dxinv[(imax + 2 * g) + g + j];
      for (v = 0; v < nv; v++) { QX[p + v] *= dxi; QY[p + v] *= dyi; }
    }
#define VISC_COEFFS(T)                                                                   \
  double T_d = (T) * P->Tref;                                                            \
  double mu = exp(1.5 * log(T_d / P->T0)) * (P->T0 + P->TS) / (T_d + P->TS);             \
  double kappa = exp(1.5 * log(T_d / P->T0)) * (P->T0 + P->TA * exp(-P->TB / P->T0))     \
               / (T_d + P->TA * exp(-P->TB / T_d));
  for (i = -g; i < imax + g; i++)
    for (j = -g; j < jmax + g; j++) {
      long p = PIX(P, i, j) * nv;
      double uvel = Q[p + 1], vvel = Q[p + 2], T = Q[p + 3], Tx = QX[p + 3];
      double ux = QX[p + 1], vx = QX[p + 2], uy = QY[p + 1], vy = QY[p + 2];
      double tau_xx, tau_xy, qx;
      VISC_COEFFS(T)
      tau_xx = two_third * (mu * inv_Re) * (2 * ux - vy);
      tau_xy = (mu * inv_Re) * (uy + vx);
      qx = (kappa * inv_Re * inv_gamma_m1 * inv_Pr) * Tx;
      FV[p + 0] = 0.0; FV[p + 1] = tau_xx; FV[p + 2] = tau_xy;
      FV[p + 3] = uvel * tau_xx + vvel * tau_xy + qx;
    }
  orc_first_derivative(P, FD, FV, 0, -1, nv);
  for (i = 0; i < imax; i++)
    for (j = 0; j < jmax; j++) {
      long p = PIX(P, i, j) * nv;
      double dxi = dxinv[g + i];
      for (v = 0; v < nv; v++) par[p + v] += (dxi * FD[p + v]);
    }
  for (i = -g; i < imax + g; i++)
    for (j = -g; j < jmax + g; j++) {
      long p = PIX(P, i, j) * nv;
      double uvel = Q[p + 1], vvel = Q[p + 2], T = Q[p + 3], Ty = QY[p + 3];
      double ux = QX[p + 1], vx = QX[p + 2], uy = QY[p + 1], vy = QY[p + 2];
      double tau_yx, tau_yy, qy;
      VISC_COEFFS(T)
      tau_yx = (mu * inv_Re) * (uy + vx);
      tau_yy = two_third * (mu * inv_Re) * (-ux + 2 * vy);
      qy = (kappa * inv_Re * inv_gamma_m1 * inv_Pr) * Ty;
      FV[p + 0] = 0.0; FV[p + 1] = tau_yx; FV[p + 2] = tau_yy;
      FV[p + 3] = uvel * tau_yx + vvel * tau_yy + qy;
    }
#undef VISC_COEFFS
  orc_first_derivative(P, FD, FV, 1, -1, nv);
  for (i = 0; i < imax; i++)
    for (j = 0; j < jmax; j++) {
      long p = PIX(P, i, j) * nv;
      double dyi = dxinv[(imax + 2 * g) + g + j];
      for (v = 0; v < nv; v++) par[p + v] += (dyi * FD[p + v]);
    }
  free(Q); free(QX); free(QY); free(FV); free(FD);
  return 0;
}

/* ------------------------------------------------------------------- source */
/* SourceFunction (SourceFunction.c:21-60) -> NavierStokes2DSource / Euler1DSource
 * -> ChemistrySource + ChemistrySetPhotonDensity (ChemistrySolve.c:18-115,
 * chemistry.h:30-137) */
int orc_source(const orc_params* P, double* src, const double* u, const double* imap, double t) {
  int nv = P->nvars, nz = P->nz, i, j, iz;
  long np = orc_npoints_ghosted(P);
  int jmax = P->ndims == 2 ? P->dim[1] : 1;
  double* nv_hnu;
  memset(src, 0, sizeof(double) * np * nv);
  if (!P->include_chem) return 0;
  nv_hnu = (double*)calloc(np * nz, sizeof(double));
  for (j = 0; j < jmax; j++)
    for (i = 0; i < P->dim[0]; i++) {
      long p = PIX(P, i, j);
      double sigma = P->t_pulse_norm / 2.35482, I0 = 0.0;
      if (t > P->t_start_norm) {
        double tp = t - (P->t_start_norm + P->t_pulse_norm);
        I0 = P->I0 * exp(-(tp * tp) / (2 * sigma * sigma)) * imap[p];
      }
      nv_hnu[nz * p + 0] = I0 / (P->c * P->h * P->nu * P->n_O2);
      for (iz = 1; iz < nz; iz++) {
        double sg = P->sO3 * P->n_O2;
        double damp_fac = 1.0 - P->dz * sg * u[P->grid_stride * p + P->n_flow_vars + P->z_stride * (iz - 1) + 1];
        nv_hnu[nz * p + iz] = nv_hnu[nz * p + (iz - 1)] * damp_fac;
      }
    }
  for (iz = 0; iz < nz; iz++)
    for (j = 0; j < jmax; j++)
      for (i = 0; i < P->dim[0]; i++) {
        long p = PIX(P, i, j);
        const double* up = u + (long)P->grid_stride * p;
        double* f = src + (long)P->grid_stride * p;
        int nfv = P->n_flow_vars + P->z_stride * iz;
        double n_hnu = nv_hnu[nz * p + iz];
        double n_O2 = up[nfv + 0], n_O3 = up[nfv + 1], n_1D = up[nfv + 2], n_1Dg = up[nfv + 3];
        double n_3Su = up[nfv + 4], n_1Sg = up[nfv + 5], n_CO2 = up[nfv + 6];
        const double* k = P->k; const double* q = P->q;
        double k0a = k[0], k0b = k[1], k1a = k[2], k1b = k[3], k2a = k[4], k2b = k[5];
        double k3a = k[6], k3b = k[7], k4 = k[8], k5 = k[9], k6 = k[10];
        f[nfv + 0] = 0.0;
        f[nfv + 1] = -(k0a + k0b) * n_hnu * n_O3 - (k2a + k2b) * n_O3 * n_1D
                     - (k3a + k3b) * n_O3 * n_1Sg - k5 * n_O3 * n_3Su - k6 * n_1Dg * n_O3;
        f[nfv + 2] = k0a * n_hnu * n_O3 - (k1a + k1b) * n_1D * n_O2 - (k2a + k2b) * n_1D * n_O3
                     - k4 * n_1D * n_CO2;
        f[nfv + 3] = k0a * n_hnu * n_O3 + k5 * n_O3 * n_3Su - k6 * n_1Dg * n_O3;
        f[nfv + 4] = k2a * n_O3 * n_1D - k5 * n_O3 * n_3Su;
        f[nfv + 5] = k1a * n_1D * n_O2 - (k3a + k3b) * n_O3 * n_1Sg;
        f[nfv + 6] = 0.0;
        f[P->n_flow_vars - 1] = ((q[0] * k0a + q[1] * k0b) * n_hnu * n_O3
                                 + (q[2] * k1a + q[3] * k1b) * n_O2 * n_1D
                                 + (q[4] * k2a + q[5] * k2b) * n_O3 * n_1D
                                 + (q[6] * k3a + q[7] * k3b) * n_O3 * n_1Sg
                                 + q[8] * k4 * n_1D * n_CO2
                                 + q[9] * k5 * n_O3 * n_3Su
                                 + q[10] * k6 * n_1Dg * n_O3) / (P->chem_gamma - 1.0);
      }
  free(nv_hnu);
  return 0;
}

/* ---------------------------------------------------------------------- RHS */
/* TimeRHSFunctionExplicit (TimeRHSFunctionExplicit.c:29-77) */
int orc_rhs(const orc_params* P, double* rhs, double* u, const double* dxinv, const double* imap,
            double t) {
  long n = orc_npoints_ghosted(P) * P->nvars, i;
  double* tmp = (double*)calloc(n, sizeof(double));
  int ret;
  orc_apply_bc(P, u);
  memset(rhs, 0, sizeof(double) * n);
  ret = orc_hyperbolic(P, tmp, u, dxinv);
  for (i = 0; i < n; i++) rhs[i] += -1.0 * tmp[i];
  if (P->model == ORC_NS2D) {
    orc_parabolic(P, tmp, u, dxinv);
    for (i = 0; i < n; i++) rhs[i] += 1.0 * tmp[i];
  }
  orc_source(P, tmp, u, imap, t);
  for (i = 0; i < n; i++) rhs[i] += 1.0 * tmp[i];
  free(tmp);
  return ret;
}

/* --------------------------------------------------------------------- RK */
/* TimePreStep (BC on u, TimePreStep.c:36-41) + TimeRK (TimeRK.c:34-102) */
int orc_run(const orc_params* P, double* u, const double* dxinv, const double* imap, double t0,
            int nsteps) {
  long n = orc_npoints_ghosted(P) * P->nvars, i;
  int ns = P->nstages, s, j, it, ret = 0;
  double** U = (double**)calloc(ns, sizeof(double*));
  double** Ud = (double**)calloc(ns, sizeof(double*));
  double t = t0;
  for (s = 0; s < ns; s++) {
    U[s] = (double*)calloc(n, sizeof(double));
    Ud[s] = (double*)calloc(n, sizeof(double));
  }
  for (it = 0; it < nsteps; it++) {
    orc_apply_bc(P, u);
    for (s = 0; s < ns; s++) {
      double st = t + P->cst[s] * P->dt;
      memcpy(U[s], u, sizeof(double) * n);
      for (j = 0; j < s; j++) {
        double a = P->dt * P->A[s * ns + j];
        for (i = 0; i < n; i++) U[s][i] += a * Ud[j][i];
      }
      ret |= orc_rhs(P, Ud[s], U[s], dxinv, imap, st);
    }
    for (s = 0; s < ns; s++) {
      double b = P->dt * P->b[s];
      for (i = 0; i < n; i++) u[i] += b * Ud[s][i];
    }
    t += P->dt;
  }
  for (s = 0; s < ns; s++) { free(U[s]); free(Ud[s]); }
  free(U); free(Ud);
  return ret;
}

/* NavierStokes2DComputeCFL / Euler1DComputeCFL (max over interior points) */
double orc_cfl(const orc_params* P, const double* u, const double* dxinv) {
  int nv = P->nvars, i, j, jmax = P->ndims == 2 ? P->dim[1] : 1;
  double max_cfl = 0, dt = P->dt;
  for (j = 0; j < jmax; j++)
    for (i = 0; i < P->dim[0]; i++) {
      long p = PIX(P, i, j);
      if (P->model == ORC_NS2D) {
        double rho, vx, vy, e, Pp, c, dxi = dxinv[G + i], dyi = dxinv[(P->dim[0] + 2 * G) + G + j];
        double lx, ly;
        ns_flowvar(u + nv * p, P->gamma, &rho, &vx, &vy, &e, &Pp);
        c = sqrt(P->gamma * Pp / rho);
        lx = (absolute(vx) + c) * dt * dxi;
        ly = (absolute(vy) + c) * dt * dyi;
        if (lx > max_cfl) max_cfl = lx;
        if (ly > max_cfl) max_cfl = ly;
      } else {
        double rho, v, e, Pp, c, l;
        eu_flowvar(u + nv * p, P->gamma, &rho, &v, &e, &Pp);
        c = sqrt(P->gamma * Pp / rho);
        l = (absolute(v) + c) * dt * dxinv[G + i];
        if (l > max_cfl) max_cfl = l;
      }
    }
  return max_cfl;
}
