// Viscosity and photochemistry point functions shared by the
// single-simulation kernels (kernels.cu) and the batched stage kernel
// (batch.cu).
#pragma once
#include "common.cuh"

namespace piafs {

// Sutherland-type viscosity and conductivity of NavierStokes2DParabolicFunction
template <typename T>
__device__ __forceinline__ void visc_coeffs(const DevParams& P, T Temp, T& mu, T& kappa) {
  const T Td = Temp * (T)P.Tref, T0 = (T)P.T0;
  const T r15 = exp(T(1.5) * log(Td / T0));   // raiseto (math_ops.h:40)
  mu = r15 * (T0 + (T)P.TS) / (Td + (T)P.TS);
  kappa = r15 * (T0 + (T)P.TA * exp(-(T)P.TB / T0)) / (Td + (T)P.TA * exp(-(T)P.TB / Td));
}

// _ChemistrySetRHS_ / _ChemistrySetQ_ (chemistry.h:30-137) of one layer in T:
// sources of O3, 1D, 1Dg, 3Su, 1Sg (src[0..4]) and the heating Q from the
// photon density and the layer's seven species densities.
template <typename T>
__device__ __forceinline__ void chem_layer(const DevParams& P, T n_hnu, T nO2, T nO3, T n1D, T n1Dg, T n3Su, T n1Sg,
                                           T nCO2, T* src, T& Q) {
  const T k0a = (T)P.k[0], k0b = (T)P.k[1], k1a = (T)P.k[2], k1b = (T)P.k[3], k2a = (T)P.k[4], k2b = (T)P.k[5];
  const T k3a = (T)P.k[6], k3b = (T)P.k[7], k4 = (T)P.k[8], k5 = (T)P.k[9], k6 = (T)P.k[10];
  src[0] = -(k0a + k0b) * n_hnu * nO3 - (k2a + k2b) * nO3 * n1D - (k3a + k3b) * nO3 * n1Sg
           - k5 * nO3 * n3Su - k6 * n1Dg * nO3;
  src[1] = k0a * n_hnu * nO3 - (k1a + k1b) * n1D * nO2 - (k2a + k2b) * n1D * nO3 - k4 * n1D * nCO2;
  src[2] = k0a * n_hnu * nO3 + k5 * nO3 * n3Su - k6 * n1Dg * nO3;
  src[3] = k2a * nO3 * n1D - k5 * nO3 * n3Su;
  src[4] = k1a * n1D * nO2 - (k3a + k3b) * nO3 * n1Sg;
  Q = (((T)P.q[0] * k0a + (T)P.q[1] * k0b) * n_hnu * nO3 + ((T)P.q[2] * k1a + (T)P.q[3] * k1b) * nO2 * n1D
       + ((T)P.q[4] * k2a + (T)P.q[5] * k2b) * nO3 * n1D + ((T)P.q[6] * k3a + (T)P.q[7] * k3b) * nO3 * n1Sg
       + (T)P.q[8] * k4 * n1D * nCO2 + (T)P.q[9] * k5 * nO3 * n3Su + (T)P.q[10] * k6 * n1Dg * nO3)
      / ((T)P.chem_gamma - T(1));
}

// photon density of the first layer (ChemistrySetPhotonDensity)
template <typename T>
__device__ __forceinline__ T chem_hnu0(const DevParams& P, double hnu_factor, double imap_p) {
  return (T)(hnu_factor * imap_p / (P.ch_c * P.ch_h * P.ch_nu * P.n_O2));
}

// ChemistrySetPhotonDensity (ChemistrySolve.c:18-65) + _ChemistrySetRHS_ /
// _ChemistrySetQ_ (chemistry.h:30-137) at point p, arithmetic in T, added to
// the FP64 rhs; the energy slot takes the heating of the last layer.  With
// hnu set, the photon density of layer iz is also stored at hnu[iz * ps + p]
// (the reference keeps it in Chemistry::nv_hnu for the species output).
template <typename T>
__device__ void chem_source_point(const DevParams& P, const double* __restrict__ U, long long p,
                                  double hnu_factor, double imap_p, double* __restrict__ rhs,
                                  double* __restrict__ hnu = nullptr) {
  const long long ps = P.ps;
  T n_hnu = chem_hnu0<T>(P, hnu_factor, imap_p);
  T Q = T(0);
  for (int iz = 0; iz < P.nz; iz++) {
    if (iz > 0) {
      const T damp = T(1) - (T)P.dz * (T)(P.sO3 * P.n_O2) * (T)U[(P.nflow + P.zstride * (iz - 1) + 1) * ps + p];
      n_hnu = n_hnu * damp;
    }
    if (hnu) hnu[iz * ps + p] = (double)n_hnu;
    const int nfv = P.nflow + P.zstride * iz;
    T src[5];
    chem_layer<T>(P, n_hnu, (T)U[(nfv + 0) * ps + p], (T)U[(nfv + 1) * ps + p], (T)U[(nfv + 2) * ps + p],
                  (T)U[(nfv + 3) * ps + p], (T)U[(nfv + 4) * ps + p], (T)U[(nfv + 5) * ps + p],
                  (T)U[(nfv + 6) * ps + p], src, Q);
#pragma unroll
    for (int k = 0; k < 5; k++) rhs[(nfv + 1 + k) * ps + p] += (double)src[k];
  }
  rhs[(P.nflow - 1) * ps + p] += (double)Q;
}

// pulse factor I0 exp(-(t - (t_start+t_pulse))^2 / (2 sigma^2)) or 0 before t_start
__device__ __forceinline__ double pulse_factor(const DevParams& P, double t) {
  if (!(t > P.t_start_norm)) return 0.0;
  const double sigma = P.t_pulse_norm / 2.35482;
  const double tp = t - (P.t_start_norm + P.t_pulse_norm);
  return P.I0 * exp(-(tp * tp) / (2 * sigma * sigma));
}

}  // namespace piafs
