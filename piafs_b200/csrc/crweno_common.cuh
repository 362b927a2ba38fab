// Device helpers shared by the CRWENO5 line-solve kernels (crweno.cu,
// crweno_line.cu): the nonlinear CRWENO5 weights and the WENO5 boundary rows.
#pragma once
#include "common.cuh"

namespace piafs {

constexpr int WT_NOLIM = 4;   // no_limiting: optimal weights everywhere

// Nonlinear CRWENO5 weights (optimal weights 0.2, 0.5, 0.3) from the three
// smoothness indicators of one stencil; tau is the WENO-Z / Yamaleev-Carpenter
// reference indicator (interpolation.h:255-545).  The weights come back up
// to a common positive factor (the normalisation by their sum, a reciprocal
// and three products, is left out) except for the mapped weights, whose
// mapping needs them normalised: every coefficient of a compact row is linear
// in the weights, and the line solve scales each row to a unit diagonal, so
// the factor cancels.  In FP32 (mixed precision, cells relative to the line's
// first value) the products stay finite for cell values within about 1e4 of
// that reference.
template <int WT, typename R>
__device__ __forceinline__ void crw_weights(R b1, R b2, R b3, R tau, R eps, R& w1, R& w2, R& w3) {
  constexpr R c1 = R(0.2), c2 = R(0.5), c3 = R(0.3);
  if (WT == WT_NOLIM) {
    w1 = c1; w2 = c2; w3 = c3;
  } else if (WT == W_JS || WT == W_MAPPED) {
    // c_k/q_k / sum_m c_m/q_m with q = (beta + eps)^2, as c_k prod_{m!=k} q_m / sum
    const R s1 = b1 + eps, s2 = b2 + eps, s3 = b3 + eps;
    const R q1 = s1 * s1, q2 = s2 * s2, q3 = s3 * s3;
    const R a1 = c1 * q2 * q3, a2 = c2 * q1 * q3, a3 = c3 * q1 * q2;
    if (WT == W_JS) { w1 = a1; w2 = a2; w3 = a3; return; }
    const R inv = rcp_nr(a1 + a2 + a3);
    w1 = a1 * inv; w2 = a2 * inv; w3 = a3 * inv;
    if (WT == W_MAPPED) {   // Henrick-Aslam-Powers mapping
      const R x1 = w1, x2 = w2, x3 = w3;
      const R A1 = x1 * (c1 + c1 * c1 - R(3) * c1 * x1 + x1 * x1) * rcp_nr(c1 * c1 + x1 * (R(1) - R(2) * c1));
      const R A2 = x2 * (c2 + c2 * c2 - R(3) * c2 * x2 + x2 * x2) * rcp_nr(c2 * c2 + x2 * (R(1) - R(2) * c2));
      const R A3 = x3 * (c3 + c3 * c3 - R(3) * c3 * x3 + x3 * x3) * rcp_nr(c3 * c3 + x3 * (R(1) - R(2) * c3));
      const R inv2 = rcp_nr(A1 + A2 + A3);
      w1 = A1 * inv2; w2 = A2 * inv2; w3 = A3 * inv2;
    }
  } else {
    const R r1 = tau * rcp_nr(b1 + eps), r2 = tau * rcp_nr(b2 + eps), r3 = tau * rcp_nr(b3 + eps);
    w1 = c1 * (R(1) + r1 * r1); w2 = c2 * (R(1) + r2 * r2); w3 = c3 * (R(1) + r3 * r3);
  }
}

// WENO5 boundary-row value at interface i (optimal weights 0.1, 0.6, 0.3,
// Interp1PrimFifthOrderCRWENO.c:164-175 with the explicit WENO5 candidates)
__device__ __forceinline__ double crw_edge(const DevParams& P, const double* src, long long st, int i, int upw) {
  double m3, m2, m1, p1, p2;
  if (upw > 0) { m3 = src[(i - 3) * st]; m2 = src[(i - 2) * st]; m1 = src[(i - 1) * st]; p1 = src[i * st]; p2 = src[(i + 1) * st]; }
  else         { m3 = src[(i + 2) * st]; m2 = src[(i + 1) * st]; m1 = src[i * st]; p1 = src[(i - 1) * st]; p2 = src[(i - 2) * st]; }
  double w1, w2, w3;
  if (P.no_limiting) { w1 = 0.1; w2 = 0.6; w3 = 0.3; }
  else weno_weights(P.weno_type, 0.1, 0.6, 0.3, m3, m2, m1, p1, p2, P.eps, w1, w2, w3);
  return weno5_value(w1, w2, w3, m3, m2, m1, p1, p2);
}

// the same on values taken relative to `ref`, in FP32 (mixed precision)
__device__ __forceinline__ float crw_edge_f(const DevParams& P, const double* src, long long st, int i, int upw,
                                            double ref) {
  auto at = [&](int c) { return (float)(src[c * st] - ref); };
  float m3, m2, m1, p1, p2;
  if (upw > 0) { m3 = at(i - 3); m2 = at(i - 2); m1 = at(i - 1); p1 = at(i); p2 = at(i + 1); }
  else         { m3 = at(i + 2); m2 = at(i + 1); m1 = at(i); p1 = at(i - 1); p2 = at(i - 2); }
  float w1, w2, w3;
  if (P.no_limiting) { w1 = 0.1f; w2 = 0.6f; w3 = 0.3f; }
  else weno_weights(P.weno_type, 0.1f, 0.6f, 0.3f, m3, m2, m1, p1, p2, (float)P.eps, w1, w2, w3);
  return weno5_value(w1, w2, w3, m3, m2, m1, p1, p2);
}

}  // namespace piafs
