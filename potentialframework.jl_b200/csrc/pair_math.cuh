// pair_math.cuh — pair model parameters and the per-pair energy/gradient
// factor shared by the cell-list and the skin-list pair kernels.
//
// SmoothPair: E = A_ab q³, q = 1 - r²/c², dE/dr / r = -6 A q² / c²
// (PairPotentials/models.jl:45-70 BoundSmooth, :138-176 PreparedSmooth).
// Lennard-Jones, energy-shifted: E = 4ε[(σ/r)¹² - (σ/r)⁶] - shift,
// dE/dr / r = 24ε[(σ/r)⁶ - 2(σ/r)¹²] / r² (PairPotentials/lennard_jones.jl:10-17).
#pragma once
#include <cstdint>

#include "pfw_internal.h"

namespace pfw {

struct PairParams {
  int kind, nz;
  double A[16];  // SmoothPair amplitudes (nz <= 4)
  double invc2;
  double eps4, eps24, sigma2, shift;  // LJ
  int want_f, want_v, want_e;
  int n_owned;  // atoms [0, n_owned) (original order) own their E/W shares; the rest are ghost copies
};

// Energy and gradient factor g/d of one directed pair at squared distance r2;
// a is A[z_i][z_j] for SmoothPair (unused for LJ).
template <int KIND>
__device__ __forceinline__ void pair_term(const PairParams& prm, double a, double r2, double& en, double& coef) {
  if (KIND == 0) {
    const double q = 1.0 - r2 * prm.invc2;
    const double aq2 = a * q * q;
    en = aq2 * q;
    coef = -6.0 * aq2 * prm.invc2;
  } else {
    // 1/r² by two Newton steps y ← y(2 - r²y) from an FP32 seed (≈1 ulp)
    double ir2 = (double)__frcp_rn((float)r2);
    ir2 = fma(ir2, fma(-r2, ir2, 1.0), ir2);
    ir2 = fma(ir2, fma(-r2, ir2, 1.0), ir2);
    const double s2 = prm.sigma2 * ir2;
    const double s6 = s2 * s2 * s2;
    en = prm.eps4 * (s6 * s6 - s6) - prm.shift;
    coef = prm.eps24 * (s6 - 2.0 * s6 * s6) * ir2;
  }
}

PairParams make_pair_params(const pfw_ws* ws, uint32_t req);

}  // namespace pfw
