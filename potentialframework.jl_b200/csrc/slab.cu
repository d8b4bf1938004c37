// slab.cu — the device half of a slab decomposition's per-step exchange.
//
// The reference is single-process (README.md:327).  One periodic box split
// into slabs along one cell axis needs, every step, each rank's atoms within
// the halo of its two faces: they become the neighbouring ranks' ghosts.
// k_slab_flags marks the two bands, the library's exclusive scan orders them
// (stable: owned order), and k_slab_scatter writes each band as
// (x, y, z, species) with the Cartesian image shift the receiving rank needs.
#include <algorithm>
#include <cmath>

#include "pfw_internal.h"

namespace pfw {

__global__ void k_slab_flags(int n, const double* __restrict__ X, double r0, double r1, double r2, double blo,
                             double bhi, int* __restrict__ flo, int* __restrict__ fhi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double f = fma(r2, X[3 * i + 2], fma(r1, X[3 * i + 1], r0 * X[3 * i]));
  flo[i] = f < blo ? 1 : 0;
  fhi[i] = f >= bhi ? 1 : 0;
}

__global__ void k_slab_scatter(int n, const double* __restrict__ X, const int* __restrict__ species,
                               const int* __restrict__ flo, const int* __restrict__ olo, const int* __restrict__ fhi,
                               const int* __restrict__ ohi, double3 slo, double3 shi, double4* __restrict__ lower,
                               double4* __restrict__ upper, int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    counts[0] = olo[n];
    counts[1] = ohi[n];
  }
  if (i >= n) return;
  const double x = X[3 * i], y = X[3 * i + 1], z = X[3 * i + 2], w = (double)species[i];
  if (flo[i]) lower[olo[i]] = make_double4(x + slo.x, y + slo.y, z + slo.z, w);
  if (fhi[i]) upper[ohi[i]] = make_double4(x + shi.x, y + shi.y, z + shi.z, w);
}

void slab_bands(pfw_ws* ws, int64_t n64, const double* X, const int32_t* species, const double fr[3], double lo,
                double hi, double d, const double sl[3], const double su[3], double* lower, double* upper,
                int32_t* counts) {
  if (n64 < 0 || n64 > (int64_t)INT32_MAX / 4) throw Error(PFW_EINVAL, "atom count out of range");
  if (!counts) throw Error(PFW_EINVAL, "counts buffer required");
  if (!(std::isfinite(lo) && std::isfinite(hi) && std::isfinite(d) && d >= 0 && lo <= hi))
    throw Error(PFW_EINVAL, "slab bounds must be finite with lo <= hi and d >= 0");
  for (int k = 0; k < 3; ++k)
    if (!(std::isfinite(fr[k]) && std::isfinite(sl[k]) && std::isfinite(su[k])))
      throw Error(PFW_EINVAL, "slab axis row and shifts must be finite");
  const int n = (int)n64;
  if (n > 0 && (!X || !species || !lower || !upper)) throw Error(PFW_EINVAL, "positions, species and bands required");
  int* buf = static_cast<int*>(ws->slab_scratch.ensure(sizeof(int) * (4 * (size_t)n + 2)));
  int *flo = buf, *fhi = buf + n, *olo = buf + 2 * n, *ohi = buf + 3 * n + 1;
  cudaStream_t st = ws->stream;
  if (n > 0) {
    k_slab_flags<<<grid_for(n, 256), 256, 0, st>>>(n, X, fr[0], fr[1], fr[2], lo + d, hi - d, flo, fhi);
    ws->launches += 1;
  }
  exclusive_scan_i32(ws, flo, olo, n);
  exclusive_scan_i32(ws, fhi, ohi, n);
  k_slab_scatter<<<grid_for(std::max(n, 1), 256), 256, 0, st>>>(
      n, X, species, flo, olo, fhi, ohi, make_double3(sl[0], sl[1], sl[2]), make_double3(su[0], su[1], su[2]),
      reinterpret_cast<double4*>(lower), reinterpret_cast<double4*>(upper), counts);
  ws->launches += 1;
  PFW_CUDA(cudaGetLastError());
}

}  // namespace pfw
