// noalloc.cu — pair evaluation that allocates no memory.
//
// Some callers cannot call cudaMalloc: hosts that own all device memory
// through their own pool allocator (a Julia or MD-engine runtime that hands
// out every byte itself), and code that must not trigger the device-wide
// synchronisation a fresh allocation can cause, for example while another
// component is recording work on the same device.  For them,
// pfw_pair_evaluate_noalloc evaluates SmoothPair or Lennard-Jones energy,
// forces and virial for a small system with every input and output supplied
// by the caller as device memory.  Its only scratch, the per-block energy
// and virial partial sums, lives in the file-scope array below, which every
// GPU that loads this library keeps for the lifetime of the process.
//
// The kernel is the brute-force variant of the pair kernel: every atom is
// compared with every other atom under the orthorhombic minimum image, with
// the reference's exact geometry (mod(x, L) wrap, d - round(d/L)·L, r² < c²;
// NeighbourList/storage.jl:160-163, geometry.jl:5-17), so its neighbour set
// equals the cell-list path's.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "pfw_common.cuh"
#include "pfw_internal.h"

namespace pfw {

constexpr int NOALLOC_BLOCK = 128;
constexpr int NOALLOC_MAX_BLOCKS = PFW_NOALLOC_MAX_ATOMS / NOALLOC_BLOCK;

// Scratch: 8 doubles (E, six virial components, pad) per block.  Every call
// overwrites every entry it later reads, so nothing needs clearing between
// calls; calls that overlap on the GPU race on this array.
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_BLOCKS * 8];

struct NoallocParams {
  int kind, nz, n;
  double A[16];
  double invc2, eps4, eps24, sigma2, shift;
  double L[3];
  int pbc[3];
  double c2;
  int want_f;
};

template <int KIND>
__global__ void __launch_bounds__(NOALLOC_BLOCK)
    k_pair_noalloc(NoallocParams p, const double* __restrict__ X, const int* __restrict__ species,
                   double* __restrict__ F, double* __restrict__ partials) {
  __shared__ double stage[NOALLOC_BLOCK][4];
  __shared__ double red[7][NOALLOC_BLOCK];
  const int i = blockIdx.x * NOALLOC_BLOCK + threadIdx.x;
  const bool have = i < p.n;
  double xi[3] = {0, 0, 0};
  int zi = 0;
  if (have) {
#pragma unroll
    for (int a = 0; a < 3; ++a) xi[a] = p.pbc[a] ? jl_mod(X[3 * i + a], p.L[a]) : X[3 * i + a];
    zi = min(max(species[i], 0), p.nz - 1);
  }
  double fx = 0, fy = 0, fz = 0, e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  for (int j0 = 0; j0 < p.n; j0 += NOALLOC_BLOCK) {
    __syncthreads();
    const int jj = j0 + threadIdx.x;
    if (jj < p.n) {
#pragma unroll
      for (int a = 0; a < 3; ++a) stage[threadIdx.x][a] = p.pbc[a] ? jl_mod(X[3 * jj + a], p.L[a]) : X[3 * jj + a];
      stage[threadIdx.x][3] = (double)min(max(species[jj], 0), p.nz - 1);
    }
    __syncthreads();
    if (!have) continue;
    const int nj = min(NOALLOC_BLOCK, p.n - j0);
    for (int t = 0; t < nj; ++t) {
      if (j0 + t == i) continue;
      double d[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double dd = xsub(stage[t][a], xi[a]);
        d[a] = p.pbc[a] ? xsub(dd, xmul(rint(xdiv(dd, p.L[a])), p.L[a])) : dd;
      }
      const double r2 = xr2(d[0], d[1], d[2]);
      if (!(r2 < p.c2)) continue;
      double en, coef;
      if (KIND == 0) {
        const double a = p.A[zi * p.nz + (int)stage[t][3]];
        const double q = 1.0 - r2 * p.invc2;
        en = a * q * q * q;
        coef = -6.0 * a * q * q * p.invc2;
      } else {
        const double ir2 = 1.0 / r2;
        const double s2 = p.sigma2 * ir2, s6 = s2 * s2 * s2;
        en = p.eps4 * (s6 * s6 - s6) - p.shift;
        coef = p.eps24 * (s6 - 2.0 * s6 * s6) * ir2;
      }
      const double gx = coef * d[0], gy = coef * d[1], gz = coef * d[2];
      fx += gx; fy += gy; fz += gz;
      e += en;
      w[0] += d[0] * gx; w[1] += d[1] * gy; w[2] += d[2] * gz;
      w[3] += d[0] * gy; w[4] += d[0] * gz; w[5] += d[1] * gz;
    }
  }
  if (have && p.want_f) {
    F[3 * i] = fx;
    F[3 * i + 1] = fy;
    F[3 * i + 2] = fz;
  }
  // each directed pair is seen from both ends: half of E and W per side
  red[0][threadIdx.x] = 0.5 * e;
#pragma unroll
  for (int k = 0; k < 6; ++k) red[k + 1][threadIdx.x] = -0.5 * w[k];
  __syncthreads();
  for (int s = NOALLOC_BLOCK / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
#pragma unroll
      for (int k = 0; k < 7; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 8) partials[8 * blockIdx.x + threadIdx.x] = threadIdx.x < 7 ? red[threadIdx.x][0] : 0.0;
}

__global__ void k_reduce_noalloc(int nblocks, const double* __restrict__ partials, double* __restrict__ E,
                                 double* __restrict__ W) {
  if (threadIdx.x != 0) return;
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nblocks; ++b)
#pragma unroll
    for (int k = 0; k < 7; ++k) s[k] += partials[8 * b + k];
  if (E) E[0] = s[0];
  if (W) {
    W[0] = s[1]; W[4] = s[2]; W[8] = s[3];
    W[1] = W[3] = s[4];
    W[2] = W[6] = s[5];
    W[5] = W[7] = s[6];
  }
}

// Device address of the scratch array, looked up once per device with that
// device current (a host-side reference to the array is only a stand-in).
static double* scratch_address(int device, cudaError_t* err) {
  constexpr int MAXDEV = 64;
  static std::mutex mu;
  static double* addr[MAXDEV] = {};
  if (device < 0 || device >= MAXDEV) {
    *err = cudaErrorInvalidDevice;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* ptr = nullptr;
    *err = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
    if (*err != cudaSuccess) return nullptr;
    addr[device] = static_cast<double*>(ptr);
  }
  *err = cudaSuccess;
  return addr[device];
}

}  // namespace pfw

extern "C" pfw_status pfw_pair_evaluate_noalloc(int32_t device, void* stream, int64_t n, const double* X_dev,
                                                const int32_t* species_dev, const double H[9], const uint8_t pbc[3],
                                                int32_t kind, int32_t nz, const double* params, double cutoff,
                                                uint32_t request, double* E_dev, double* F_dev, double* W_dev,
                                                char* errbuf, int32_t errlen) {
  auto fail = [&](pfw_status code, const char* msg) {
    if (errbuf && errlen > 0) {
      std::strncpy(errbuf, msg, (size_t)errlen - 1);
      errbuf[errlen - 1] = '\0';
    }
    return code;
  };
  if (errbuf && errlen > 0) errbuf[0] = '\0';
  if (n < 0 || n > PFW_NOALLOC_MAX_ATOMS) return fail(PFW_EINVAL, "pfw_pair_evaluate_noalloc: at most 8192 atoms");
  if (!H || !pbc || !params || (n > 0 && (!X_dev || !species_dev)))
    return fail(PFW_EINVAL, "pfw_pair_evaluate_noalloc: null argument");
  if (!(std::isfinite(cutoff) && cutoff > 0)) return fail(PFW_EINVAL, "cutoff must be finite and positive (Å)");
  pfw::NoallocParams p{};
  p.n = (int)n;
  p.kind = kind;
  p.c2 = cutoff * cutoff;
  p.want_f = (request & PFW_REQ_FORCES) != 0;
  for (int a = 0; a < 3; ++a) {
    p.pbc[a] = pbc[a] ? 1 : 0;
    p.L[a] = H[a + 3 * a];
    for (int b = 0; b < 3; ++b)
      if (a != b && H[a + 3 * b] != 0.0) return fail(PFW_EINVAL, "pfw_pair_evaluate_noalloc: orthorhombic cells only");
    if (p.pbc[a] && !(std::isfinite(p.L[a]) && p.L[a] > 2 * cutoff))
      return fail(PFW_EINVAL, "pfw_pair_evaluate_noalloc: every periodic length must exceed twice the cutoff");
  }
  if (kind == 0) {
    if (nz < 1 || nz > 4) return fail(PFW_EINVAL, "SmoothPair supports 1 to 4 species channels");
    for (int k = 0; k < nz * nz; ++k) p.A[k] = params[k];
    p.nz = nz;
    p.invc2 = 1.0 / (cutoff * cutoff);
  } else if (kind == 1) {
    const double eps = params[0], sigma = params[1];
    if (!(eps > 0 && sigma > 0 && std::isfinite(eps) && std::isfinite(sigma)))
      return fail(PFW_EINVAL, "LJ parameters must be positive and finite");
    p.nz = 1;
    p.eps4 = 4.0 * eps;
    p.eps24 = 24.0 * eps;
    p.sigma2 = sigma * sigma;
    const double rc = sigma / cutoff, qc2 = rc * rc, qc = qc2 * qc2 * qc2;
    p.shift = 4.0 * eps * (qc * qc - qc);
  } else {
    return fail(PFW_EINVAL, "kind must be 0 (SmoothPair) or 1 (Lennard-Jones)");
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(PFW_ECUDA, cudaGetErrorString(e));
  double* partials = pfw::scratch_address(device, &e);
  if (!partials) return fail(PFW_ECUDA, cudaGetErrorString(e));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int blocks = std::max(1, (int)((n + pfw::NOALLOC_BLOCK - 1) / pfw::NOALLOC_BLOCK));
  if (n > 0) {
    if (kind == 0)
      pfw::k_pair_noalloc<0><<<blocks, pfw::NOALLOC_BLOCK, 0, st>>>(p, X_dev, species_dev, F_dev, partials);
    else
      pfw::k_pair_noalloc<1><<<blocks, pfw::NOALLOC_BLOCK, 0, st>>>(p, X_dev, species_dev, F_dev, partials);
    pfw::k_reduce_noalloc<<<1, 32, 0, st>>>(blocks, partials, (request & PFW_REQ_ENERGY) ? E_dev : nullptr,
                                            (request & PFW_REQ_VIRIAL) ? W_dev : nullptr);
  } else {
    pfw::k_reduce_noalloc<<<1, 32, 0, st>>>(0, partials, (request & PFW_REQ_ENERGY) ? E_dev : nullptr,
                                            (request & PFW_REQ_VIRIAL) ? W_dev : nullptr);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PFW_ECUDA, cudaGetErrorString(e));
  return PFW_OK;
}
