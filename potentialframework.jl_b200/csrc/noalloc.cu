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
constexpr int NOALLOC_STATUS = NOALLOC_MAX_BLOCKS * 8;  // index of the status word (as 64-bit flags)

// Scratch: 8 doubles (E, six virial components, pad) per block, then one
// 64-bit word of input flags.  The partials are overwritten by every call
// before they are read; the flag word is cleared by the first kernel of every
// call.  Calls that overlap on the GPU race on this array.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_BLOCKS * 8 + 8];

// Input flags raised by the pair kernel (bits of the status word).
constexpr unsigned long long NOALLOC_BAD_SPECIES = 1ull, NOALLOC_BAD_POSITION = 2ull;

struct NoallocParams {
  int kind, nz, n;
  double A[16];
  double invc2, eps4, eps24, sigma2, shift;
  double L[3];
  int pbc[3];
  double c2;
  int want_f;
};

// A species channel outside [0, nz) or a non-finite position raises a flag
// in the status word (the channel is then read as 0, so no table is indexed
// out of range).
__device__ __forceinline__ int noalloc_species(const NoallocParams& p, int z, unsigned long long* status) {
  if (z < 0 || z >= p.nz) {
    atomicOr(status, NOALLOC_BAD_SPECIES);
    return 0;
  }
  return z;
}

template <int KIND>
__global__ void __launch_bounds__(NOALLOC_BLOCK)
    k_pair_noalloc(NoallocParams p, const double* __restrict__ X, const int* __restrict__ species,
                   double* __restrict__ F, double* __restrict__ partials, unsigned long long* __restrict__ status) {
  __shared__ double stage[NOALLOC_BLOCK][4];
  __shared__ double red[7][NOALLOC_BLOCK];
  const int i = blockIdx.x * NOALLOC_BLOCK + threadIdx.x;
  const bool have = i < p.n;
  double xi[3] = {0, 0, 0};
  int zi = 0;
  if (have) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double x = X[3 * i + a];
      if (!isfinite(x)) atomicOr(status, NOALLOC_BAD_POSITION);
      xi[a] = p.pbc[a] ? jl_mod(x, p.L[a]) : x;
    }
    zi = noalloc_species(p, species[i], status);
  }
  double fx = 0, fy = 0, fz = 0, e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  for (int j0 = 0; j0 < p.n; j0 += NOALLOC_BLOCK) {
    __syncthreads();
    const int jj = j0 + threadIdx.x;
    if (jj < p.n) {
#pragma unroll
      for (int a = 0; a < 3; ++a) stage[threadIdx.x][a] = p.pbc[a] ? jl_mod(X[3 * jj + a], p.L[a]) : X[3 * jj + a];
      stage[threadIdx.x][3] = (double)min(max(species[jj], 0), p.nz - 1);  // flagged on its own row
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

__global__ void k_noalloc_clear(unsigned long long* __restrict__ status) { *status = 0ull; }

// Totals of the block partials in block order, and the call's status: the
// input flags first (PFW_EINVAL), then a non-finite energy or virial
// (PFW_EDOMAIN, as the allocating entry point reports coincident atoms of a
// singular model).
__global__ void k_reduce_noalloc(int nblocks, const double* __restrict__ partials,
                                 const unsigned long long* __restrict__ flags, double* __restrict__ E,
                                 double* __restrict__ W, int32_t* __restrict__ status_out) {
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
  if (status_out) {
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 7; ++k) finite = finite && isfinite(s[k]);
    *status_out = *flags ? PFW_EINVAL : (finite ? PFW_OK : PFW_EDOMAIN);
  }
}

// Device address of the scratch array on the current device.  A host-side
// reference to the array is only a stand-in, so the address is looked up on
// every call (cheap once the module is loaded; no stale pointer survives a
// device reset).
static double* scratch_address(cudaError_t* err) {
  void* ptr = nullptr;
  *err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  return *err == cudaSuccess ? static_cast<double*>(ptr) : nullptr;
}

}  // namespace pfw

extern "C" pfw_status pfw_pair_evaluate_noalloc(int32_t device, void* stream, int64_t n, const double* X_dev,
                                                const int32_t* species_dev, const double H[9], const uint8_t pbc[3],
                                                int32_t kind, int32_t nz, const double* params, double cutoff,
                                                uint32_t request, double* E_dev, double* F_dev, double* W_dev,
                                                int32_t* status_dev, char* errbuf, int32_t errlen) {
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
  if ((request & PFW_REQ_FORCES) && n > 0 && !F_dev)
    return fail(PFW_EINVAL, "pfw_pair_evaluate_noalloc: forces requested without a force buffer");
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
    // the amplitude table must be finite and symmetric (PairPotentials/models.jl:39)
    for (int a = 0; a < nz; ++a)
      for (int b = 0; b < nz; ++b)
        if (!std::isfinite(params[a * nz + b]) || params[a * nz + b] != params[b * nz + a])
          return fail(PFW_EINVAL, "SmoothPair amplitudes must be finite and symmetric");
    for (int k = 0; k < nz * nz; ++k) p.A[k] = params[k];
    p.nz = nz;
    p.invc2 = 1.0 / (cutoff * cutoff);
  } else if (kind == 1) {
    const double eps = params[0], sigma = params[1];
    if (!(eps > 0 && sigma > 0 && std::isfinite(eps) && std::isfinite(sigma)))
      return fail(PFW_EINVAL, "LJ parameters must be positive and finite");
    p.nz = INT32_MAX;  // any nonnegative species channel
    p.eps4 = 4.0 * eps;
    p.eps24 = 24.0 * eps;
    p.sigma2 = sigma * sigma;
    const double rc = sigma / cutoff, qc2 = rc * rc, qc = qc2 * qc2 * qc2;
    p.shift = 4.0 * eps * (qc * qc - qc);
  } else {
    return fail(PFW_EINVAL, "kind must be 0 (SmoothPair) or 1 (Lennard-Jones)");
  }
  // the caller's current device is restored on every return below
  int caller_device = -1;
  cudaError_t e = cudaGetDevice(&caller_device);
  if (e != cudaSuccess) return fail(PFW_ECUDA, cudaGetErrorString(e));
  auto done = [&](pfw_status code, const char* msg) {
    cudaSetDevice(caller_device);
    return code == PFW_OK ? code : fail(code, msg);
  };
  if (device != caller_device) {
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return done(PFW_ECUDA, cudaGetErrorString(e));
  }
  double* scratch = pfw::scratch_address(&e);
  if (!scratch) return done(PFW_ECUDA, cudaGetErrorString(e));
  unsigned long long* flags = reinterpret_cast<unsigned long long*>(scratch + pfw::NOALLOC_STATUS);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int blocks = (int)((n + pfw::NOALLOC_BLOCK - 1) / pfw::NOALLOC_BLOCK);
  pfw::k_noalloc_clear<<<1, 1, 0, st>>>(flags);
  if (n > 0) {
    if (kind == 0)
      pfw::k_pair_noalloc<0><<<blocks, pfw::NOALLOC_BLOCK, 0, st>>>(p, X_dev, species_dev, F_dev, scratch, flags);
    else
      pfw::k_pair_noalloc<1><<<blocks, pfw::NOALLOC_BLOCK, 0, st>>>(p, X_dev, species_dev, F_dev, scratch, flags);
  }
  pfw::k_reduce_noalloc<<<1, 32, 0, st>>>(blocks, scratch, flags, (request & PFW_REQ_ENERGY) ? E_dev : nullptr,
                                          (request & PFW_REQ_VIRIAL) ? W_dev : nullptr, status_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) return done(PFW_ECUDA, cudaGetErrorString(e));
  return done(PFW_OK, "");
}
