// reduce.cu — deterministic two-stage column sums of per-cell / per-site
// partials into the energy and the 3×3 virial (the host-side sums of
// PairPotentials/evaluation.jl:8-25 and execute_sites!, execution.jl:153-167).
//
// Stage 1: each block Kahan-sums one contiguous chunk of the partials (every
// thread a strided subset, then a fixed tree), so the memory latency of the
// strided partial rows is spread over many SMs.  Stage 2: one block sums the
// block results in block order and writes E and W.  The order of every
// addition is fixed by the launch shape, so results are bitwise repeatable.
#include <algorithm>

#include "pfw_internal.h"

namespace pfw {

constexpr int RED_BLOCK = 256;
constexpr int RED_MAXCOLS = 10;

template <int NC>
__device__ __forceinline__ void block_tree(double (&sh)[RED_MAXCOLS][RED_BLOCK], const Kahan (&acc)[NC]) {
#pragma unroll
  for (int k = 0; k < NC; ++k) sh[k][threadIdx.x] = acc[k].s - acc[k].c;
  __syncthreads();
  for (int h = RED_BLOCK / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
#pragma unroll
      for (int k = 0; k < NC; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + h];
    __syncthreads();
  }
}

template <int NC>
__global__ void __launch_bounds__(RED_BLOCK)
    k_colsum_blocks(const double* __restrict__ parts, int nparts, int stride, int chunk, double* __restrict__ partial) {
  __shared__ double sh[RED_MAXCOLS][RED_BLOCK];
  const int p0 = blockIdx.x * chunk, p1 = min(p0 + chunk, nparts);
  Kahan acc[NC];
  for (int p = p0 + threadIdx.x; p < p1; p += RED_BLOCK)
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k].add(parts[(size_t)stride * p + k]);
  block_tree<NC>(sh, acc);
  if (threadIdx.x < NC) partial[NC * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// layout 0: pair partials (E, xx, yy, zz, xy, xz, yz) → symmetric W;
// layout 1: site partials (E, W column-major).
template <int NC>
__global__ void __launch_bounds__(RED_BLOCK)
    k_colsum_final(const double* __restrict__ partial, int nblocks, double* __restrict__ E, double* __restrict__ W) {
  __shared__ double sh[RED_MAXCOLS][RED_BLOCK];
  Kahan acc[NC];
  for (int b = threadIdx.x; b < nblocks; b += RED_BLOCK)
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k].add(partial[NC * b + k]);
  block_tree<NC>(sh, acc);
  if (threadIdx.x != 0) return;
  if (E) E[0] = sh[0][0];
  if (!W) return;
  if (NC == 7) {
    W[0] = sh[1][0];
    W[4] = sh[2][0];
    W[8] = sh[3][0];
    W[3] = W[1] = sh[4][0];
    W[6] = W[2] = sh[5][0];
    W[7] = W[5] = sh[6][0];
  } else {
    for (int k = 0; k < 9; ++k) W[k] = sh[k + 1][0];
  }
}

template <int NC>
static void reduce_columns(pfw_ws* ws, const double* parts, int nparts, int stride, double* E, double* W) {
  int sms = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws->opt.device));
  const int nblocks = std::max(1, std::min(2 * sms, (nparts + RED_BLOCK - 1) / RED_BLOCK));
  const int chunk = std::max(1, (nparts + nblocks - 1) / nblocks);
  double* partial = static_cast<double*>(ws->red_partial.ensure(sizeof(double) * NC * nblocks));
  k_colsum_blocks<NC><<<nblocks, RED_BLOCK, 0, ws->stream>>>(parts, nparts, stride, chunk, partial);
  k_colsum_final<NC><<<1, RED_BLOCK, 0, ws->stream>>>(partial, nblocks, E, W);
  ws->launches += 2;
}

void reduce_pair_parts(pfw_ws* ws, const double* parts, int nparts, int stride, double* E, double* W) {
  reduce_columns<7>(ws, parts, nparts, stride, E, W);
}

void reduce_site_parts(pfw_ws* ws, const double* parts, int nparts, double* E, double* W) {
  reduce_columns<10>(ws, parts, nparts, 10, E, W);
}

}  // namespace pfw
