// snapshot.cu — materialised directed neighbour snapshot
// (neighbour_list/materialize/visit_directed_images!, NeighbourList/interface.jl:85-143).
//
// Count pass (entries per centre), exclusive scan into original-order CSR
// offsets, fill pass writing (j, S, R) for each centre in traversal order.
// Every entry is emitted by its own centre's lane, so the two directions of
// an unordered pair are produced by different lanes with no shared writes.
#include <algorithm>

#include "pfw_internal.h"
#include "traverse.cuh"

namespace pfw {

constexpr int NB_WARPS = 4;

template <int MODE>
__global__ void __launch_bounds__(NB_WARPS * 32)
    k_nb_count(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
               const double4* __restrict__ pos, const int* __restrict__ perm, int ncells, int* __restrict__ count) {
  __shared__ WarpStage stage[NB_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * NB_WARPS + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  // each atom is visited by one lane within one contiguous chunk pass
  int cur_i = -1, cnt = 0;
  warp_traverse_cell<MODE>(g, cell, cell_start, pos, stage[warp], lane,
                           [&](int i, int, const double4&, const double4&, const StencilEntry&, const double*, double) {
                             if (i != cur_i) {
                               if (cur_i >= 0) count[perm[cur_i]] = cnt;
                               cur_i = i;
                               cnt = 0;
                             }
                             ++cnt;
                           });
  if (cur_i >= 0) count[perm[cur_i]] = cnt;
}

template <int MODE>
__global__ void __launch_bounds__(NB_WARPS * 32)
    k_nb_fill(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
              const double4* __restrict__ pos, const int* __restrict__ perm, const int* __restrict__ wind, int ncells,
              const int64_t* __restrict__ offsets, int* __restrict__ jout, int* __restrict__ Sout,
              double* __restrict__ Rout) {
  __shared__ WarpStage stage[NB_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * NB_WARPS + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  int cur_i = -1;
  int64_t o = 0;
  int wi[3] = {0, 0, 0};
  warp_traverse_cell<MODE>(g, cell, cell_start, pos, stage[warp], lane,
                           [&](int i, int j, const double4& pi, const double4& pj, const StencilEntry& se,
                               const double* d, double) {
                             const int a = perm[i], bb = perm[j];
                             if (i != cur_i) {
                               cur_i = i;
                               o = offsets[a];
                               wi[0] = wind[3 * a]; wi[1] = wind[3 * a + 1]; wi[2] = wind[3 * a + 2];
                             }
                             const int wj[3] = {wind[3 * bb], wind[3 * bb + 1], wind[3 * bb + 2]};
                             int S[3];
                             pair_image(g, se, pi, pj, wi, wj, S);
                             if (jout) jout[o] = bb;
                             if (Sout) {
                               Sout[3 * o] = S[0]; Sout[3 * o + 1] = S[1]; Sout[3 * o + 2] = S[2];
                             }
                             if (Rout) {
                               Rout[3 * o] = d[0]; Rout[3 * o + 1] = d[1]; Rout[3 * o + 2] = d[2];
                             }
                             ++o;
                           });
}

static bool all_shift_mode(const Prepared& P) {
  for (auto& g : P.sys)
    if (g.minimum_image && !g.fast_shift) return false;
  return true;
}

int64_t neighbour_build(pfw_ws* ws, double cutoff, bool with_R) {
  ws->prep.valid = false;
  prepare(ws, cutoff);
  const Prepared& P = ws->prep;
  cudaStream_t st = ws->stream;
  const int n = P.n;
  int* count = static_cast<int*>(ws->nb_count.ensure(sizeof(int) * std::max(n, 1)));
  int64_t* offsets = static_cast<int64_t*>(ws->nb_offsets.ensure(sizeof(int64_t) * (n + 1)));
  PFW_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * std::max(n, 1), st));
  const bool shift = all_shift_mode(P);
  dim3 grid(grid_for(P.ncells, NB_WARPS)), block(NB_WARPS * 32);
  if (P.ncells > 0) {
    if (shift)
      k_nb_count<0><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                            ws->pos.as<double4>(), ws->perm.as<int>(), P.ncells, count);
    else
      k_nb_count<1><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                            ws->pos.as<double4>(), ws->perm.as<int>(), P.ncells, count);
    ws->launches += 1;
  }
  exclusive_scan_i64(ws, count, offsets, n);
  int64_t total = 0;
  PFW_CUDA(cudaMemcpyAsync(&total, offsets + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaStreamSynchronize(st));
  int* jd = static_cast<int*>(ws->nb_j.ensure(sizeof(int) * std::max<int64_t>(total, 1)));
  int* Sd = static_cast<int*>(ws->nb_S.ensure(sizeof(int) * 3 * std::max<int64_t>(total, 1)));
  double* Rd = with_R ? static_cast<double*>(ws->nb_R.ensure(sizeof(double) * 3 * std::max<int64_t>(total, 1)))
                      : nullptr;
  if (P.ncells > 0 && total > 0) {
    if (shift)
      k_nb_fill<0><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                           ws->pos.as<double4>(), ws->perm.as<int>(), ws->wind.as<int>(), P.ncells,
                                           offsets, jd, Sd, Rd);
    else
      k_nb_fill<1><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                           ws->pos.as<double4>(), ws->perm.as<int>(), ws->wind.as<int>(), P.ncells,
                                           offsets, jd, Sd, Rd);
    ws->launches += 1;
  }
  PFW_CUDA(cudaGetLastError());
  ws->nb_total = total;
  return total;
}

void neighbour_fill(pfw_ws* ws, int64_t* offsets, int32_t* j, int32_t* S, double* R) {
  if (ws->nb_total < 0) throw Error(PFW_ESTATE, "call pfw_neighbour_count first");
  cudaStream_t st = ws->stream;
  const int64_t M = ws->nb_total;
  const int n = ws->prep.n;
  if (offsets)
    PFW_CUDA(cudaMemcpyAsync(offsets, ws->nb_offsets.ptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, st));
  if (j && M) PFW_CUDA(cudaMemcpyAsync(j, ws->nb_j.ptr, sizeof(int) * M, cudaMemcpyDeviceToHost, st));
  if (S && M) PFW_CUDA(cudaMemcpyAsync(S, ws->nb_S.ptr, sizeof(int) * 3 * M, cudaMemcpyDeviceToHost, st));
  if (R && M) PFW_CUDA(cudaMemcpyAsync(R, ws->nb_R.ptr, sizeof(double) * 3 * M, cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaStreamSynchronize(st));
}

}  // namespace pfw
