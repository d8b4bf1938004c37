// snapshot.cu — materialised directed neighbour snapshot
// (neighbour_list/materialize/visit_directed_images!, NeighbourList/interface.jl:85-143).
//
// Count pass (entries per centre), exclusive scan into original-order CSR
// offsets, fill pass writing (j, S, R) for each centre in traversal order.
// Every entry is selected by its own centre's lane and written to that
// centre's range only, so no two threads write the same entry.
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

// The fill traverses exactly as the count pass, so each centre's entries land
// in [offsets[a], offsets[a+1]).  At every drain each lane first keeps its
// in-range candidates, in visit order, at the front of its own list; then
// the warp writes the lanes' entries one lane after another, consecutive
// threads taking consecutive entries, so the j, S and R stores of a warp are
// contiguous instead of 32 scattered lists.  The displacement is recomputed
// by the writing thread with the same arithmetic, so R is bit-identical to
// the tested value.
template <int MODE>
__global__ void __launch_bounds__(NB_WARPS * 32)
    k_nb_fill(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
              const double4* __restrict__ pos, const int* __restrict__ perm, const int* __restrict__ wind, int ncells,
              const int64_t* __restrict__ offsets, int* __restrict__ jout, int* __restrict__ Sout,
              double* __restrict__ Rout) {
  __shared__ WarpStage stage[NB_WARPS];
  __shared__ double s_pi[NB_WARPS][3][32];  // each lane's centre, read by the writing warp
  __shared__ long long s_o[NB_WARPS][32];   // each lane's next output entry
  __shared__ int s_w[NB_WARPS][3][32];      // each lane's centre wrap count
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * NB_WARPS + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  WarpStage& sg = stage[warp];
  int cur_i = -1;
  int64_t o = 0;
  int wi[3] = {0, 0, 0};
  traverse_lists<MODE>(
      g, cell, cell_start, pos, sg, lane,
      [&](bool have, int i, const double4& pi, int& cnt) {
        __syncwarp();
        int np = 0;
        if (have) {
          if (i != cur_i) {
            cur_i = i;
            const int a = perm[i];
            o = offsets[a];
            wi[0] = wind[3 * a];
            wi[1] = wind[3 * a + 1];
            wi[2] = wind[3 * a + 2];
          }
          // compaction in place: slot np <= q was already read
          for (int q = 0; q < cnt; ++q) {
            const unsigned item = sg.list[list_slot(q, lane)];
            const double4 pj = pos[item & 0xFFFFFFu];
            double d[3];
            candidate_displacement<MODE>(g, sg.ent[item >> 24], pi, pj, d);
            if (xr2(d[0], d[1], d[2]) < g.c2) sg.list[list_slot(np++, lane)] = item;
          }
        }
        cnt = 0;
        s_pi[warp][0][lane] = pi.x;
        s_pi[warp][1][lane] = pi.y;
        s_pi[warp][2][lane] = pi.z;
        s_o[warp][lane] = o;
        s_w[warp][0][lane] = wi[0];
        s_w[warp][1][lane] = wi[1];
        s_w[warp][2][lane] = wi[2];
        __syncwarp();
        unsigned pending = __ballot_sync(0xffffffffu, np > 0);
        while (pending) {
          const int L = __ffs(pending) - 1;
          pending &= pending - 1;
          const int nL = __shfl_sync(0xffffffffu, np, L);
          const double4 piL = make_double4(s_pi[warp][0][L], s_pi[warp][1][L], s_pi[warp][2][L], 0.0);
          const int64_t oL = s_o[warp][L];
          const int wL[3] = {s_w[warp][0][L], s_w[warp][1][L], s_w[warp][2][L]};
          for (int t = lane; t < nL; t += 32) {
            const unsigned item = sg.list[list_slot(t, L)];
            const int j = (int)(item & 0xFFFFFFu);
            const StencilEntry& se = sg.ent[item >> 24];
            const double4 pj = pos[j];
            double d[3];
            candidate_displacement<MODE>(g, se, piL, pj, d);
            const int bb = perm[j];
            const int wj[3] = {wind[3 * bb], wind[3 * bb + 1], wind[3 * bb + 2]};
            int S[3];
            pair_image(g, se, piL, pj, wL, wj, S);
            const int64_t e = oL + t;
            if (jout) jout[e] = bb;
            if (Sout) {
              Sout[3 * e] = S[0]; Sout[3 * e + 1] = S[1]; Sout[3 * e + 2] = S[2];
            }
            if (Rout) {
              Rout[3 * e] = d[0]; Rout[3 * e + 1] = d[1]; Rout[3 * e + 2] = d[2];
            }
          }
        }
        o += np;
        __syncwarp();
      },
      [](bool, int, const double4&) {});
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
