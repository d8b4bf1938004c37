// traverse.cuh — warp-per-home-cell traversal of all directed neighbours.
//
// Lanes are the home cell's atoms (chunks of 32); each stencil cell-image is
// staged in shared memory and walked as a broadcast.  visit(i, j, se, d, r2)
// is called on the lane that owns sorted atom i for every j within the cutoff
// (j == i only for nonzero images), in a fixed order: stencil entry, then the
// neighbour cell's sorted order.  The displacement d is bit-identical to the
// reference's geometry_lanes (NeighbourList/geometry.jl:5-19).
#pragma once
#include "pfw_common.cuh"

namespace pfw {

constexpr int TRAVERSE_STAGE = 32;

template <int MODE, class Visit>
__device__ __forceinline__ void warp_traverse_cell(const SysGeom& g, int cell, const int* __restrict__ cell_start,
                                                   const double4* __restrict__ pos, double4* stage, int lane,
                                                   Visit&& visit) {
  const int b = cell_start[cell], e = cell_start[cell + 1];
  const int local = cell - g.cell_begin;
  const int key[3] = {local / (g.dims[1] * g.dims[2]), (local / g.dims[2]) % g.dims[1], local % g.dims[2]};
  const int cnt0 = stencil_count(g, 0), cnt1 = stencil_count(g, 1), cnt2 = stencil_count(g, 2);
  for (int i0 = b; i0 < e; i0 += 32) {
    const int i = i0 + lane;
    const bool have = i < e;
    const double4 pi = have ? pos[i] : make_double4(0, 0, 0, 0);
    for (int t0 = 0; t0 < cnt0; ++t0)
      for (int t1 = 0; t1 < cnt1; ++t1)
        for (int t2 = 0; t2 < cnt2; ++t2) {
          const int off[3] = {stencil_offset(g, 0, t0), stencil_offset(g, 1, t1), stencil_offset(g, 2, t2)};
          StencilEntry se;
          stencil_entry(g, key, off, se);
          if (se.cell < 0) continue;
          const int jb = cell_start[se.cell], je = cell_start[se.cell + 1];
          for (int j0 = jb; j0 < je; j0 += TRAVERSE_STAGE) {
            const int nj = min(TRAVERSE_STAGE, je - j0);
            __syncwarp();
            if (lane < nj) stage[lane] = pos[j0 + lane];
            __syncwarp();
            if (!have) continue;
            for (int t = 0; t < nj; ++t) {
              const double4 pj = stage[t];
              const int j = j0 + t;
              if (se.zero && j == i) continue;
              double d[3];
              if (MODE == 0) {
                d[0] = xadd(xsub(pj.x, pi.x), se.sh[0]);
                d[1] = xadd(xsub(pj.y, pi.y), se.sh[1]);
                d[2] = xadd(xsub(pj.z, pi.z), se.sh[2]);
              } else {
                displacement(g, se, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, d);
              }
              const double r2 = xr2(d[0], d[1], d[2]);
              if (r2 < g.c2) visit(i, j, pi, pj, se, d);
            }
          }
        }
  }
}

// Integer image of the directed pair i→j relative to the ORIGINAL
// coordinates: S = lattice + wind[i] - wind[j] (interface.jl:126-134).
__device__ __forceinline__ void pair_image(const SysGeom& g, const StencilEntry& se, const double4& pi,
                                           const double4& pj, const int* wi, const int* wj, int S[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int lattice;
    if (g.minimum_image) {
      const double dd = xsub(a == 0 ? pj.x : a == 1 ? pj.y : pj.z, a == 0 ? pi.x : a == 1 ? pi.y : pi.z);
      lattice = g.pbc[a] ? -(int)rint(xdiv(dd, g.L[a])) : 0;
    } else {
      lattice = se.s[a];
    }
    S[a] = lattice + wi[a] - wj[a];
  }
}

}  // namespace pfw
