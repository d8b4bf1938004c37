// traverse.cuh — warp-per-home-cell traversal of all directed neighbours.
//
// Lanes are the home cell's atoms (chunks of 32).  For each stencil
// cell-image the warp stages up to 32 neighbour atoms in shared memory twice:
// exact FP64 (double4 x,y,z,species) and FP32 coordinates relative to the
// home cell's first atom with the image shift already applied in FP64.
//
//   phase A (FP32 pipe)  every lane tests all staged atoms with r² computed in
//                        FP32 against c²·(1 + 2⁻¹⁰) and keeps a 32-bit mask;
//   phase B (FP64 pipe)  only masked candidates are re-tested with the exact
//                        reference arithmetic (NeighbourList/geometry.jl:5-19)
//                        and, when r² < c², visited.
//
// The FP32 test can only reject pairs whose exact r² exceeds c²: with
// coordinates relative to a point at most R away, |r²₃₂ - r²| ≤ c²·(4e-7·R/c
// + 2e-7), far inside the 2⁻¹⁰ guard for any R < 1000 c.  So the visited set
// is exactly the reference's.  visit(i, j, pi, pj, se, d) runs on the lane
// owning sorted atom i, in a fixed order (stencil entry, then the neighbour
// cell's sorted order).
#pragma once
#include "pfw_common.cuh"

namespace pfw {

// Compile-time tuning knobs (both variants are exact):
//   PFW_PREFILTER       1: FP32 guard-band prefilter before the exact test
//   PFW_PHASEA_DYNAMIC  1: prefilter loop bounded by the staged count
#ifndef PFW_PREFILTER
#define PFW_PREFILTER 1
#endif
#ifndef PFW_PHASEA_DYNAMIC
#define PFW_PHASEA_DYNAMIC 1
#endif

constexpr int TRAVERSE_STAGE = 32;
constexpr float PREFILTER_GUARD = 1.0f + 1.0f / 1024.0f;

struct WarpStage {
  double4 p64[TRAVERSE_STAGE];
  float4 p32[TRAVERSE_STAGE];
};

template <int MODE, class Visit>
__device__ __forceinline__ void warp_traverse_cell(const SysGeom& g, int cell, const int* __restrict__ cell_start,
                                                   const double4* __restrict__ pos, WarpStage& stage, int lane,
                                                   Visit&& visit) {
  const int b = cell_start[cell], e = cell_start[cell + 1];
  if (b == e) return;
  const int local = cell - g.cell_begin;
  const int key[3] = {local / (g.dims[1] * g.dims[2]), (local / g.dims[2]) % g.dims[1], local % g.dims[2]};
  const int cnt0 = stencil_count(g, 0), cnt1 = stencil_count(g, 1), cnt2 = stencil_count(g, 2);
  const double c2 = g.c2;
  const float c2hi = (float)c2 * PREFILTER_GUARD;
  const double4 ref = pos[b];
  for (int i0 = b; i0 < e; i0 += 32) {
    const int i = i0 + lane;
    const bool have = i < e;
    const double4 pi = have ? pos[i] : ref;
    const float xi = (float)(pi.x - ref.x), yi = (float)(pi.y - ref.y), zi = (float)(pi.z - ref.z);
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
            if (lane < nj) {
              const double4 q = pos[j0 + lane];
              stage.p64[lane] = q;
              if (MODE == 0)
                stage.p32[lane] = make_float4((float)((q.x + se.sh[0]) - ref.x), (float)((q.y + se.sh[1]) - ref.y),
                                              (float)((q.z + se.sh[2]) - ref.z), 0.f);
            } else if (MODE == 0) {
              stage.p32[lane] = make_float4(1e30f, 1e30f, 1e30f, 0.f);
            }
            __syncwarp();
            if (!have) continue;
            unsigned mask;
            if (MODE == 0 && PFW_PREFILTER) {
              mask = 0u;
#if PFW_PHASEA_DYNAMIC
#pragma unroll 4
              for (int t = 0; t < nj; ++t) {
#else
#pragma unroll
              for (int t = 0; t < TRAVERSE_STAGE; ++t) {
#endif
                const float4 q = stage.p32[t];
                const float dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                mask |= (r2 < c2hi ? 1u : 0u) << t;
              }
            } else {
              mask = nj == 32 ? 0xffffffffu : ((1u << nj) - 1u);
            }
            while (mask) {
              const int t = __ffs(mask) - 1;
              mask &= mask - 1u;
              const int j = j0 + t;
              if (se.zero && j == i) continue;
              const double4 pj = stage.p64[t];
              double d[3];
              if (MODE == 0) {
                d[0] = xadd(xsub(pj.x, pi.x), se.sh[0]);
                d[1] = xadd(xsub(pj.y, pi.y), se.sh[1]);
                d[2] = xadd(xsub(pj.z, pi.z), se.sh[2]);
              } else {
                displacement(g, se, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, d);
              }
              const double r2 = xr2(d[0], d[1], d[2]);
              if (r2 < c2) visit(i, j, pi, pj, se, d, r2);
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
