// traverse.cuh — warp-per-home-cell traversal of all directed neighbours.
//
// Lanes are the home cell's atoms (chunks of 32).  The warp first resolves up
// to 32 stencil cell-images at once (one per lane: neighbour cell, image
// shift, atom range) and concatenates their atoms into one flat list.  That
// list is staged 32 atoms at a time in shared memory as packed FP32 pairs
// relative to the home cell's first atom (each atom's image shift applied in
// FP64 first), and each lane runs the candidate test on two neighbours per
// packed instruction (__ffma2_rn) against c²·(1 + 2⁻¹⁰).  Survivors are
// appended to the lane's own list; when any list could overflow, or at the
// end of a stencil block, the lists are drained: each lane walks its list,
// re-tests with the exact reference arithmetic
// (NeighbourList/geometry.jl:5-19) and calls visit for pairs with r² < c².
//
// Pair kernels (a staging ring of 64) test and drain differently.  The test
// is transposed: lanes hold the staged atoms, the warp walks the home atoms
// and a ballot appends each home atom's survivors at consecutive slots of its
// list (the zero-shift self pair is left to the drain).  The drain is a
// callable of traverse_lists: the pair kernels walk all lanes' lists as one
// sequence.  For both, the list is stored with the lane index xor-ed with the
// slot, so that 32 consecutive slots of ONE lane sit in 32 distinct banks,
// while one slot of all lanes still does.
//
// The FP32 test can only reject pairs whose exact r² exceeds c²: with
// coordinates relative to a point at most R away, |r²₃₂ - r²| ≤ c²·(4e-7·R/c
// + 2e-7), far inside the 2⁻¹⁰ guard for any R < 1000 c.  The visited set is
// therefore exactly the reference's.  The box prune is as safe: the box
// distance of the FP32 coordinates is at most their distance to any home
// atom, so a staged atom within c of a home atom has a box distance below
// c²·(1 + 2⁻¹⁰) by the same bound.  visit(i, j, pi, pj, se, d, r2) runs
// on the lane owning sorted atom i in a fixed order (stencil entry, then the
// neighbour cell's sorted order).
#pragma once
#include "pfw_common.cuh"

namespace pfw {

constexpr int TRAVERSE_STAGE = 32;
#ifndef PFW_LIST_K
#define PFW_LIST_K 64
#endif
constexpr int LIST_K = PFW_LIST_K;  // list capacity per lane (> TRAVERSE_STAGE)
constexpr int LIST_NE = 32;  // stencil entries per block (one per lane)
constexpr float PREFILTER_GUARD = 1.0f + 1.0f / 1024.0f;

#ifndef PFW_DRAIN_UNROLL
#define PFW_DRAIN_UNROLL 1
#endif

// Per-warp traversal state; K is the list capacity per lane (> TRAVERSE_STAGE).
// RING = 64 turns on the box prune (MODE 0): a staged atom farther than the
// cutoff from the bounding box of the home atoms cannot be a neighbour of any
// of them and is dropped before the per-lane test; the survivors are packed
// into a ring of 64 slots so that each per-lane test still sees 32 of them.
template <int K, int RING = TRAVERSE_STAGE>
struct WarpStageK {
  static constexpr int capacity = K;
  static constexpr int ring = RING;
  float2 x2[RING / 2], y2[RING / 2], z2[RING / 2];
  unsigned sitem[RING];             // staged atom: j | entry << 24
  int start[LIST_NE + 1];           // flat-list offsets of the entries
  StencilEntry ent[LIST_NE];
  unsigned int list[K * 32];        // list_slot(slot, lane): j | entry << 24
};
using WarpStage = WarpStageK<LIST_K>;

__device__ __forceinline__ int list_slot(int slot, int lane) { return slot * 32 + (lane ^ (slot & 31)); }

// Exact displacement of a listed candidate j from centre i: the stencil
// entry's shift added to the sorted coordinates' difference (MODE 0), or the
// cell's minimum-image / explicit-image rule (MODE 1).
template <int MODE>
__device__ __forceinline__ void candidate_displacement(const SysGeom& g, const StencilEntry& se, const double4& pi,
                                                       const double4& pj, double d[3]) {
  if (MODE == 0) {
    d[0] = xadd(xsub(pj.x, pi.x), se.sh[0]);
    d[1] = xadd(xsub(pj.y, pi.y), se.sh[1]);
    d[2] = xadd(xsub(pj.z, pi.z), se.sh[2]);
  } else {
    displacement(g, se, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, d);
  }
}

// Walk the lane's list: PFW_DRAIN_UNROLL neighbour loads are issued before
// any of them is used, so their latencies overlap.
template <int MODE, class Stage, class Visit>
__device__ __forceinline__ void drain_lists(const SysGeom& g, const double4* __restrict__ pos, Stage& stage,
                                            int lane, bool have, int i, const double4& pi, int& cnt, Visit& visit) {
  constexpr int U = PFW_DRAIN_UNROLL;
  __syncwarp();
  if (have) {
    for (int q0 = 0; q0 < cnt; q0 += U) {
      unsigned item[U];
      double4 pj[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        item[u] = stage.list[list_slot(min(q0 + u, cnt - 1), lane)];
        pj[u] = pos[item[u] & 0xFFFFFFu];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (q0 + u >= cnt) break;
        const int j = (int)(item[u] & 0xFFFFFFu);
        const StencilEntry& se = stage.ent[item[u] >> 24];
        double d[3];
        candidate_displacement<MODE>(g, se, pi, pj[u], d);
        const double r2 = xr2(d[0], d[1], d[2]);
        if (r2 < g.c2) visit(i, j, pi, pj[u], se, d, r2);
      }
    }
  }
  cnt = 0;
  __syncwarp();
}

// The prefilter of one home cell.  drain(have, i, pi, cnt) consumes the
// lanes' lists (and sets cnt to 0); chunk_end(have, i, pi) runs after each
// chunk of 32 home atoms.
template <int MODE, class Stage, class Drain, class ChunkEnd>
__device__ __forceinline__ void traverse_lists(const SysGeom& g, int cell, const int* __restrict__ cell_start,
                                               const double4* __restrict__ pos, Stage& stage, int lane,
                                               Drain&& drain, ChunkEnd&& chunk_end, int part = 0, int parts = 1) {
  const int b = cell_start[cell], e = cell_start[cell + 1];
  if (b == e) return;
  const int local = cell - g.cell_begin;
  const int key[3] = {local / (g.dims[1] * g.dims[2]), (local / g.dims[2]) % g.dims[1], local % g.dims[2]};
  const int cnt0 = stencil_count(g, 0), cnt1 = stencil_count(g, 1), cnt2 = stencil_count(g, 2);
  const int nall = cnt0 * cnt1 * cnt2;
  // stencil entries [k_first, nstencil) of this part (parts split the stencil in order)
  const int k_first = (int)((int64_t)part * nall / parts), nstencil = (int)((int64_t)(part + 1) * nall / parts);
  const float c2hi = (float)g.c2 * PREFILTER_GUARD;
  constexpr int RING = Stage::ring;
  constexpr bool PAIR = RING == 2 * TRAVERSE_STAGE;  // the pair kernels' staging
  constexpr bool PRUNE = MODE == 0 && PAIR;
  const double4 ref = pos[b];
  for (int i0 = b; i0 < e; i0 += 32) {
    const int i = i0 + lane;
    const bool have = i < e;
    const int nh = min(32, e - i0);  // home atoms of this chunk
    const double4 pi = have ? pos[i] : ref;
    const float2 nx = make_float2(-(float)(pi.x - ref.x), -(float)(pi.x - ref.x));
    const float2 ny = make_float2(-(float)(pi.y - ref.y), -(float)(pi.y - ref.y));
    const float2 nz = make_float2(-(float)(pi.z - ref.z), -(float)(pi.z - ref.z));
    // bounding box of the home atoms' FP32 coordinates (lanes without an atom
    // sit at ref, an atom of the home cell, so they only widen it)
    float3 box_lo = make_float3(-nx.x, -ny.x, -nz.x), box_hi = box_lo;
    if (PRUNE) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        box_lo.x = fminf(box_lo.x, __shfl_xor_sync(0xffffffffu, box_lo.x, o));
        box_lo.y = fminf(box_lo.y, __shfl_xor_sync(0xffffffffu, box_lo.y, o));
        box_lo.z = fminf(box_lo.z, __shfl_xor_sync(0xffffffffu, box_lo.z, o));
        box_hi.x = fmaxf(box_hi.x, __shfl_xor_sync(0xffffffffu, box_hi.x, o));
        box_hi.y = fmaxf(box_hi.y, __shfl_xor_sync(0xffffffffu, box_hi.y, o));
        box_hi.z = fmaxf(box_hi.z, __shfl_xor_sync(0xffffffffu, box_hi.z, o));
      }
    }
    int cnt = 0;
    for (int s0 = k_first; s0 < nstencil; s0 += LIST_NE) {
      // ---- resolve up to 32 stencil entries, one per lane ----
      __syncwarp();
      int len = 0, jb = 0;
      {
        const int k = s0 + lane;
        StencilEntry se;
        se.cell = -1;
        if (k < nstencil) {
          const int t0 = k / (cnt1 * cnt2), t1 = (k / cnt2) % cnt1, t2 = k % cnt2;
          const int off[3] = {stencil_offset(g, 0, t0), stencil_offset(g, 1, t1), stencil_offset(g, 2, t2)};
          stencil_entry(g, key, off, se);
          if (se.cell >= 0) {
            jb = cell_start[se.cell];
            len = cell_start[se.cell + 1] - jb;
          }
        }
        stage.ent[lane] = se;
      }
      int incl = len;  // inclusive warp scan of the entry lengths
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      stage.start[lane] = incl - len;
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      if (lane == 31) stage.start[32] = total;
      const int jb_lane = jb;
      __syncwarp();
      // ---- stage the flat list 32 atoms at a time ----
      // slots [rpos, wpos) of the ring hold staged atoms not yet tested;
      // rpos is a multiple of 32 whenever a test starts.
      int wpos = 0, rpos = 0;
      auto test_window = [&](int n) {
        const int base = rpos & (RING - 1);
        if (PAIR) {
          // transposed: lane t holds staged atom t; the warp walks the home
          // atoms two at a time and each ballot appends one home's survivors
          // at consecutive slots of its list (the self pair is left to the
          // drain, which sees the entry's owner)
          const bool mine = lane < n;
          const unsigned it = stage.sitem[base + (mine ? lane : 0)];
          float2 cx = make_float2(1e30f, 1e30f), cy = cx, cz = cx;
          if (MODE == 0 && mine) {
            const float x = reinterpret_cast<const float*>(stage.x2)[base + lane];
            const float y = reinterpret_cast<const float*>(stage.y2)[base + lane];
            const float z = reinterpret_cast<const float*>(stage.z2)[base + lane];
            cx = make_float2(x, x); cy = make_float2(y, y); cz = make_float2(z, z);
          }
          const unsigned below = (1u << lane) - 1u;
          for (int h = 0; h < nh; h += 2) {
            const int h1 = min(h + 1, 31);
            bool a = mine, b = mine && h + 1 < nh;
            if (MODE == 0) {
              const float2 hx = make_float2(__shfl_sync(0xffffffffu, nx.x, h), __shfl_sync(0xffffffffu, nx.x, h1));
              const float2 hy = make_float2(__shfl_sync(0xffffffffu, ny.x, h), __shfl_sync(0xffffffffu, ny.x, h1));
              const float2 hz = make_float2(__shfl_sync(0xffffffffu, nz.x, h), __shfl_sync(0xffffffffu, nz.x, h1));
              const float2 dx = __fadd2_rn(cx, hx), dy = __fadd2_rn(cy, hy), dz = __fadd2_rn(cz, hz);
              const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
              a = a && r2.x < c2hi;
              b = b && r2.y < c2hi;
            }
            const unsigned ma = __ballot_sync(0xffffffffu, a), mb = __ballot_sync(0xffffffffu, b);
            const int ca = __shfl_sync(0xffffffffu, cnt, h), cb = __shfl_sync(0xffffffffu, cnt, h1);
            if (a) stage.list[list_slot(ca + __popc(ma & below), h)] = it;
            if (b) stage.list[list_slot(cb + __popc(mb & below), h1)] = it;
            if (lane == h) cnt += __popc(ma);
            if (lane == h + 1) cnt += __popc(mb);
          }
          rpos += n;
          if (__reduce_max_sync(0xffffffffu, cnt) > Stage::capacity - TRAVERSE_STAGE) drain(have, i, pi, cnt);
          return;
        }
        unsigned mask;
        if (MODE == 0) {
          mask = 0u;
          const float2 lim = make_float2(c2hi, c2hi);
          const int npair = (n + 1) >> 1;
#pragma unroll 4
          for (int u = 0; u < npair; ++u) {
            const float2 dx = __fadd2_rn(stage.x2[(base >> 1) + u], nx);
            const float2 dy = __fadd2_rn(stage.y2[(base >> 1) + u], ny);
            const float2 dz = __fadd2_rn(stage.z2[(base >> 1) + u], nz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            mask |= ((r2.x < lim.x ? 1u : 0u) | (r2.y < lim.y ? 2u : 0u)) << (2 * u);
          }
          if (n < 32) mask &= (1u << n) - 1u;
        } else {
          mask = n == 32 ? 0xffffffffu : ((1u << n) - 1u);
        }
        if (!have) mask = 0u;
        while (mask) {
          const int t = __ffs(mask) - 1;
          mask &= mask - 1u;
          const unsigned it = stage.sitem[base + t];
          if ((int)(it & 0xFFFFFFu) == i && stage.ent[it >> 24].zero) continue;  // the zero-shift self pair
          stage.list[list_slot(cnt++, lane)] = it;
        }
        rpos += n;
        if (__reduce_max_sync(0xffffffffu, cnt) > Stage::capacity - TRAVERSE_STAGE) drain(have, i, pi, cnt);
      };
      for (int f0 = 0; f0 < total; f0 += TRAVERSE_STAGE) {
        const int nj = min(TRAVERSE_STAGE, total - f0);
        __syncwarp();
        {
          float px = 1e30f, py = 1e30f, pz = 1e30f;
          int jj = 0, kk = 0;
          if (lane < nj) {
            const int f = f0 + lane;
            int lo = 0, hi = 31;  // last entry with start <= f
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (stage.start[mid] <= f) lo = mid;
              else hi = mid - 1;
            }
            kk = lo;
          }
          // atom index of the flat position: entry kk's first atom + offset
          const int jbk = __shfl_sync(0xffffffffu, jb_lane, kk);
          bool keep = lane < nj;
          if (keep) {
            jj = jbk + (f0 + lane - stage.start[kk]);
            if (MODE == 0) {
              const double4 q = pos[jj];
              const StencilEntry& se = stage.ent[kk];
              px = (float)((q.x + se.sh[0]) - ref.x);
              py = (float)((q.y + se.sh[1]) - ref.y);
              pz = (float)((q.z + se.sh[2]) - ref.z);
              if (PRUNE) {
                const float ex = fmaxf(fmaxf(box_lo.x - px, px - box_hi.x), 0.f);
                const float ey = fmaxf(fmaxf(box_lo.y - py, py - box_hi.y), 0.f);
                const float ez = fmaxf(fmaxf(box_lo.z - pz, pz - box_hi.z), 0.f);
                keep = fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < c2hi;
              }
            }
          }
          const unsigned kb = __ballot_sync(0xffffffffu, keep);
          if (keep) {
            const int slot = (wpos + __popc(kb & ((1u << lane) - 1u))) & (RING - 1);
            if (MODE == 0) {
              reinterpret_cast<float*>(stage.x2)[slot] = px;
              reinterpret_cast<float*>(stage.y2)[slot] = py;
              reinterpret_cast<float*>(stage.z2)[slot] = pz;
            }
            stage.sitem[slot] = (unsigned)jj | ((unsigned)kk << 24);
          }
          wpos += __popc(kb);
        }
        __syncwarp();
        if (wpos - rpos >= TRAVERSE_STAGE) test_window(TRAVERSE_STAGE);
      }
      if (wpos > rpos) test_window(wpos - rpos);
      // entries are reused by the next block: drain what refers to them
      drain(have, i, pi, cnt);
    }
    chunk_end(have, i, pi);
  }
}

// Every directed neighbour of the home cell's atoms, visited on the lane that
// owns the centre: visit(i, j, pi, pj, se, d, r2).
template <int MODE, class Visit>
__device__ __forceinline__ void warp_traverse_cell(const SysGeom& g, int cell, const int* __restrict__ cell_start,
                                                   const double4* __restrict__ pos, WarpStage& stage, int lane,
                                                   Visit&& visit, int part = 0, int parts = 1) {
  traverse_lists<MODE>(
      g, cell, cell_start, pos, stage, lane,
      [&](bool have, int i, const double4& pi, int& cnt) {
        drain_lists<MODE>(g, pos, stage, lane, have, i, pi, cnt, visit);
      },
      [](bool, int, const double4&) {}, part, parts);
}

// Integer image of the directed pair i→j relative to the ORIGINAL
// coordinates: S = lattice + wind[i] - wind[j] (interface.jl:126-134).
// Minimum image takes lattice = -rint((x_j - x_i)/L) per periodic axis.
// With the per-cell wrap (fast_shift: at least 4 bins of width >= c, so
// L >= 4c) an in-range pair has x_j - x_i = d - s·L with |d| < c <= L/4 for
// its stencil entry's shift s, so that rint is -s with a margin of a quarter
// and the lattice is the entry's own s: no division.
__device__ __forceinline__ void pair_image(const SysGeom& g, const StencilEntry& se, const double4& pi,
                                           const double4& pj, const int* wi, const int* wj, int S[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int lattice;
    if (g.minimum_image && !g.fast_shift) {
      const double dd = xsub(a == 0 ? pj.x : a == 1 ? pj.y : pj.z, a == 0 ? pi.x : a == 1 ? pi.y : pi.z);
      lattice = g.pbc[a] ? -(int)rint(xdiv(dd, g.L[a])) : 0;
    } else {
      lattice = se.s[a];
    }
    S[a] = lattice + wi[a] - wj[a];
  }
}

}  // namespace pfw
