// pair.cu — SmoothPair / Lennard-Jones energy, force and virial.
//
// Replaces cell_task!/execute! (NeighbourList/execution.jl:173-238) with the
// pair callbacks of PairPotentials/models.jl:138-176 (PreparedSmooth) and
// lennard_jones.jl:5-33 (LennardJonesRadial).
//
// Decomposition: one warp owns one home cell and walks every directed
// neighbour of its atoms with the shared traversal (traverse.cuh: stencil
// entries resolved per lane, FP32x2 prefilter, per-lane candidate lists,
// exact FP64 re-test).  Each lane accumulates the force on ITS atom only
// (full directed list), so forces are written once, in place, with no racing
// scatter; E and W take half of every directed pair.  Per-cell partials (E, 6
// virial components) are reduced deterministically (reduce.cu).
#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <mutex>

#include "pfw_internal.h"
#include "pair_math.cuh"
#include "traverse.cuh"

namespace pfw {

constexpr int PAIR_WARPS = 4;  // warps (home cells) per CTA

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void write_cell_parts(double* cellpart, int cell, int lane, double e, const double w[6],
                                                 unsigned long long np, unsigned long long* npairs) {
  e = warp_sum(e);
  double ws[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) ws[k] = warp_sum(w[k]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) np += __shfl_xor_sync(0xffffffffu, np, o);
  if (lane == 0) {
    // every directed pair is seen from both ends: E and W take one half each
    double* cp = cellpart + 8 * (size_t)cell;
    cp[0] = 0.5 * e;
#pragma unroll
    for (int k = 0; k < 6; ++k) cp[1 + k] = -0.5 * ws[k];
    cp[7] = 0;
    if (np) atomicAdd(npairs, np);
  }
}

// 4 resident 4-warp blocks per SM: 128 registers/thread and 4 × 54 KB of
// traversal state (72 list slots per lane, the 64-slot pruned staging ring,
// the drain's partial sums) in dynamic shared memory.  Longer lists mean
// fewer drains: 72 slots measured faster than 60-68, and than 5 blocks with
// 40-56 slots.
#ifndef PFW_PAIR_MINBLOCKS
#define PFW_PAIR_MINBLOCKS 4
#endif
#ifndef PFW_PAIR_LIST_K
#define PFW_PAIR_LIST_K 72
#endif
using PairStage = WarpStageK<PFW_PAIR_LIST_K, 2 * TRAVERSE_STAGE>;

// Flat drain of the lanes' lists: the warp treats them as ONE owner-major
// sequence (lane 0's entries, then lane 1's, ...) and gives each lane a
// contiguous 1/32 of it, so every lane evaluates the same number of entries
// whatever the number of home atoms and the spread of the per-lane counts.
// A lane accumulates the gradient of its current owner in registers and, when
// the owner changes, stores that partial sum in slot (lane + owner) — unique,
// because along the sequence either the lane or the owner grows.  Each owner
// then adds the partials of the lanes its entries went to, in lane order: the
// result is deterministic.  Energy and virial accumulate on the lane that
// evaluated the entry (inside eval).
template <class T>
struct FlatScratch {
  T part[63][3];  // partial gradient sums, slot lane + owner
  int off[33];    // exclusive scan of the lanes' counts; off[32] = total
};

// eval(ph, ownh, pj, d, r2, hit, gx, gy, gz): the pair of home atom ph
// (owning its E/W share when ownh) and neighbour pj at exact squared distance
// r2; it returns the gradient g (force on ph += g), zero unless hit (r2 < c²),
// and accumulates E and W of hits.  It is evaluated without branches, so two
// entries of one owner run as independent instruction streams.
template <int MODE>
__device__ __forceinline__ double entry_geometry(const SysGeom& g, const StencilEntry& se, const double4& ph,
                                                 const double4& pj, double d[3]) {
  if (MODE == 0) {
    d[0] = xadd(xsub(pj.x, ph.x), se.sh[0]);
    d[1] = xadd(xsub(pj.y, ph.y), se.sh[1]);
    d[2] = xadd(xsub(pj.z, ph.z), se.sh[2]);
  } else {
    displacement(g, se, ph.x, ph.y, ph.z, pj.x, pj.y, pj.z, d);
  }
  return xr2(d[0], d[1], d[2]);
}

// tick() runs after every step of one or two entries.
template <int MODE, class T, class Eval, class Tick>
__device__ __forceinline__ void flat_drain(const SysGeom& g, const double4* __restrict__ pos,
                                           const PairStage& stage, FlatScratch<T>& fs, int lane, int i0,
                                           unsigned ownmask, int& cnt, T f[3], Eval&& eval, Tick&& tick) {
  constexpr unsigned FULL = 0xffffffffu;
  __syncwarp();
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  const int off = incl - cnt;
  const int total = __shfl_sync(FULL, incl, 31);
  fs.off[lane] = off;
  if (lane == 31) fs.off[32] = total;
  __syncwarp();
  const int R = (total + 31) >> 5;  // entries per lane
  int q = lane * R;
  const int qend = min(q + R, total);
  if (q < qend) {
    int h = 0;  // owner of q: last lane with off <= q
#pragma unroll
    for (int st = 16; st > 0; st >>= 1)
      if (fs.off[h + st] <= q) h += st;
    int hoff = fs.off[h], hend = fs.off[h + 1];
    double4 ph = pos[i0 + h];
    bool ownh = (ownmask >> h) & 1u;
    T px = 0, py = 0, pz = 0;
    while (q < qend) {
      if (q >= hend) {  // the next owner with entries
        fs.part[lane + h][0] = px; fs.part[lane + h][1] = py; fs.part[lane + h][2] = pz;
        px = py = pz = 0;
        do {
          ++h;
        } while (fs.off[h + 1] <= q);
        hoff = fs.off[h];
        hend = fs.off[h + 1];
        ph = pos[i0 + h];
        ownh = (ownmask >> h) & 1u;
      }
      // entries q and q + 1 when both are this owner's (else q twice, the copy masked)
      const bool two = q + 1 < min(qend, hend);
      const unsigned ia = stage.list[list_slot(q - hoff, h)];
      const unsigned ib = stage.list[list_slot(q - hoff + (two ? 1 : 0), h)];
      const double4 pa = pos[ia & 0xFFFFFFu], pb = pos[ib & 0xFFFFFFu];
      double da[3], db[3];
      const StencilEntry& ea = stage.ent[ia >> 24];
      const StencilEntry& eb = stage.ent[ib >> 24];
      const double r2a = entry_geometry<MODE>(g, ea, ph, pa, da);
      const double r2b = entry_geometry<MODE>(g, eb, ph, pb, db);
      // the zero-shift self pair is in the list (the prefilter does not see owners)
      const int ih = i0 + h;
      const bool hita = r2a < g.c2 && !((int)(ia & 0xFFFFFFu) == ih && ea.zero);
      const bool hitb = two && r2b < g.c2 && !((int)(ib & 0xFFFFFFu) == ih && eb.zero);
      T ax, ay, az, bx, by, bz;
      eval(ph, ownh, pa, da, r2a, hita, ax, ay, az);
      eval(ph, ownh, pb, db, r2b, hitb, bx, by, bz);
      px += ax; py += ay; pz += az;
      px += bx; py += by; pz += bz;
      q += two ? 2 : 1;
      tick();
    }
    fs.part[lane + h][0] = px; fs.part[lane + h][1] = py; fs.part[lane + h][2] = pz;
  }
  __syncwarp();
  if (cnt > 0) {  // this lane's entries [off, off + cnt) went to lanes off / R .. (off + cnt - 1) / R
    const int la = off / R, lb = (off + cnt - 1) / R;
    for (int l = la; l <= lb; ++l) {
      f[0] += fs.part[l + lane][0];
      f[1] += fs.part[l + lane][1];
      f[2] += fs.part[l + lane][2];
    }
  }
  cnt = 0;
  __syncwarp();
}

// One home cell of a pair kernel: the prefilter, the flat drains, and the
// force of each home atom written once, in place, at the end of its chunk.
template <int MODE, class T, class Eval, class Tick>
__device__ __forceinline__ void pair_cell(const SysGeom& g, int cell, const int* __restrict__ cell_start,
                                          const double4* __restrict__ pos, const int* __restrict__ perm,
                                          const PairParams& prm, PairStage& stage, FlatScratch<T>& fs, int lane,
                                          double* __restrict__ F, Eval&& eval, Tick&& tick) {
  T f[3] = {0, 0, 0};
  unsigned ownmask = 0u;  // home atoms of the chunk that own their E/W shares
  int cur = -1;
  traverse_lists<MODE>(
      g, cell, cell_start, pos, stage, lane,
      [&](bool have, int i, const double4&, int& cnt) {
        if (i != cur) {
          cur = i;
          ownmask = __ballot_sync(0xffffffffu, have && perm[i] < prm.n_owned);
        }
        flat_drain<MODE>(g, pos, stage, fs, lane, i - lane, ownmask, cnt, f, eval, tick);
      },
      [&](bool have, int i, const double4&) {
        if (have && prm.want_f) {
          const int o = perm[i];
          F[3 * o] = f[0]; F[3 * o + 1] = f[1]; F[3 * o + 2] = f[2];
        }
        f[0] = f[1] = f[2] = 0;
      });
}

__device__ __forceinline__ void load_amplitudes(const PairParams& prm, int kind, double* sA) {
  if (threadIdx.x < 16) {
    const int a = threadIdx.x >> 2, b = threadIdx.x & 3;
    sA[threadIdx.x] = (kind == 0 && a < prm.nz && b < prm.nz) ? prm.A[a * prm.nz + b] : 0.0;
  }
  __syncthreads();
}

__device__ __forceinline__ int species_index(double w) { return min(max((int)w, 0), 3); }

// Plain FP64 path.  MODE 0: displacement = (x_j - x_i) + cell shift;
// MODE 1: per-pair minimum image (small boxes).
template <int KIND, int MODE>
__global__ void __launch_bounds__(PAIR_WARPS * 32, PFW_PAIR_MINBLOCKS)
    k_pair64(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
             const double4* __restrict__ pos, const int* __restrict__ perm, int ncells, PairParams prm,
             double* __restrict__ F, double* __restrict__ cellpart, unsigned long long* __restrict__ npairs) {
  extern __shared__ __align__(16) unsigned char pair_smem[];
  PairStage* stage = reinterpret_cast<PairStage*>(pair_smem);
  FlatScratch<double>* scratch = reinterpret_cast<FlatScratch<double>*>(pair_smem + sizeof(PairStage) * PAIR_WARPS);
  __shared__ double sA[16];  // SmoothPair amplitudes A[zi][zj], 4 × 4, zero-padded
  load_amplitudes(prm, KIND, sA);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * PAIR_WARPS + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  double e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long np = 0;
  pair_cell<MODE, double>(
      g, cell, cell_start, pos, perm, prm, stage[warp], scratch[warp], lane, F,
      [&](const double4& ph, bool ownh, const double4& pj, const double* d, double r2, bool hit, double& gx,
          double& gy, double& gz) {
        np += hit;
        double en, coef;
        pair_term<KIND>(prm, KIND == 0 ? sA[species_index(ph.w) * 4 + species_index(pj.w)] : 0.0, r2, en, coef);
        coef = hit ? coef : 0.0;
        gx = coef * d[0]; gy = coef * d[1]; gz = coef * d[2];
        const double o = ownh ? 1.0 : 0.0;  // W terms of non-hits are zero already
        e += (hit && ownh) ? en : 0.0;
        w[0] += o * (d[0] * gx); w[1] += o * (d[1] * gy); w[2] += o * (d[2] * gz);
        w[3] += o * (d[0] * gy); w[4] += o * (d[0] * gz); w[5] += o * (d[1] * gz);
      },
      [] {});
  write_cell_parts(cellpart, cell, lane, e, w, np, npairs);
}

// Mixed form: the same traversal and the same FP64 cutoff decision as the
// plain path (so the neighbour set is the reference's), with the pair
// arithmetic in FP32 on the FP64 displacement rounded to FP32.  Forces
// accumulate per atom in FP32; energy and virial terms accumulate in FP32
// over at most MIXED_CHUNK pairs and are then folded into Kahan-compensated
// FP64 accumulators.
constexpr int MIXED_CHUNK = 16;

#ifndef PFW_PAIR32_MINBLOCKS
#define PFW_PAIR32_MINBLOCKS 4
#endif

template <int KIND, int MODE>
__global__ void __launch_bounds__(PAIR_WARPS * 32, PFW_PAIR32_MINBLOCKS)
    k_pair32(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
             const double4* __restrict__ pos, const int* __restrict__ perm, int ncells, PairParams prm,
             double* __restrict__ F, double* __restrict__ cellpart, unsigned long long* __restrict__ npairs) {
  extern __shared__ __align__(16) unsigned char pair_smem[];
  PairStage* stage = reinterpret_cast<PairStage*>(pair_smem);
  FlatScratch<float>* scratch = reinterpret_cast<FlatScratch<float>*>(pair_smem + sizeof(PairStage) * PAIR_WARPS);
  __shared__ double sA[16];
  load_amplitudes(prm, KIND, sA);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * PAIR_WARPS + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  Kahan ke, kw[6];
  float ce = 0.f, cw[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int cn = 0;
  unsigned long long np = 0;
  const float invc2 = (float)prm.invc2, eps4 = (float)prm.eps4, eps24 = (float)prm.eps24,
              sigma2 = (float)prm.sigma2, shift = (float)prm.shift;
  auto fold = [&]() {
    ke.add((double)ce);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      kw[k].add((double)cw[k]);
      cw[k] = 0.f;
    }
    ce = 0.f;
    cn = 0;
  };
  pair_cell<MODE, float>(
      g, cell, cell_start, pos, perm, prm, stage[warp], scratch[warp], lane, F,
      [&](const double4& ph, bool ownh, const double4& pj, const double* d, double r2d, bool hit, float& gx,
          float& gy, float& gz) {
        np += hit;
        const float d0 = (float)d[0], d1 = (float)d[1], d2 = (float)d[2];
        const float r2 = (float)r2d;
        float en, coef;
        if (KIND == 0) {
          const float a = (float)sA[species_index(ph.w) * 4 + species_index(pj.w)];
          const float q = 1.f - r2 * invc2;
          const float aq2 = a * q * q;
          en = aq2 * q;
          coef = -6.f * aq2 * invc2;
        } else {
          const float ir2 = __frcp_rn(r2);
          const float s2 = sigma2 * ir2;
          const float s6 = s2 * s2 * s2;
          en = eps4 * (s6 * s6 - s6) - shift;
          coef = eps24 * (s6 - 2.f * s6 * s6) * ir2;
        }
        coef = hit ? coef : 0.f;  // without branches: a miss has r2 >= c², finite terms
        gx = coef * d0; gy = coef * d1; gz = coef * d2;
        const float o = ownh ? 1.f : 0.f;
        ce += (hit && ownh) ? en : 0.f;
        cw[0] += o * (d0 * gx); cw[1] += o * (d1 * gy); cw[2] += o * (d2 * gz);
        cw[3] += o * (d0 * gy); cw[4] += o * (d0 * gz); cw[5] += o * (d1 * gz);
      },
      [&] {  // at most MIXED_CHUNK pairs (two per step) in the FP32 partial sums
        if (++cn == MIXED_CHUNK / 2) fold();
      });
  fold();
  double w[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) w[k] = kw[k].s - kw[k].c;
  write_cell_parts(cellpart, cell, lane, ke.s - ke.c, w, np, npairs);
}

// Per-system reduction of a batch: block s sums the cells of system s.
__global__ void k_reduce_systems(const double* __restrict__ parts, const SysGeom* __restrict__ sys, int stride,
                                 double* __restrict__ E, double* __restrict__ W) {
  __shared__ double sh[7][128];
  const int s = blockIdx.x;
  const int c0 = sys[s].cell_begin, c1 = c0 + sys[s].ncells;
  Kahan acc[7];
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x)
#pragma unroll
    for (int k = 0; k < 7; ++k) acc[k].add(parts[(size_t)stride * c + k]);
#pragma unroll
  for (int k = 0; k < 7; ++k) sh[k][threadIdx.x] = acc[k].s - acc[k].c;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
#pragma unroll
      for (int k = 0; k < 7; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (E) E[s] = sh[0][0];
    if (W) {
      double* w = W + 9 * (size_t)s;
      w[0] = sh[1][0]; w[4] = sh[2][0]; w[8] = sh[3][0];
      w[3] = w[1] = sh[4][0];
      w[6] = w[2] = sh[5][0];
      w[7] = w[5] = sh[6][0];
    }
  }
}

PairParams make_pair_params(const pfw_ws* ws, uint32_t req) {
  const PairModel& m = ws->pair;
  PairParams prm{};
  prm.kind = m.kind;
  prm.nz = m.nz;
  for (size_t k = 0; k < m.A.size() && k < 16; ++k) prm.A[k] = m.A[k];
  prm.invc2 = 1.0 / (m.cutoff * m.cutoff);
  if (m.kind == 1) {
    prm.eps4 = 4.0 * m.eps;
    prm.eps24 = 24.0 * m.eps;
    prm.sigma2 = m.sigma * m.sigma;
    double rc = m.sigma / m.cutoff, qc2 = rc * rc, qc = qc2 * qc2 * qc2;
    prm.shift = 4.0 * m.eps * (qc * qc - qc);
  }
  prm.want_f = (req & PFW_REQ_FORCES) != 0;
  prm.want_v = (req & PFW_REQ_VIRIAL) != 0;
  prm.want_e = (req & PFW_REQ_ENERGY) != 0;
  prm.n_owned = ws->n_owned < 0 ? INT32_MAX : ws->n_owned;
  return prm;
}

// Device work of one pair evaluation on a planned cell list: cell-list build,
// output clears, the pair kernel and the reductions (no allocation once the
// buffers are sized, no host synchronisation: capturable).
template <class T>
constexpr int pair_smem_bytes() {
  return (int)((sizeof(PairStage) + sizeof(FlatScratch<T>)) * PAIR_WARPS);
}

static void pair_launch(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev, bool per_system,
                        bool wrapped) {
  const PairModel& m = ws->pair;
  ws->stage_begin(0);
  prepare_launch(ws, !wrapped);
  ws->stage_end(0);
  const Prepared& P = ws->prep;
  cudaStream_t st = ws->stream;
  const PairParams prm = make_pair_params(ws, req);
  const int ncells = P.ncells;
  double* parts = static_cast<double*>(ws->cellpart.ensure(sizeof(double) * 8 * std::max(ncells, 1)));
  unsigned long long* np = static_cast<unsigned long long*>(ws->counters.ensure(64)) + 4;
  PFW_CUDA(cudaMemsetAsync(np, 0, sizeof(unsigned long long), st));
  // the half-stencil path folds every atom's force into F (no clear needed)
  const bool half = pair_half_eligible(P);
  if (F_dev && P.n > 0 && !(half && prm.want_f)) PFW_CUDA(cudaMemsetAsync(F_dev, 0, sizeof(double) * 3 * P.n, st));
  bool all_shift = true;
  for (auto& g : P.sys)
    if (g.minimum_image && !g.fast_shift) all_shift = false;
  const SysGeom* dsys = ws->sysgeom.as<SysGeom>();
  const int* cell_sys = ws->cell_sys.as<int>();
  const int* cs = ws->cell_start.as<int>();
  const double4* pos = ws->pos.as<double4>();
  const int* perm = ws->perm.as<int>();
  double* F = F_dev ? F_dev : static_cast<double*>(ws->out_F.ensure(sizeof(double) * 3 * std::max(P.n, 1)));
  ws->stage_begin(1);
  if (half) {
    pair_half_kernel(ws, prm, parts, np);
  } else if (ncells > 0) {
    dim3 grid(grid_for(ncells, PAIR_WARPS)), block(PAIR_WARPS * 32);
    bool mixed = ws->opt.precision == PFW_PRECISION_MIXED;
    if (mixed && all_shift) {
      if (m.kind == 0) k_pair32<0, 0><<<grid, block, pair_smem_bytes<float>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
      else k_pair32<1, 0><<<grid, block, pair_smem_bytes<float>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
    } else if (mixed) {
      if (m.kind == 0) k_pair32<0, 1><<<grid, block, pair_smem_bytes<float>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
      else k_pair32<1, 1><<<grid, block, pair_smem_bytes<float>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
    } else if (all_shift) {
      if (m.kind == 0) k_pair64<0, 0><<<grid, block, pair_smem_bytes<double>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
      else k_pair64<1, 0><<<grid, block, pair_smem_bytes<double>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
    } else {
      if (m.kind == 0) k_pair64<0, 1><<<grid, block, pair_smem_bytes<double>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
      else k_pair64<1, 1><<<grid, block, pair_smem_bytes<double>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, prm, F, parts, np);
    }
    ws->launches += 1;
  }
  ws->stage_end(1);
  double* E = E_dev ? E_dev : static_cast<double*>(ws->out_E.ensure(sizeof(double)));
  double* W = W_dev ? W_dev : static_cast<double*>(ws->out_W.ensure(sizeof(double) * 9));
  ws->stage_begin(2);
  if (half && prm.want_f) pair_half_fold(ws, F);
  if (per_system) {
    if (P.nsys > 0) {
      k_reduce_systems<<<P.nsys, 128, 0, st>>>(parts, dsys, 8, E_dev, W_dev);
      ws->launches += 1;
    }
  } else {
    reduce_pair_parts(ws, parts, ncells, 8, E, W);  // counts its own launches
  }
  ws->stage_end(2);
  PFW_CUDA(cudaGetLastError());
}

// A captured pair evaluation and what it was captured for.
struct PairGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<SysGeom> sys;
  const void *E = nullptr, *F = nullptr, *W = nullptr;
  uint32_t req = 0;
  uint64_t model_version = 0, alloc_epoch = 0, kernels = 0;
  int32_t n_owned = 0;
  int precision = 0;
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  bool matches(const pfw_ws* ws, const void* e, const void* f, const void* w, uint32_t r) const {
    const auto& ps = ws->prep.sys;
    return exec && E == e && F == f && W == w && req == r && model_version == ws->model_version &&
           alloc_epoch == g_alloc_epoch.load() && n_owned == ws->n_owned && precision == ws->opt.precision &&
           sys.size() == ps.size() && std::memcmp(sys.data(), ps.data(), sizeof(SysGeom) * ps.size()) == 0;
  }
};

void pair_graph_free(pfw_ws* ws) {
  if (!ws->pair_graph) return;
  ws->pair_graph->release();
  delete ws->pair_graph;
  ws->pair_graph = nullptr;
}

void pair_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev, bool per_system) {
  const PairModel& m = ws->pair;
  if (m.kind < 0) throw Error(PFW_ESTATE, "no pair model loaded");
  if (m.kind == 0 && ws->max_species >= m.nz)
    throw Error(PFW_EINVAL, "potential has no parameters for species channel " + std::to_string(ws->max_species));
  ws->species_limit = m.kind == 0 ? m.nz : INT32_MAX;
  if (!per_system && skin_pair_evaluate(ws, req, E_dev, F_dev, W_dev)) return;
  ws->prep.valid = false;  // evaluate! rebuilds topology on every call
  // the per-warp traversal state makes shared memory a residency limit: ask
  // for the largest carveout (once per device)
  static std::mutex attr_mu;
  static bool attr_done[64] = {};
  {
    std::lock_guard<std::mutex> lock(attr_mu);
    const int dev = ws->opt.device;
    if (dev < 0 || dev >= 64 || !attr_done[dev]) {
      for (const void* k : {(const void*)k_pair64<0, 0>, (const void*)k_pair64<1, 0>, (const void*)k_pair64<0, 1>,
                            (const void*)k_pair64<1, 1>, (const void*)k_pair32<0, 0>, (const void*)k_pair32<1, 0>,
                            (const void*)k_pair32<0, 1>, (const void*)k_pair32<1, 1>}) {
        PFW_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        PFW_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, pair_smem_bytes<double>()));
      }
      pair_half_setup();
      if (dev >= 0 && dev < 64) attr_done[dev] = true;
    }
  }
  // cell list without a mid-call synchronisation: its input flags are read
  // once at the end (a bad input only makes clamped cells and NaN sums)
  const bool wrapped = prepare_plan(ws, m.cutoff);
  // Repeated calls on the same structure (cells, grid, atom count, outputs,
  // model) replay one CUDA graph of the whole device sequence: the same work,
  // without the per-kernel launch gaps.  A new structure runs eagerly once
  // (sizing every buffer) and captures the graph for the calls after it.
  const bool graphable = !per_system && !wrapped && !ws->diag;
  if (graphable) {
    if (!ws->pair_graph) ws->pair_graph = new PairGraph();
    PairGraph& pg = *ws->pair_graph;
    if (pg.matches(ws, E_dev, F_dev, W_dev, req)) {
      PFW_CUDA(cudaGraphLaunch(pg.exec, ws->stream));
      ws->launches += pg.kernels;
    } else {
      pg.release();
      pair_launch(ws, req, E_dev, F_dev, W_dev, false, wrapped);
      const uint64_t l0 = ws->launches;
      cudaStream_t st = ws->stream;
      PFW_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        pair_launch(ws, req, E_dev, F_dev, W_dev, false, wrapped);
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        ws->launches = l0;
        throw;
      }
      PFW_CUDA(cudaStreamEndCapture(st, &pg.graph));
      PFW_CUDA(cudaGraphInstantiate(&pg.exec, pg.graph, 0));
      pg.kernels = ws->launches - l0;
      ws->launches = l0;
      pg.sys = ws->prep.sys;
      pg.E = E_dev;
      pg.F = F_dev;
      pg.W = W_dev;
      pg.req = req;
      pg.model_version = ws->model_version;
      pg.alloc_epoch = g_alloc_epoch.load();
      pg.n_owned = ws->n_owned;
      pg.precision = ws->opt.precision;
    }
  } else {
    pair_launch(ws, req, E_dev, F_dev, W_dev, per_system, wrapped);
  }
  prepare_check(ws);
  ws->prep.valid = true;
}

}  // namespace pfw
