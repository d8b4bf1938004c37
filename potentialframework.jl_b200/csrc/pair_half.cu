// pair_half.cu — pair energy, force and virial with every unordered pair
// evaluated once (half stencil), for grids whose stencil is 3×3×3 with a
// per-cell image shift (orthorhombic minimum image with >= 4 bins per
// periodic axis, or explicit images of radius 1).
//
// Replaces cell_task!/execute! (NeighbourList/execution.jl:173-238): the
// reference's owner rule is "the lower cell owns the pair" (j >= i in the
// cell stencil of minimum_topology!, storage.jl:244-261) and its task writes
// force[i] += g, force[j] -= g.  Here one warp owns one home cell and takes
// the pairs of its atoms with the atoms of the cell itself (j after i in
// sorted order) and of the 13 cells of the forward half of the 3×3×3
// stencil (offsets lexicographically after 0).  The reverse offset from the
// neighbour cell is in the backward half, so every unordered pair (i, j, S)
// is visited exactly once, and the displacement is exactly antisymmetric, so
// the pair set is the full list's.
//
// Per home chunk (<= 32 atoms) the candidates of the 14 cells stream through
// a box prune (a candidate farther than c from the bounding box of the home
// atoms is dropped) into a staging buffer of up to 160 candidates (FP32
// coordinates relative to the home cell's first atom).  A full buffer is one
// pass: first every 32-candidate window is tested transposed (lanes hold
// candidates, the warp walks the home atoms, a ballot per home atom gives
// its mask of candidates within c²(1 + 2⁻¹⁰)); then the pass's entries,
// home-major (home h, its candidates in staging order), are split into
// contiguous equal shares, one per lane, and evaluated two per step (exact
// FP64 displacement and cutoff, or FP32 from the staged coordinates for the
// mixed form with an FP64 re-test in the guard band).  A lane walks its
// share directly on the per-home masks, so no entry list is built.
//
// Reductions, all in a fixed order (deterministic without atomics): the
// home side accumulates in registers per owner and leaves one partial per
// (lane, owner) in slot lane + owner, which the owner adds in lane order;
// the j side groups the lanes of one step that hold the same candidate
// (match), and the lowest lane adds the group's gradients in lane order to
// the candidate's accumulator in shared memory.  After the pass each staged
// candidate's accumulator is complete for this home chunk.
//
// Forces leave the kernel as partial sums per (slot, sorted atom): slot 0 the
// home side, slot 1 the j side of the home cell's own pairs, slots 2..14 the
// j side received through each forward offset (written by exactly one home
// cell).  k_pair_fold adds the slots of an atom in slot order and writes the
// force in the original order.  Energy and virial take each unordered pair
// once (per home cell partials, reduce.cu).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>

#include "pair_math.cuh"
#include "pfw_internal.h"

namespace pfw {

constexpr int HALF_WARPS = 8;   // home cells per CTA
constexpr int HALF_NE = 14;     // self + 13 forward neighbour cells
constexpr int HALF_CAP = 160;   // staged candidates of one pass
constexpr int HALF_WIN = HALF_CAP / 32;
constexpr int HALF_NSLOT = 15;  // force slots (see above)
constexpr float HALF_GUARD = 1.0f / 1024.0f;
#ifndef PFW_HALF_MINBLOCKS
#define PFW_HALF_MINBLOCKS 2
#endif

// forward half of the 3×3×3 stencil, lexicographic order
__constant__ int8_t c_half_off[13][3] = {{0, 0, 1},  {0, 1, -1}, {0, 1, 0},  {0, 1, 1},  {1, -1, -1},
                                         {1, -1, 0}, {1, -1, 1}, {1, 0, -1}, {1, 0, 0},  {1, 0, 1},
                                         {1, 1, -1}, {1, 1, 0},  {1, 1, 1}};

template <class T>
struct alignas(16) HalfStage {
  double sh[HALF_NE][3];     // image shift of each entry (added to x_j - x_i)
  int jb[HALF_NE];           // first sorted atom of each entry's cell
  int start[HALF_NE + 1];    // flat-list offsets of the entries
  float rx[HALF_CAP], ry[HALF_CAP], rz[HALF_CAP];  // staged candidates (FP32, shifted, relative to ref)
  unsigned item[HALF_CAP];   // staged candidate: j | entry << 24 | owned << 28 | species << 29
  unsigned mh[HALF_WIN][32]; // per window and home atom: the window's candidates within c²(1 + 2⁻¹⁰)
  alignas(16) float hx[32];  // home atoms (FP32, relative to ref); read as float2 pairs
  alignas(16) float hy[32];
  alignas(16) float hz[32];
  double hxd[32], hyd[32], hzd[32];  // home atoms (FP64, as stored)
  unsigned char hsp[32];     // home atoms' species channels (clamped to 0..3)
  int off[33];               // exclusive scan of the home atoms' entry counts in the pass
  T part[63][3];             // home-side partial sums, slot lane + owner
  T fj[HALF_CAP][3];         // j-side sums of the staged candidates
};
static_assert(sizeof(HalfStage<double>) % 16 == 0 && sizeof(HalfStage<float>) % 16 == 0, "stage stride");
static_assert(offsetof(HalfStage<double>, hx) % 8 == 0 && offsetof(HalfStage<double>, hy) % 8 == 0 &&
                  offsetof(HalfStage<double>, hz) % 8 == 0 && offsetof(HalfStage<float>, hx) % 8 == 0 &&
                  offsetof(HalfStage<float>, hy) % 8 == 0 && offsetof(HalfStage<float>, hz) % 8 == 0,
              "home coordinates are read as float2");

__device__ __forceinline__ int half_slot(int entry) { return entry == 0 ? 1 : entry + 1; }

// Energy/virial accumulation of one lane: FP64 directly, or FP32 terms of at
// most 16 pairs folded into Kahan-compensated FP64 sums (mixed form).
template <class T>
struct HalfAcc;
template <>
struct HalfAcc<double> {
  double e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  __device__ __forceinline__ void add(double en, const double d[3], double gx, double gy, double gz, double o) {
    e += o * en;
    w[0] += o * (d[0] * gx); w[1] += o * (d[1] * gy); w[2] += o * (d[2] * gz);
    w[3] += o * (d[0] * gy); w[4] += o * (d[0] * gz); w[5] += o * (d[1] * gz);
  }
  __device__ __forceinline__ void tick() {}
  __device__ __forceinline__ void result(double& E, double W[6]) {
    E = e;
#pragma unroll
    for (int k = 0; k < 6; ++k) W[k] = w[k];
  }
};
template <>
struct HalfAcc<float> {
  Kahan ke, kw[6];
  float ce = 0.f, cw[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int cn = 0;
  __device__ __forceinline__ void add(float en, const float d[3], float gx, float gy, float gz, float o) {
    ce += o * en;
    cw[0] += o * (d[0] * gx); cw[1] += o * (d[1] * gy); cw[2] += o * (d[2] * gz);
    cw[3] += o * (d[0] * gy); cw[4] += o * (d[0] * gz); cw[5] += o * (d[1] * gz);
  }
  __device__ __forceinline__ void fold() {
    ke.add((double)ce);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      kw[k].add((double)cw[k]);
      cw[k] = 0.f;
    }
    ce = 0.f;
    cn = 0;
  }
  __device__ __forceinline__ void tick() {  // after each step of two pairs
    if (++cn == 8) fold();
  }
  __device__ __forceinline__ void result(double& E, double W[6]) {
    fold();
    E = ke.s - ke.c;
#pragma unroll
    for (int k = 0; k < 6; ++k) W[k] = kw[k].s - kw[k].c;
  }
};

// Per-kernel constants of one home cell's evaluation.
struct HalfCtx {
  double c2;
  float c2f, invc2f, eps4f, eps24f, sigma2f, shiftf;
  unsigned ownmask;
  bool all_own;
};

// One entry (home h, staged candidate t): returns the gradient (force on h
// += g, on t -= g), zero unless the pair is within the cutoff, and
// accumulates its energy and virial.
template <int KIND, class T>
struct HalfEval;

template <int KIND>
struct HalfEval<KIND, double> {
  __device__ __forceinline__ static void run(const HalfCtx& cx, const PairParams& prm, const double* sA,
                                             const double4* __restrict__ pos, const HalfStage<double>& st, int t,
                                             int h, bool valid, HalfAcc<double>& acc, int& np, double& gx,
                                             double& gy, double& gz) {
    const unsigned it = st.item[t];
    const int k = (it >> 24) & 15;
    const double4 pj = pos[it & 0xFFFFFFu];
    double d[3];
    d[0] = xadd(xsub(pj.x, st.hxd[h]), st.sh[k][0]);
    d[1] = xadd(xsub(pj.y, st.hyd[h]), st.sh[k][1]);
    d[2] = xadd(xsub(pj.z, st.hzd[h]), st.sh[k][2]);
    const double r2 = xr2(d[0], d[1], d[2]);
    const bool hit = valid && r2 < cx.c2;
    double en, coef;
    pair_term<KIND>(prm, KIND == 0 ? sA[st.hsp[h] * 4 + ((it >> 29) & 3u)] : 0.0, hit ? r2 : cx.c2, en, coef);
    coef = hit ? coef : 0.0;
    gx = coef * d[0]; gy = coef * d[1]; gz = coef * d[2];
    const double o = !hit ? 0.0 : cx.all_own ? 1.0 : 0.5 * (double)(((cx.ownmask >> h) & 1u) + ((it >> 28) & 1u));
    acc.add(en, d, gx, gy, gz, o);
    np += hit ? 1 : 0;
  }
};

template <int KIND>
struct HalfEval<KIND, float> {
  __device__ __forceinline__ static void run(const HalfCtx& cx, const PairParams&, const double* sA,
                                             const double4* __restrict__ pos, const HalfStage<float>& st, int t,
                                             int h, bool valid, HalfAcc<float>& acc, int& np, float& gx, float& gy,
                                             float& gz) {
    const unsigned it = st.item[t];
    float d[3] = {st.rx[t] - st.hx[h], st.ry[t] - st.hy[h], st.rz[t] - st.hz[h]};
    const float r2 = fmaf(d[0], d[0], fmaf(d[1], d[1], d[2] * d[2]));
    bool hit = valid && r2 < cx.c2f * (1.f - HALF_GUARD);
    if (valid && !hit && r2 < cx.c2f * (1.f + HALF_GUARD)) {
      // guard band: the exact reference decision (NeighbourList/geometry.jl:5-19)
      const int k = (it >> 24) & 15;
      const double4 pj = pos[it & 0xFFFFFFu];
      const double e0 = xadd(xsub(pj.x, st.hxd[h]), st.sh[k][0]);
      const double e1 = xadd(xsub(pj.y, st.hyd[h]), st.sh[k][1]);
      const double e2 = xadd(xsub(pj.z, st.hzd[h]), st.sh[k][2]);
      hit = xr2(e0, e1, e2) < cx.c2;
    }
    const float rr = hit ? r2 : cx.c2f;
    float en, coef;
    if (KIND == 0) {
      const float a = (float)sA[st.hsp[h] * 4 + ((it >> 29) & 3u)];
      const float q = 1.f - rr * cx.invc2f;
      const float aq2 = a * q * q;
      en = aq2 * q;
      coef = -6.f * aq2 * cx.invc2f;
    } else {
      const float ir2 = __frcp_rn(rr);
      const float s2 = cx.sigma2f * ir2;
      const float s6 = s2 * s2 * s2;
      en = cx.eps4f * (s6 * s6 - s6) - cx.shiftf;
      coef = cx.eps24f * (s6 - 2.f * s6 * s6) * ir2;
    }
    coef = hit ? coef : 0.f;
    gx = coef * d[0]; gy = coef * d[1]; gz = coef * d[2];
    const float o = !hit ? 0.f : cx.all_own ? 1.f : 0.5f * (float)(((cx.ownmask >> h) & 1u) + ((it >> 28) & 1u));
    acc.add(en, d, gx, gy, gz, o);
    np += hit ? 1 : 0;
  }
};

template <int KIND, class T>
__global__ void __launch_bounds__(HALF_WARPS * 32, PFW_HALF_MINBLOCKS)
    k_pair_half(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
                const double4* __restrict__ pos, const int* __restrict__ perm, int ncells, int natoms,
                PairParams prm, T* __restrict__ P, double* __restrict__ cellpart,
                unsigned long long* __restrict__ npairs) {
  extern __shared__ __align__(16) unsigned char half_smem[];
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ double sA[16];
  if (KIND == 0) {
    if (threadIdx.x < 16) {
      const int a = threadIdx.x >> 2, b = threadIdx.x & 3;
      sA[threadIdx.x] = (a < prm.nz && b < prm.nz) ? prm.A[a * prm.nz + b] : 0.0;
    }
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  HalfStage<T>& st = reinterpret_cast<HalfStage<T>*>(half_smem)[warp];
  const int cell = blockIdx.x * HALF_WARPS + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  const int b = cell_start[cell], e = cell_start[cell + 1];
  HalfAcc<T> acc;
  int np = 0;
  HalfCtx cx;
  cx.c2 = g.c2;
  cx.c2f = (float)g.c2;
  cx.invc2f = (float)prm.invc2;
  cx.eps4f = (float)prm.eps4;
  cx.eps24f = (float)prm.eps24;
  cx.sigma2f = (float)prm.sigma2;
  cx.shiftf = (float)prm.shift;
  cx.all_own = prm.n_owned == INT32_MAX;
  const bool want_f = prm.want_f != 0;
  const unsigned below = (1u << lane) - 1u;
  if (b < e) {
    // ---- the 14 entries: neighbour cell, image shift, atom range ----
    int len = 0;
    if (lane < HALF_NE) {
      const int local = cell - g.cell_begin;
      const int key[3] = {local / (g.dims[1] * g.dims[2]), (local / g.dims[2]) % g.dims[1], local % g.dims[2]};
      int off[3] = {0, 0, 0};
      if (lane > 0) {
        off[0] = c_half_off[lane - 1][0];
        off[1] = c_half_off[lane - 1][1];
        off[2] = c_half_off[lane - 1][2];
      }
      StencilEntry se;
      stencil_entry(g, key, off, se);
      int jb = 0;
      if (se.cell >= 0) {
        jb = cell_start[se.cell];
        len = cell_start[se.cell + 1] - jb;
      }
      st.jb[lane] = jb;
      st.sh[lane][0] = se.cell >= 0 ? se.sh[0] : 0.0;
      st.sh[lane][1] = se.cell >= 0 ? se.sh[1] : 0.0;
      st.sh[lane][2] = se.cell >= 0 ? se.sh[2] : 0.0;
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < HALF_NE) st.start[lane] = incl - len;
    const int total = __shfl_sync(FULL, incl, HALF_NE - 1);
    if (lane == 0) st.start[HALF_NE] = total;
    const double4 ref = pos[b];
    const float c2hi = cx.c2f * (1.f + HALF_GUARD);
    const size_t slotstride = 3 * (size_t)natoms;
    __syncwarp();
    for (int i0 = b; i0 < e; i0 += 32) {
      const int nh = min(32, e - i0);
      const bool have = lane < nh;
      const bool first = i0 == b;
      const double4 pi = pos[have ? i0 + lane : i0];
      const float hx = (float)(pi.x - ref.x), hy = (float)(pi.y - ref.y), hz = (float)(pi.z - ref.z);
      st.hx[lane] = hx;
      st.hy[lane] = hy;
      st.hz[lane] = hz;
      st.hxd[lane] = pi.x;
      st.hyd[lane] = pi.y;
      st.hzd[lane] = pi.z;
      st.hsp[lane] = (unsigned char)min(max((int)pi.w, 0), 3);
      cx.ownmask = __ballot_sync(FULL, have && (cx.all_own || perm[i0 + lane] < prm.n_owned));
      // bounding box of the home atoms (lanes without an atom sit at ref)
      float blx = hx, bly = hy, blz = hz, bhx = hx, bhy = hy, bhz = hz;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        blx = fminf(blx, __shfl_xor_sync(FULL, blx, o));
        bly = fminf(bly, __shfl_xor_sync(FULL, bly, o));
        blz = fminf(blz, __shfl_xor_sync(FULL, blz, o));
        bhx = fmaxf(bhx, __shfl_xor_sync(FULL, bhx, o));
        bhy = fmaxf(bhy, __shfl_xor_sync(FULL, bhy, o));
        bhz = fmaxf(bhz, __shfl_xor_sync(FULL, bhz, o));
      }
      T fh[3] = {0, 0, 0};
      __syncwarp();
      // ---- one pass over the n staged candidates ----
      auto pass = [&](int n) {
        const int W = (n + 31) >> 5;
        int cnt = 0;
        // transposed test, window by window: lanes hold candidates, the warp walks the home atoms
        for (int w = 0; w < W; ++w) {
          const int t = (w << 5) + lane;
          const bool mine = t < n;
          const unsigned it = st.item[mine ? t : 0];
          const int jt = (int)(it & 0xFFFFFFu);
          const bool self = mine && ((it >> 24) & 15) == 0;
          const bool any_self = __any_sync(FULL, self);
          float2 qx = make_float2(1e30f, 1e30f), qy = qx, qz = qx;
          if (mine) {
            qx = make_float2(st.rx[t], st.rx[t]);
            qy = make_float2(st.ry[t], st.ry[t]);
            qz = make_float2(st.rz[t], st.rz[t]);
          }
          unsigned Mh = 0u;
          const float2 m1 = make_float2(-1.f, -1.f);  // q - h as one exactly rounded fma
          for (int h = 0; h < nh; h += 2) {
            const float2 ux = *reinterpret_cast<const float2*>(&st.hx[h]);
            const float2 uy = *reinterpret_cast<const float2*>(&st.hy[h]);
            const float2 uz = *reinterpret_cast<const float2*>(&st.hz[h]);
            const float2 dx = __ffma2_rn(ux, m1, qx), dy = __ffma2_rn(uy, m1, qy), dz = __ffma2_rn(uz, m1, qz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            bool a = r2.x < c2hi, bb = h + 1 < nh && r2.y < c2hi;
            if (any_self) {  // the home cell's own pairs: j after i only (this also drops i == j)
              a = a && (!self || jt > i0 + h);
              bb = bb && (!self || jt > i0 + h + 1);
            }
            const unsigned ma = __ballot_sync(FULL, a), mb = __ballot_sync(FULL, bb);
            if (lane == h) Mh = ma;
            if (lane == h + 1) Mh = mb;
          }
          st.mh[w][lane] = Mh;
          cnt += __popc(Mh);
        }
        for (int t = lane; t < n; t += 32) {
          st.fj[t][0] = 0; st.fj[t][1] = 0; st.fj[t][2] = 0;
        }
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(FULL, inc, o);
          if (lane >= o) inc += y;
        }
        const int offh = inc - cnt;
        const int ntot = __shfl_sync(FULL, inc, 31);
        st.off[lane] = offh;
        if (lane == 31) st.off[32] = ntot;
        __syncwarp();
        // this lane's share [q, q + mine) of the home-major entries, walked on the masks
        const int R = (ntot + 31) >> 5;
        const int q = lane * R;
        const int nmine = max(0, min(q + R, ntot) - q);
        int h = 0, w = 0;
        unsigned m = 0u;
        if (nmine > 0) {
#pragma unroll
          for (int stp = 16; stp > 0; stp >>= 1)  // owner of q: the last home atom with off <= q
            if (h + stp <= 32 && st.off[h + stp] <= q) h += stp;
          h = min(h, 31);
          int r = q - st.off[h];
          m = st.mh[0][h];
          while (r >= __popc(m) && w + 1 < W) {
            r -= __popc(m);
            m = st.mh[++w][h];
          }
          for (; r > 0; --r) m &= m - 1u;
        }
        int left = nmine;
        auto take = [&](int& hh, int& tt) {  // the next entry of the share (left > 0, m != 0)
          hh = h;
          tt = (w << 5) + __ffs(m) - 1;
          m &= m - 1u;
          if (--left > 0) {
            while (m == 0u) {
              if (++w == W) {
                w = 0;
                if (++h == 32) break;
              }
              m = st.mh[w][h];
            }
          }
        };
        int cur = -1;
        T px = 0, py = 0, pz = 0;
        auto home_add = [&](bool v, int hh, T x, T y, T z) {
          if (!v) return;
          if (hh != cur) {
            if (cur >= 0) {
              st.part[lane + cur][0] = px; st.part[lane + cur][1] = py; st.part[lane + cur][2] = pz;
            }
            px = py = pz = 0;
            cur = hh;
          }
          px += x; py += y; pz += z;
        };
        // j side: the lanes of one step holding the same candidate form a group; its lowest lane adds
        // the group's gradients in lane order to the candidate's sum
        auto j_add = [&](bool v, int tt, T x, T y, T z) {
          const unsigned grp = __match_any_sync(FULL, v ? (unsigned)tt : 0x10000u + (unsigned)lane);
          const bool lead = v && (grp & below) == 0u;
          unsigned rest = lead ? (grp & ~(1u << lane)) : 0u;
          T sx = x, sy = y, sz = z;
          while (__any_sync(FULL, rest != 0u)) {
            const int src = rest ? __ffs(rest) - 1 : lane;
            const T vx = __shfl_sync(FULL, x, src), vy = __shfl_sync(FULL, y, src), vz = __shfl_sync(FULL, z, src);
            if (rest) {
              sx += vx; sy += vy; sz += vz;
              rest &= rest - 1u;
            }
          }
          if (lead) {
            st.fj[tt][0] -= sx; st.fj[tt][1] -= sy; st.fj[tt][2] -= sz;
          }
          __syncwarp();
        };
        for (int u = 0; u < R; u += 2) {
          const bool va = u < nmine, vb = u + 1 < nmine;
          int ha = 0, ta = 0, hb = 0, tb = 0;
          if (va) take(ha, ta);
          if (vb) take(hb, tb);
          T ax, ay, az, bx, by, bz;
          HalfEval<KIND, T>::run(cx, prm, sA, pos, st, ta, ha, va, acc, np, ax, ay, az);
          HalfEval<KIND, T>::run(cx, prm, sA, pos, st, tb, hb, vb, acc, np, bx, by, bz);
          acc.tick();
          home_add(va, ha, ax, ay, az);
          home_add(vb, hb, bx, by, bz);
          j_add(va, ta, ax, ay, az);
          j_add(vb, tb, bx, by, bz);
        }
        if (cur >= 0) {
          st.part[lane + cur][0] = px; st.part[lane + cur][1] = py; st.part[lane + cur][2] = pz;
        }
        __syncwarp();
        if (cnt > 0) {  // this home atom's entries went to lanes offh / R .. (offh + cnt - 1) / R
          const int la = offh / R, lb = (offh + cnt - 1) / R;
          for (int l = la; l <= lb; ++l) {
            fh[0] += st.part[l + lane][0]; fh[1] += st.part[l + lane][1]; fh[2] += st.part[l + lane][2];
          }
        }
        if (want_f) {
          for (int t = lane; t < n; t += 32) {
            const unsigned it = st.item[t];
            T* p = P + (size_t)half_slot((it >> 24) & 15) * slotstride + (it & 0xFFFFFFu);
            if (first) {
              p[0] = st.fj[t][0]; p[natoms] = st.fj[t][1]; p[2 * (size_t)natoms] = st.fj[t][2];
            } else {
              p[0] += st.fj[t][0]; p[natoms] += st.fj[t][1]; p[2 * (size_t)natoms] += st.fj[t][2];
            }
          }
        }
        __syncwarp();
      };
      // ---- stream the flat candidate list through the prune into the staging buffer ----
      int ns = 0;
      for (int f0 = 0; f0 < total; f0 += 32) {
        const int f = f0 + lane;
        const bool valid = f < total;
        int kk = 0;  // the entry of flat position f: the last k with start[k] <= f
#pragma unroll
        for (int stp = 8; stp > 0; stp >>= 1)
          if (kk + stp < HALF_NE && st.start[kk + stp] <= f) kk += stp;
        const int jj = valid ? st.jb[kk] + (f - st.start[kk]) : 0;
        float px = 0.f, py = 0.f, pz = 0.f;
        bool keep = false;
        double4 qd = make_double4(0.0, 0.0, 0.0, 0.0);
        if (valid) {
          qd = pos[jj];
          px = (float)((qd.x + st.sh[kk][0]) - ref.x);
          py = (float)((qd.y + st.sh[kk][1]) - ref.y);
          pz = (float)((qd.z + st.sh[kk][2]) - ref.z);
          const float ex = fmaxf(fmaxf(blx - px, px - bhx), 0.f);
          const float ey = fmaxf(fmaxf(bly - py, py - bhy), 0.f);
          const float ez = fmaxf(fmaxf(blz - pz, pz - bhz), 0.f);
          keep = fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < c2hi;
          if (!keep && first && want_f) {  // a pruned candidate receives nothing from this cell
            T* p = P + (size_t)half_slot(kk) * slotstride + jj;
            p[0] = 0; p[natoms] = 0; p[2 * (size_t)natoms] = 0;
          }
        }
        const unsigned kb = __ballot_sync(FULL, keep);
        if (keep) {
          const int slot = ns + __popc(kb & below);
          st.rx[slot] = px;
          st.ry[slot] = py;
          st.rz[slot] = pz;
          const unsigned own = (cx.all_own || perm[jj] < prm.n_owned) ? 1u : 0u;
          const unsigned zj = (unsigned)min(max((int)qd.w, 0), 3);
          st.item[slot] = (unsigned)jj | ((unsigned)kk << 24) | (own << 28) | (zj << 29);
        }
        ns += __popc(kb);
        __syncwarp();
        if (ns > HALF_CAP - 32 || (f0 + 32 >= total && ns > 0)) {
          pass(ns);
          ns = 0;
        }
      }
      if (have && want_f) {
        T* p = P + (i0 + lane);
        p[0] = fh[0]; p[natoms] = fh[1]; p[2 * (size_t)natoms] = fh[2];
      }
      __syncwarp();
    }
  }
  // ---- energy and virial partials of the home cell (each unordered pair once) ----
  double E, W[6];
  acc.result(E, W);
  unsigned long long npl = (unsigned long long)np;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    E += __shfl_xor_sync(FULL, E, o);
#pragma unroll
    for (int k = 0; k < 6; ++k) W[k] += __shfl_xor_sync(FULL, W[k], o);
    npl += __shfl_xor_sync(FULL, npl, o);
  }
  if (lane == 0) {
    double* cp = cellpart + 8 * (size_t)cell;
    cp[0] = E;
#pragma unroll
    for (int k = 0; k < 6; ++k) cp[1 + k] = -W[k];
    cp[7] = 0;
    if (npl) atomicAdd(npairs, 2 * npl);  // the directed count, as the full-list kernels report it
  }
}

// Forces: the slots of each atom added in slot order (home side, own-cell j
// side, then the forward offsets whose source cell exists and has atoms),
// written in the original order.  One warp per cell, lanes over its atoms.
template <class T>
__global__ void __launch_bounds__(256)
    k_pair_fold(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
                const int* __restrict__ perm, int ncells, int natoms, const T* __restrict__ P, double* __restrict__ F) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= ncells) return;
  const int cell = warp;
  const int b = cell_start[cell], e = cell_start[cell + 1];
  if (b == e) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  // which forward offsets reach this cell from an existing, non-empty source
  unsigned srcmask = 0u;
  if (lane < 13) {
    const int local = cell - g.cell_begin;
    const int key[3] = {local / (g.dims[1] * g.dims[2]), (local / g.dims[2]) % g.dims[1], local % g.dims[2]};
    const int off[3] = {-c_half_off[lane][0], -c_half_off[lane][1], -c_half_off[lane][2]};
    StencilEntry se;
    stencil_entry(g, key, off, se);
    if (se.cell >= 0 && cell_start[se.cell + 1] > cell_start[se.cell]) srcmask = 1u;
  }
  srcmask = __ballot_sync(0xffffffffu, srcmask != 0u);
  const size_t ss = 3 * (size_t)natoms;
  for (int i = b + lane; i < e; i += 32) {
    double f[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) f[x] = (double)P[(size_t)x * natoms + i] + (double)P[ss + (size_t)x * natoms + i];
    for (int k = 0; k < 13; ++k) {
      if (!((srcmask >> k) & 1u)) continue;
      const T* p = P + (size_t)(k + 2) * ss + i;
#pragma unroll
      for (int x = 0; x < 3; ++x) f[x] += (double)p[(size_t)x * natoms];
    }
    const int o = perm[i];
    F[3 * o] = f[0];
    F[3 * o + 1] = f[1];
    F[3 * o + 2] = f[2];
  }
}

template <class T>
static int half_smem_bytes() {
  return (int)(sizeof(HalfStage<T>) * HALF_WARPS);
}

// Every system's grid has a 3×3×3 stencil with a per-cell image shift.
bool pair_half_eligible(const Prepared& P) {
  if (P.sys.empty() || P.n >= (1 << 24)) return false;  // staged candidates carry j in 24 bits
  for (const SysGeom& g : P.sys) {
    if (g.brute) return false;
    if (g.minimum_image && !g.fast_shift) return false;
    for (int a = 0; a < 3; ++a)
      if (!g.minimum_image && g.radius[a] != 1) return false;
  }
  return true;
}

void pair_half_setup() {
  for (const void* k : {(const void*)k_pair_half<0, double>, (const void*)k_pair_half<1, double>}) {
    PFW_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    PFW_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, half_smem_bytes<double>()));
  }
  for (const void* k : {(const void*)k_pair_half<0, float>, (const void*)k_pair_half<1, float>}) {
    PFW_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    PFW_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, half_smem_bytes<float>()));
  }
}

// The half-stencil pair kernel on a built cell list (energy/virial partials
// per cell, forces as per-slot partial sums).
void pair_half_kernel(pfw_ws* ws, const PairParams& prm, double* parts, unsigned long long* np) {
  const Prepared& Pp = ws->prep;
  const int ncells = Pp.ncells, n = Pp.n;
  cudaStream_t st = ws->stream;
  const bool mixed = ws->opt.precision == PFW_PRECISION_MIXED;
  const size_t esz = mixed ? sizeof(float) : sizeof(double);
  void* Pbuf = ws->pair_slots.ensure(esz * HALF_NSLOT * 3 * (size_t)std::max(n, 1));
  if (ncells <= 0) return;
  const SysGeom* dsys = ws->sysgeom.as<SysGeom>();
  const int* cell_sys = ws->cell_sys.as<int>();
  const int* cs = ws->cell_start.as<int>();
  const double4* pos = ws->pos.as<double4>();
  const int* perm = ws->perm.as<int>();
  const dim3 grid(grid_for(ncells, HALF_WARPS)), block(HALF_WARPS * 32);
  if (mixed) {
    float* Pf = static_cast<float*>(Pbuf);
    if (ws->pair.kind == 0)
      k_pair_half<0, float><<<grid, block, half_smem_bytes<float>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, n,
                                                                          prm, Pf, parts, np);
    else
      k_pair_half<1, float><<<grid, block, half_smem_bytes<float>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells, n,
                                                                          prm, Pf, parts, np);
  } else {
    double* Pd = static_cast<double*>(Pbuf);
    if (ws->pair.kind == 0)
      k_pair_half<0, double><<<grid, block, half_smem_bytes<double>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells,
                                                                            n, prm, Pd, parts, np);
    else
      k_pair_half<1, double><<<grid, block, half_smem_bytes<double>(), st>>>(dsys, cell_sys, cs, pos, perm, ncells,
                                                                            n, prm, Pd, parts, np);
  }
  ws->launches += 1;
}

// Forces of the half-stencil kernel: the slots folded into F (original order).
void pair_half_fold(pfw_ws* ws, double* F) {
  const Prepared& Pp = ws->prep;
  const int ncells = Pp.ncells, n = Pp.n;
  if (ncells <= 0) return;
  const SysGeom* dsys = ws->sysgeom.as<SysGeom>();
  const int* cell_sys = ws->cell_sys.as<int>();
  const int* cs = ws->cell_start.as<int>();
  const int* perm = ws->perm.as<int>();
  const int grid = grid_for((int64_t)ncells * 32, 256);
  if (ws->opt.precision == PFW_PRECISION_MIXED)
    k_pair_fold<float><<<grid, 256, 0, ws->stream>>>(dsys, cell_sys, cs, perm, ncells, n,
                                                     ws->pair_slots.as<float>(), F);
  else
    k_pair_fold<double><<<grid, 256, 0, ws->stream>>>(dsys, cell_sys, cs, perm, ncells, n,
                                                      ws->pair_slots.as<double>(), F);
  ws->launches += 1;
}

}  // namespace pfw
