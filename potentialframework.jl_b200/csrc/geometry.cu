// geometry.cu — device preparation of the cell list: prepare! of
// NeighbourList/storage.jl:130-241 as one-pass GPU kernels.
//
//   host   prepare_system  path decision, periodic basis, reciprocal, bins
//   k_wrap                 canonical wrap (minimum image: mod(x, L); explicit
//                          images: basis·mod(basis⁻¹x, 1)), bin coordinates,
//                          image windings of the original coordinates
//   k_key_count            bin key → dense cell index; per-cell population
//   exclusive scan         cell offsets (no atomics)
//   k_scatter, k_cell_rank stable placement: atoms of a cell ordered by
//                          original index = the reference's sortperm order
//   k_gather               sorted SoA positions (double4: x, y, z, species)
//
// Without an open axis to measure first (every periodic box, and batches of
// them) the build runs fused: k_bin (system lookup, wrap, windings, key,
// count), the scan, k_scatter, and k_cell_order (rank, gather, species
// check, cell → system); the separate kernels serve the open-axis path.
#include <algorithm>
#include <cmath>

#include "pfw_internal.h"

namespace pfw {

// ---------------------------------------------------------------------------
// host: per-system decisions (storage.jl:130-193)
// ---------------------------------------------------------------------------
// periodic_basis (storage.jl:83-108)
static void periodic_basis(const double* H, const uint8_t* pb, double* B) {
  std::vector<std::array<double, 3>> orth;
  auto dot = [](const double* q, const double* v) {
    double s = q[0] * v[0];
    s = s + q[1] * v[1];
    s = s + q[2] * v[2];
    return s;
  };
  for (int k = 0; k < 9; ++k) B[k] = 0;
  for (int a = 0; a < 3; ++a) {
    if (!pb[a]) continue;
    double v[3] = {H[3 * a], H[3 * a + 1], H[3 * a + 2]};
    for (double x : v)
      if (!std::isfinite(x)) throw Error(PFW_EINVAL, "periodic cell vectors must be finite");
    for (int c = 0; c < 3; ++c) B[3 * a + c] = v[c];
    for (auto& q : orth) {
      double s = dot(q.data(), v);
      for (int c = 0; c < 3; ++c) v[c] = v[c] - s * q[c];
    }
    double nrm = std::sqrt(dot(v, v));
    if (!(std::isfinite(nrm) && nrm > 0))
      throw Error(PFW_EINVAL, "periodic cell vectors must be linearly independent");
    std::array<double, 3> u{v[0] / nrm, v[1] / nrm, v[2] / nrm};
    orth.push_back(u);
  }
  for (int a = 0; a < 3; ++a) {
    if (pb[a]) continue;
    double cand[3][3];
    for (int k = 0; k < 3; ++k) {
      double v[3] = {0, 0, 0};
      v[k] = 1.0;
      for (auto& q : orth) {
        double s = dot(q.data(), v);
        for (int c = 0; c < 3; ++c) v[c] = v[c] - s * q[c];
      }
      for (int c = 0; c < 3; ++c) cand[k][c] = v[c];
    }
    int best = 0;
    double bestn = -1;
    for (int k = 0; k < 3; ++k) {
      double s = dot(cand[k], cand[k]);
      if (s > bestn) { bestn = s; best = k; }
    }
    double nrm = std::sqrt(dot(cand[best], cand[best]));
    std::array<double, 3> u{cand[best][0] / nrm, cand[best][1] / nrm, cand[best][2] / nrm};
    for (int c = 0; c < 3; ++c) B[3 * a + c] = u[c];
    orth.push_back(u);
  }
}

// 3×3 inverse: rows (b×c, c×a, a×b)/det for columns a, b, c.
static void inv3(const double* m, double* r) {
  const double *a = m, *b = m + 3, *c = m + 6;
  double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
  double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
  double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  double det = a[0] * bc[0];
  det = det + a[1] * bc[1];
  det = det + a[2] * bc[2];
  for (int k = 0; k < 3; ++k) {
    r[0 + 3 * k] = bc[k] / det;
    r[1 + 3 * k] = ca[k] / det;
    r[2 + 3 * k] = ab[k] / det;
  }
}

// Everything prepare! decides from the cell, flags, cutoff and atom count.
// Open-axis origins and extents need the atoms and are completed later.
static SysGeom prepare_system(const HostSystem& hs, double c, int brute_threshold) {
  SysGeom g;
  std::memset(&g, 0, sizeof(g));
  const double* H = hs.H;
  bool pb[3] = {hs.pbc[0] != 0, hs.pbc[1] != 0, hs.pbc[2] != 0};
  bool axisaligned = true;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      if (a != b && H[a + 3 * b] != 0.0) axisaligned = false;
  double L[3] = {H[0], H[4], H[8]};
  bool mi = true;
  if (pb[0] || pb[1] || pb[2]) {
    mi = axisaligned;
    for (int a = 0; a < 3; ++a)
      if (pb[a] && !(std::isfinite(L[a]) && L[a] > 2 * c)) mi = false;
  }
  g.minimum_image = mi;
  if (mi) {
    for (int k = 0; k < 9; ++k) g.basis[k] = g.recip[k] = (k % 4 == 0) ? 1.0 : 0.0;
  } else {
    uint8_t p8[3] = {hs.pbc[0], hs.pbc[1], hs.pbc[2]};
    periodic_basis(H, p8, g.basis);
    inv3(g.basis, g.recip);
    for (double v : g.recip)
      if (!std::isfinite(v)) throw Error(PFW_EINVAL, "periodic cell vectors must be linearly independent");
  }
  for (int b = 0; b < 3; ++b)
    for (int a = 0; a < 3; ++a) g.Hz[a + 3 * b] = pb[b] ? H[a + 3 * b] : 0.0;
  g.c = c;
  g.c2 = c * c;
  g.brute = hs.natoms <= brute_threshold;
  for (int a = 0; a < 3; ++a) {
    g.pbc[a] = pb[a];
    g.L[a] = L[a];
    double reach;
    if (mi) {
      reach = c;
    } else {
      double s = g.recip[a] * g.recip[a];
      s = s + g.recip[a + 3] * g.recip[a + 3];
      s = s + g.recip[a + 6] * g.recip[a + 6];
      reach = c * std::sqrt(s);
    }
    double extent = mi ? L[a] : 1.0;
    int64_t dims = pb[a] ? std::max<int64_t>(1, (int64_t)std::floor(extent / reach)) : 1;
    if (dims > (1 << 20)) throw Error(PFW_EINVAL, "cell grid too fine (cutoff too small for the box)");
    g.pdims[a] = (int32_t)dims;
    g.sizecell[a] = pb[a] ? extent / (double)dims : reach;
    g.origin[a] = 0.0;
    g.dims[a] = g.brute ? 1 : (int32_t)dims;
    if (mi) g.radius[a] = 1;
    else if (g.brute) g.radius[a] = pb[a] ? (int32_t)std::ceil(reach) : 0;
    else g.radius[a] = (int32_t)std::max<int64_t>(1, (int64_t)std::ceil(reach / g.sizecell[a]));
  }
  if (g.brute) {
    for (int a = 0; a < 3; ++a) g.dims[a] = 1;
  }
  // minimum image with a per-cell wrap shift is exact when every periodic
  // axis has at least 4 bins (see pfw_common.cuh)
  g.fast_shift = 0;
  if (mi && !g.brute) {
    g.fast_shift = 1;
    for (int a = 0; a < 3; ++a)
      if (pb[a] && g.pdims[a] < 4) g.fast_shift = 0;
  }
  g.atom_begin = hs.atom_begin;
  g.natoms = hs.natoms;
  return g;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__global__ void k_atom_sys(const SysGeom* __restrict__ sys, int nsys, int n, int* __restrict__ atom_sys) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (sys[mid].atom_begin <= i) lo = mid;
    else hi = mid - 1;
  }
  atom_sys[i] = lo;
}

// Canonical wrap (storage.jl:160-180), bin coordinates (:188) and image
// windings of the original coordinates (interface.jl:100-114).
__global__ void k_wrap(int n, const double* __restrict__ X, const int* __restrict__ atom_sys,
                       const SysGeom* __restrict__ sys, double* __restrict__ wrapped,
                       double* __restrict__ bincoord, int* __restrict__ wind, int* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SysGeom& g = sys[atom_sys[i]];
  double v[3] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]};
  if (!(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) atomicExch(bad, 1);
  double w[3], b[3];
  int wd[3];
  if (g.minimum_image) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      w[a] = g.pbc[a] ? jl_mod(v[a], g.L[a]) : v[a];
      b[a] = w[a];
      wd[a] = g.pbc[a] ? (int)floor(xdiv(v[a], g.L[a])) : 0;
    }
  } else {
    double f[3];
    xmatvec(g.recip, v[0], v[1], v[2], f);
#pragma unroll
    for (int a = 0; a < 3; ++a) wd[a] = g.pbc[a] ? (int)floor(f[a]) : 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) f[a] = g.pbc[a] ? jl_mod(f[a], 1.0) : f[a];
    xmatvec(g.basis, f[0], f[1], f[2], w);
#pragma unroll
    for (int a = 0; a < 3; ++a) b[a] = f[a];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    wrapped[3 * i + a] = w[a];
    bincoord[3 * i + a] = b[a];
    wind[3 * i + a] = wd[a];
  }
}

// Per-system min/max of bin coordinates along open axes (only when a system
// has an open axis).  One block per system.
__global__ void k_open_minmax(const SysGeom* __restrict__ sys, const double* __restrict__ bincoord,
                              double* __restrict__ out /* nsys × 6 */) {
  const SysGeom& g = sys[blockIdx.x];
  __shared__ double smin[3][256], smax[3][256];
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = g.atom_begin + threadIdx.x; i < g.atom_begin + g.natoms; i += blockDim.x)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double v = bincoord[3 * i + a];
      mn[a] = fmin(mn[a], v);
      mx[a] = fmax(mx[a], v);
    }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    smin[a][threadIdx.x] = mn[a];
    smax[a][threadIdx.x] = mx[a];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        smin[a][threadIdx.x] = fmin(smin[a][threadIdx.x], smin[a][threadIdx.x + s]);
        smax[a][threadIdx.x] = fmax(smax[a][threadIdx.x], smax[a][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int a = 0; a < 3; ++a) {
      out[6 * blockIdx.x + a] = smin[a][0];
      out[6 * blockIdx.x + 3 + a] = smax[a][0];
    }
}

// Bin key (storage.jl:194-198) → dense global cell; provisional slot.
__global__ void k_key_count(int n, const int* __restrict__ atom_sys, const SysGeom* __restrict__ sys,
                            const double* __restrict__ bincoord, int* __restrict__ cellid,
                            int* __restrict__ slot, int* __restrict__ count, int* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SysGeom& g = sys[atom_sys[i]];
  int key[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double b = bincoord[3 * i + a];
    if (g.brute) {
      key[a] = 0;
    } else if (g.pbc[a]) {
      // clamp(floor(Int, x/sizecell), 0, dims-1); NaN lands in bin 0 (flagged by k_wrap)
      double q = floor(xdiv(b, g.sizecell[a]));
      key[a] = (q >= 0.0) ? (q > g.pdims[a] - 1 ? g.pdims[a] - 1 : (int)q) : 0;
    } else {
      double q = floor(xdiv(xsub(b, g.origin[a]), g.sizecell[a]));
      if (!(q >= 0.0 && q < (double)g.dims[a])) {
        atomicExch(bad, 2);
        q = 0.0;
      }
      key[a] = (int)q;
    }
  }
  int c = g.cell_begin + (key[0] * g.dims[1] + key[1]) * g.dims[2] + key[2];
  cellid[i] = c;
  slot[i] = atomicAdd(&count[c], 1);
}

__global__ void k_scatter(int n, const int* __restrict__ cellid, const int* __restrict__ slot,
                          const int* __restrict__ cell_start, int* __restrict__ tmp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  tmp[cell_start[cellid[i]] + slot[i]] = i;
}

// Deterministic within-cell order: rank of each atom among its cell by
// original index (stable sortperm order).  One warp per cell.
__global__ void k_cell_rank(int ncells, const int* __restrict__ cell_start, const int* __restrict__ tmp,
                            int* __restrict__ perm) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= ncells) return;
  int b = cell_start[warp], e = cell_start[warp + 1];
  for (int t = b + lane; t < e; t += 32) {
    int me = tmp[t];
    int rank = 0;
    for (int u = b; u < e; ++u) rank += tmp[u] < me;
    perm[b + rank] = me;
  }
}

// Species channels are validated here, on the device, because geometry
// uploaded from device memory is never seen by the host: a channel outside
// [0, limit) (limit = the channel count of the model being evaluated) sets
// bad_species, which prepare_check turns into PFW_EINVAL, and is stored as
// channel 0 so that no kernel indexes a model table with it.
__global__ void k_gather(int n, const int* __restrict__ perm, const double* __restrict__ wrapped,
                         const int* __restrict__ species, double4* __restrict__ pos, int* __restrict__ inverse,
                         int limit, int* __restrict__ bad_species) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i = perm[k];
  int z = species[i];
  if (z < 0 || z >= limit) {
    atomicExch(bad_species, 1);
    z = 0;
  }
  pos[k] = make_double4(wrapped[3 * i], wrapped[3 * i + 1], wrapped[3 * i + 2], (double)z);
  inverse[i] = k;
}

// ---- the fused build (no open-axis pre-pass): two kernels replace five ----
__device__ __forceinline__ int system_of_atom(const SysGeom* __restrict__ sys, int nsys, int i) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sys[mid].atom_begin <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// k_atom_sys + k_wrap + k_key_count in one pass: the canonical wrap, the
// windings, the bin key and the provisional slot of every atom (the same
// arithmetic as the three kernels, without the bin-coordinate round trip).
__global__ void k_bin(int n, const double* __restrict__ X, const SysGeom* __restrict__ sys, int nsys,
                      double* __restrict__ wrapped, int* __restrict__ wind, int* __restrict__ cellid,
                      int* __restrict__ slot, int* __restrict__ count, int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SysGeom& g = sys[nsys == 1 ? 0 : system_of_atom(sys, nsys, i)];
  const double v[3] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]};
  if (!(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) atomicExch(bad, 1);
  double w[3], b[3];
  int wd[3];
  if (g.minimum_image) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      w[a] = g.pbc[a] ? jl_mod(v[a], g.L[a]) : v[a];
      b[a] = w[a];
      wd[a] = g.pbc[a] ? (int)floor(xdiv(v[a], g.L[a])) : 0;
    }
  } else {
    double f[3];
    xmatvec(g.recip, v[0], v[1], v[2], f);
#pragma unroll
    for (int a = 0; a < 3; ++a) wd[a] = g.pbc[a] ? (int)floor(f[a]) : 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) f[a] = g.pbc[a] ? jl_mod(f[a], 1.0) : f[a];
    xmatvec(g.basis, f[0], f[1], f[2], w);
#pragma unroll
    for (int a = 0; a < 3; ++a) b[a] = f[a];
  }
  int key[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    wrapped[3 * i + a] = w[a];
    wind[3 * i + a] = wd[a];
    if (g.brute) {
      key[a] = 0;
    } else if (g.pbc[a]) {
      const double q = floor(xdiv(b[a], g.sizecell[a]));
      key[a] = (q >= 0.0) ? (q > g.pdims[a] - 1 ? g.pdims[a] - 1 : (int)q) : 0;
    } else {
      // open axes take the pre-pass path; here only a brute-force system has one
      key[a] = 0;
    }
  }
  const int c = g.cell_begin + (key[0] * g.dims[1] + key[1]) * g.dims[2] + key[2];
  cellid[i] = c;
  slot[i] = atomicAdd(&count[c], 1);
}

// k_cell_rank + k_gather + k_cell_sys in one pass, one warp per cell: the
// rank of each atom among its cell by original index (stable order), the
// sorted double4 positions with their validated species channel, the
// inverse permutation, the cell's system and the largest population.
__global__ void k_cell_order(int ncells, const SysGeom* __restrict__ sys, int nsys,
                             const int* __restrict__ cell_start, const int* __restrict__ tmp,
                             const double* __restrict__ wrapped, const int* __restrict__ species,
                             int* __restrict__ perm, double4* __restrict__ pos, int* __restrict__ inverse,
                             int* __restrict__ cell_sys, int* __restrict__ maxpop, int limit,
                             int* __restrict__ bad_species) {
  const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (cell >= ncells) return;
  const int b = cell_start[cell], e = cell_start[cell + 1];
  if (lane == 0) {
    int lo = 0, hi = nsys - 1;  // the last system whose cell range starts at or before this cell
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sys[mid].cell_begin <= cell) lo = mid;
      else hi = mid - 1;
    }
    cell_sys[cell] = lo;
    if (e > b) atomicMax(maxpop, e - b);
  }
  const int pop = e - b;
  for (int t = b + lane; t < e; t += 32) {
    const int me = tmp[t];
    int rank = 0;
    if (pop <= 32) {
      // the whole cell is in this warp's lanes: count smaller indices by shuffles
      for (int u = 0; u < pop; ++u) rank += __shfl_sync(pop == 32 ? 0xffffffffu : (1u << pop) - 1u, me, u) < me;
    } else {
      for (int u = b; u < e; ++u) rank += tmp[u] < me;
    }
    const int k = b + rank;
    perm[k] = me;
    int z = species[me];
    if (z < 0 || z >= limit) {
      atomicExch(bad_species, 1);
      z = 0;
    }
    pos[k] = make_double4(wrapped[3 * me], wrapped[3 * me + 1], wrapped[3 * me + 2], (double)z);
    inverse[me] = k;
  }
}

__global__ void k_cell_sys(const SysGeom* __restrict__ sys, int nsys, int ncells, int* __restrict__ cell_sys,
                           const int* __restrict__ cell_start, int* __restrict__ maxpop) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (sys[mid].cell_begin <= c) lo = mid;
    else hi = mid - 1;
  }
  cell_sys[c] = lo;
  atomicMax(maxpop, cell_start[c + 1] - cell_start[c]);
}

// ---------------------------------------------------------------------------
// exclusive scan (three phases: tile sums, scan of sums, tile scan + offset)
// ---------------------------------------------------------------------------
constexpr int SCAN_BLOCK = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

template <class T>
__device__ T block_exclusive_scan(T v, T* total) {
  __shared__ T warp_sums[SCAN_BLOCK / 32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T s = lane < SCAN_BLOCK / 32 ? warp_sums[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < SCAN_BLOCK / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  T prefix = warp > 0 ? warp_sums[warp - 1] : T(0);
  if (total) *total = warp_sums[SCAN_BLOCK / 32 - 1];
  __syncthreads();
  return prefix + x - v;
}

template <class Tin, class T>
__global__ void k_tile_sums(const Tin* __restrict__ in, int64_t n, T* __restrict__ sums) {
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  T s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k)
    if (base + k < n) s += (T)in[base + k];
  T total;
  block_exclusive_scan<T>(s, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <class T>
__global__ void k_scan_sums(T* __restrict__ sums, int64_t nb, T* __restrict__ grand) {
  // single block, sequential over chunks of SCAN_BLOCK
  T carry = 0;
  for (int64_t base = 0; base < nb; base += SCAN_BLOCK) {
    int64_t idx = base + threadIdx.x;
    T v = idx < nb ? sums[idx] : T(0);
    T total;
    T ex = block_exclusive_scan<T>(v, &total);
    if (idx < nb) sums[idx] = ex + carry;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *grand = carry;
}

template <class Tin, class T>
__global__ void k_tile_scan(const Tin* __restrict__ in, int64_t n, const T* __restrict__ sums, T* __restrict__ out) {
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  T vals[SCAN_ITEMS];
  T s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    vals[k] = (base + k < n) ? (T)in[base + k] : T(0);
    s += vals[k];
  }
  T ex = block_exclusive_scan<T>(s, nullptr) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < n) out[base + k] = ex;
    ex += vals[k];
  }
}

template <class Tin, class T>
static void exclusive_scan(pfw_ws* ws, const Tin* in, T* out, int64_t n) {
  int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb == 0) nb = 1;
  T* sums = static_cast<T*>(ws->scan_tmp.ensure(sizeof(T) * (nb + 1)));
  k_tile_sums<Tin, T><<<(unsigned)nb, SCAN_BLOCK, 0, ws->stream>>>(in, n, sums);
  k_scan_sums<T><<<1, SCAN_BLOCK, 0, ws->stream>>>(sums, nb, out + n);
  k_tile_scan<Tin, T><<<(unsigned)nb, SCAN_BLOCK, 0, ws->stream>>>(in, n, sums, out);
  ws->launches += 3;
  PFW_CUDA(cudaGetLastError());
}

void exclusive_scan_i32(pfw_ws* ws, const int32_t* in, int32_t* out, int64_t n) { exclusive_scan(ws, in, out, n); }
void exclusive_scan_i64(pfw_ws* ws, const int32_t* in, int64_t* out, int64_t n) { exclusive_scan(ws, in, out, n); }

// ---------------------------------------------------------------------------
// prepare: cell list of the current geometry for a cutoff
// ---------------------------------------------------------------------------
// Host decisions, buffer sizing and (only when a system has an open axis) the
// wrap + min/max pass that fixes the open-axis grid.  Returns true when that
// pass already wrapped the positions.
bool prepare_plan(pfw_ws* ws, double cutoff) {
  if (!(std::isfinite(cutoff) && cutoff > 0)) throw Error(PFW_EINVAL, "cutoff must be finite and positive (Å)");
  if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
  Prepared& P = ws->prep;
  const int n = ws->n;
  const int nsys = (int)ws->systems.size();
  // neighbour lists pack sorted indices in 24 bits
  if (n >= (1 << 24)) throw Error(PFW_EINVAL, "at most 16,777,215 atoms per evaluation");
  cudaStream_t st = ws->stream;
  P.sys.resize(nsys);
  bool any_open = false, any_image = false;
  for (int s = 0; s < nsys; ++s) {
    P.sys[s] = prepare_system(ws->systems[s], cutoff, ws->opt.bruteforce_threshold);
    for (int a = 0; a < 3; ++a)
      if (!P.sys[s].pbc[a] && !P.sys[s].brute) any_open = true;
    if (!P.sys[s].minimum_image) any_image = true;
  }
  SysGeom* dsys = static_cast<SysGeom*>(ws->sysgeom.ensure(sizeof(SysGeom) * nsys));
  ws->atom_sys.ensure(sizeof(int) * std::max(n, 1));
  ws->wrapped.ensure(sizeof(double) * 3 * std::max(n, 1));
  ws->bincoord.ensure(sizeof(double) * 3 * std::max(n, 1));
  ws->wind.ensure(sizeof(int) * 3 * std::max(n, 1));
  ws->counters.ensure(64);  // int flags [0..7] (0: bad input, 4: largest cell), u64 pair count at byte 32
  bool wrapped_done = false;
  if (any_open && n > 0) {
    PFW_CUDA(cudaMemcpyAsync(dsys, P.sys.data(), sizeof(SysGeom) * nsys, cudaMemcpyHostToDevice, st));
    int* bad = ws->counters.as<int>();
    PFW_CUDA(cudaMemsetAsync(bad, 0, sizeof(int) * 8, st));
    k_atom_sys<<<grid_for(n, 256), 256, 0, st>>>(dsys, nsys, n, ws->atom_sys.as<int>());
    k_wrap<<<grid_for(n, 256), 256, 0, st>>>(n, ws->X.as<double>(), ws->atom_sys.as<int>(), dsys,
                                             ws->wrapped.as<double>(), ws->bincoord.as<double>(), ws->wind.as<int>(), bad);
    double* mm = static_cast<double*>(ws->minmax.ensure(sizeof(double) * 6 * nsys));
    k_open_minmax<<<nsys, 256, 0, st>>>(dsys, ws->bincoord.as<double>(), mm);
    ws->launches += 3;
    std::vector<double> h(6 * nsys);
    PFW_CUDA(cudaMemcpyAsync(h.data(), mm, sizeof(double) * 6 * nsys, cudaMemcpyDeviceToHost, st));
    PFW_CUDA(cudaStreamSynchronize(st));
    for (int s = 0; s < nsys; ++s) {
      SysGeom& g = P.sys[s];
      if (g.brute) continue;
      for (int a = 0; a < 3; ++a) {
        if (g.pbc[a]) continue;
        double lo = g.natoms > 0 ? h[6 * s + a] : 0.0, hi = g.natoms > 0 ? h[6 * s + 3 + a] : 0.0;
        if (!(std::isfinite(lo) && std::isfinite(hi))) throw Error(PFW_EINVAL, "positions must be finite");
        g.origin[a] = lo;
        // the largest key any atom can take (floor is monotone)
        double q = std::floor((hi - lo) / g.sizecell[a]);
        if (q > (double)(1 << 22)) throw Error(PFW_EINVAL, "open-axis extent too large for the dense cell grid");
        g.dims[a] = (int32_t)q + 1;
      }
    }
    wrapped_done = true;
  }
  int64_t ncells = 0;
  for (int s = 0; s < nsys; ++s) {
    SysGeom& g = P.sys[s];
    g.cell_begin = (int32_t)ncells;
    int64_t c = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
    g.ncells = (int32_t)c;
    ncells += c;
    if (ncells > (int64_t)1 << 30) throw Error(PFW_EINVAL, "cell grid too large");
  }
  PFW_CUDA(cudaMemcpyAsync(dsys, P.sys.data(), sizeof(SysGeom) * nsys, cudaMemcpyHostToDevice, st));
  P.ncells = (int32_t)ncells;
  P.nsys = nsys;
  P.n = n;
  P.any_image = any_image;
  P.cutoff = cutoff;
  P.species_limit = ws->species_limit;
  ws->cell_count.ensure(sizeof(int) * (ncells + 1));
  ws->cell_start.ensure(sizeof(int) * (ncells + 1));
  ws->cellid.ensure(sizeof(int) * std::max(n, 1));
  ws->slot.ensure(sizeof(int) * std::max(n, 1));
  ws->tmp_idx.ensure(sizeof(int) * std::max(n, 1));
  ws->perm.ensure(sizeof(int) * std::max(n, 1));
  ws->inverse.ensure(sizeof(int) * std::max(n, 1));
  ws->pos.ensure(sizeof(double4) * std::max(n, 1));
  ws->cell_sys.ensure(sizeof(int) * std::max<int64_t>(ncells, 1));
  const int64_t nb = (std::max<int64_t>(ncells, n) + 4095) / 4096 + 1;
  ws->scan_tmp.ensure(sizeof(int64_t) * (nb + 1));
  return wrapped_done;
}

// Device work of the cell-list build on planned buffers: no allocation and no
// host synchronisation, so it can be captured in a CUDA graph.
void prepare_launch(pfw_ws* ws, bool wrap) {
  const Prepared& P = ws->prep;
  const int n = P.n, nsys = P.nsys;
  const int64_t ncells = P.ncells;
  cudaStream_t st = ws->stream;
  const SysGeom* dsys = ws->sysgeom.as<SysGeom>();
  int* bad = ws->counters.as<int>();
  int* atom_sys = ws->atom_sys.as<int>();
  double* bincoord = ws->bincoord.as<double>();
  int* count = ws->cell_count.as<int>();
  int* cell_start = ws->cell_start.as<int>();
  if (wrap) {
    // no open-axis pre-pass: the fused build (bin; scan; scatter; order)
    PFW_CUDA(cudaMemsetAsync(bad, 0, sizeof(int) * 8, st));
    PFW_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (ncells + 1), st));
    if (n > 0) {
      k_bin<<<grid_for(n, 256), 256, 0, st>>>(n, ws->X.as<double>(), dsys, nsys, ws->wrapped.as<double>(),
                                              ws->wind.as<int>(), ws->cellid.as<int>(), ws->slot.as<int>(), count,
                                              bad);
      ws->launches += 1;
    }
    exclusive_scan_i32(ws, count, cell_start, ncells);
    if (n > 0) {
      k_scatter<<<grid_for(n, 256), 256, 0, st>>>(n, ws->cellid.as<int>(), ws->slot.as<int>(), cell_start,
                                                   ws->tmp_idx.as<int>());
      ws->launches += 1;
    }
    if (ncells > 0) {
      k_cell_order<<<grid_for((int64_t)ncells * 32, 256), 256, 0, st>>>(
          (int)ncells, dsys, nsys, cell_start, ws->tmp_idx.as<int>(), ws->wrapped.as<double>(), ws->species.as<int>(),
          ws->perm.as<int>(), ws->pos.as<double4>(), ws->inverse.as<int>(), ws->cell_sys.as<int>(), bad + 4,
          ws->species_limit, bad + 2);
      ws->launches += 1;
    }
    PFW_CUDA(cudaGetLastError());
    return;
  }
  // after the open-axis pre-pass (k_atom_sys, k_wrap, k_open_minmax in
  // prepare_plan): key, scan, placement, gather
  PFW_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (ncells + 1), st));
  if (n > 0) {
    k_key_count<<<grid_for(n, 256), 256, 0, st>>>(n, atom_sys, dsys, bincoord, ws->cellid.as<int>(),
                                                  ws->slot.as<int>(), count, bad);
    ws->launches += 1;
  }
  exclusive_scan_i32(ws, count, cell_start, ncells);
  if (n > 0) {
    k_scatter<<<grid_for(n, 256), 256, 0, st>>>(n, ws->cellid.as<int>(), ws->slot.as<int>(), cell_start,
                                                 ws->tmp_idx.as<int>());
    k_cell_rank<<<grid_for((int64_t)ncells * 32, 256), 256, 0, st>>>((int)ncells, cell_start, ws->tmp_idx.as<int>(),
                                                                      ws->perm.as<int>());
    k_gather<<<grid_for(n, 256), 256, 0, st>>>(n, ws->perm.as<int>(), ws->wrapped.as<double>(),
                                               ws->species.as<int>(), ws->pos.as<double4>(), ws->inverse.as<int>(),
                                               ws->species_limit, bad + 2);
    ws->launches += 3;
  }
  if (ncells > 0) {
    k_cell_sys<<<grid_for(ncells, 256), 256, 0, st>>>(dsys, nsys, (int)ncells, ws->cell_sys.as<int>(), cell_start,
                                                      bad + 4);
    ws->launches += 1;
  }
  PFW_CUDA(cudaGetLastError());
}

// Synchronise and turn the device flags of the build into errors.
static void raise_prepare_flags(pfw_ws* ws, const int* hbad) {
  if (hbad[0] == 1) throw Error(PFW_EINVAL, "positions must be finite");
  if (hbad[0] == 2) throw Error(PFW_EINVAL, "atom outside the open-axis cell grid");
  if (hbad[2])
    throw Error(PFW_EINVAL, "species channel outside the model's channels (must be >= 0 and < " +
                                std::to_string(ws->species_limit) + ")");
  ws->prep.max_cell = hbad[4];
}

void prepare_check(pfw_ws* ws) {
  if (ws->defer_check) {
    if (!ws->flags_host) PFW_CUDA(cudaMallocHost(&ws->flags_host, 8 * sizeof(int32_t)));
    PFW_CUDA(cudaMemcpyAsync(ws->flags_host, ws->counters.ptr, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             ws->stream));
    ws->check_pending = true;
    return;
  }
  int hbad[8];
  PFW_CUDA(cudaMemcpyAsync(hbad, ws->counters.ptr, sizeof(hbad), cudaMemcpyDeviceToHost, ws->stream));
  PFW_CUDA(cudaStreamSynchronize(ws->stream));
  PFW_CUDA(cudaGetLastError());
  raise_prepare_flags(ws, hbad);
}

void prepare_check_finish(pfw_ws* ws) {
  if (!ws->check_pending) return;
  ws->check_pending = false;
  PFW_CUDA(cudaGetLastError());
  try {
    raise_prepare_flags(ws, ws->flags_host);
  } catch (...) {
    ws->prep.valid = false;  // the cell list of a rejected input is not reused
    throw;
  }
}

void prepare(pfw_ws* ws, double cutoff) {
  Prepared& P = ws->prep;
  if (P.valid && P.cutoff == cutoff && P.species_limit == ws->species_limit) return;
  const bool wrapped = prepare_plan(ws, cutoff);
  prepare_launch(ws, !wrapped);
  prepare_check(ws);
  P.valid = true;
}

}  // namespace pfw
