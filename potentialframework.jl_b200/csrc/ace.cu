// ace.cu — ACE site energy, force and virial on the device.
//
// Replaces the prepared ACE executor (ACE/cpu.jl:162-275 NI.evaluate_site!,
// execute_prepared_impl!; ACE/serial.jl:260-366 site_data/site_reverse) and
// the reference's AMD kernels (ACE/gpu.jl: ace_density!, ace_products!,
// ace_edges!) with:
//
//   k_edge_count/scan/k_edge_fill  complete directed environments (the
//                 neighbour snapshot, NeighbourList/environments.jl:33-76) as a
//                 CSR over sorted centres; edge displacement X_j - X_i + H·S
//                 from the ORIGINAL coordinates (environments.jl:97-102)
//   k_edge_rev    index of the reverse edge (j→i, -S) of every edge
//   k_ace_sites   persistent site kernel (ace_site.cuh) over work units (one
//                 site, or up to 8 sites of one system of a batch)
//   k_ace_gather  F_k = Σ_{e∈out(k)} g_e - g_{rev(e)}  (reduce_site!,
//                 NeighbourList/execution.jl:256-273, without a racing scatter)
//   reduce_site_parts  E and the 3×3 virial from per-site partials (reduce.cu)
//
// Batches of systems evaluate in units that never span two systems, summed
// per system in a fixed order, so energies, virials and the per-structure
// fitting features (ACE/fitting.jl:28-29) come out per system; the batch path
// can be captured once as a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ace_design.cuh"
#include "ace_math.cuh"
#include "ace_site.cuh"
#include "mlp_tc.cuh"
#include "pfw_internal.h"
#include "traverse.cuh"

namespace pfw {

// What a captured batch graph was recorded for.
struct GraphKey {
  uint64_t geometry_version = ~0ull;
  uint64_t alloc_epoch = ~0ull;
  const void *E = nullptr, *F = nullptr, *W = nullptr, *feat = nullptr;
  uint32_t req = 0;
  int chunk = 0, groups = 0, precision = 0;
  bool operator==(const GraphKey& o) const {
    return geometry_version == o.geometry_version && alloc_epoch == o.alloc_epoch && E == o.E && F == o.F &&
           W == o.W && feat == o.feat && req == o.req && chunk == o.chunk && groups == o.groups && precision == o.precision;
  }
};

struct AceDevice {
  int nz = 0, lmax = 0, nY = 0, nR = 0, nQ = 0, D = 0, P = 0, T = 0, nB = 0, max_order = 0, solid = 0;
  double cutoff = 0;
  RadialDev R{}, Q{};
  DevBuf r_len, r_nodes, r_coeff, r_tr, r_pow, r_envk, r_env;
  DevBuf q_len, q_nodes, q_coeff, q_tr, q_pow, q_envk, q_env;
  DevBuf r_coeff32, q_coeff32, weights32;  // FP32 copies for the mixed form
  DevBuf density, dn_off, dn, dm_off, dm, prods, term_off, terms, weights, wpair, ref, pair_ok, Fnorm;
  DevBuf crow_off, crow_k, crow_val;
  // per evaluation
  DevBuf edge_count, edge_off, edge_j, edge_d, edge_S, edge_rev, edge_g, site_out, site_E_orig, status;
  DevBuf edge_countp;  // per stencil part (but the last) and atom: the part's edge count
  int edge_parts = 1;
  DevBuf unit_begin, unit_out;  // single system: one unit per site
  // batch: units of at most BATCH_UNIT_SITES sites, never spanning two systems
  DevBuf batch_units, batch_sys_units, batch_out, batch_feat;
  DevBuf design_G;      // design rows: product factor gradients, one row per site group
  DevBuf design_order;  // design rows: systems largest first, then the work counter
  uint64_t batch_version = ~0ull;
  int batch_nunits = 0;
  std::vector<int> h_batch_units, h_batch_sys_units;
  std::vector<SysGeom> graph_sys;  // cell-list plan the graph was captured with
  int64_t nedges = 0;
  int cap = 0;  // edge capacity of the buffers
  int n = 0;
  bool evaluated = false;
  int sched_chunk = 0, sched_groups = 0;  // 0: automatic
  // captured batch evaluation
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  GraphKey graph_key{};
  uint64_t graph_kernels = 0;
};

// ---------------------------------------------------------------------------
// environments
// ---------------------------------------------------------------------------
// Environments of a home cell's atoms over one part of the stencil (the
// stencil split in order into `parts` ranges, one warp each): the edge count
// of every atom is added to count (integers: order-free), and the part's own
// count is kept in countp[part][atom] for the parts after it.
template <int MODE>
__global__ void __launch_bounds__(128)
    k_edge_count(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
                 const double4* __restrict__ pos, int ncells, int parts, int natoms, int* __restrict__ count,
                 int* __restrict__ countp) {
  __shared__ WarpStage stage[4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * 4 + warp;
  const int cell = w / parts, part = w - cell * parts;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  int cur = -1, cnt = 0;
  auto flush = [&]() {
    if (cur < 0) return;
    if (parts == 1) {
      count[cur] = cnt;
    } else {
      atomicAdd(count + cur, cnt);
      if (part < parts - 1) countp[(size_t)part * natoms + cur] = cnt;
    }
  };
  warp_traverse_cell<MODE>(
      g, cell, cell_start, pos, stage[warp], lane,
      [&](int i, int, const double4&, const double4&, const StencilEntry&, const double*, double) {
        if (i != cur) {
          flush();
          cur = i;
          cnt = 0;
        }
        ++cnt;
      },
      part, parts);
  flush();
}

// Writes edges below `cap` only; an edge past the capacity sets status bit 8.
// A part's edges of atom i start after the earlier parts' (countp).
template <int MODE>
__global__ void __launch_bounds__(128)
    k_edge_fill(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
                const double4* __restrict__ pos, const int* __restrict__ perm, const int* __restrict__ wind,
                const double* __restrict__ X, int ncells, int parts, int natoms, const int* __restrict__ countp,
                const int* __restrict__ off, int cap, int* __restrict__ ej, int4* __restrict__ eS,
                double4* __restrict__ ed, int* __restrict__ status) {
  __shared__ WarpStage stage[4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * 4 + warp;
  const int cell = w / parts, part = w - cell * parts;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  int cur = -1, o = 0, a = 0;
  int wi[3] = {0, 0, 0};
  double xi[3] = {0, 0, 0};
  warp_traverse_cell<MODE>(
      g, cell, cell_start, pos, stage[warp], lane,
      [&](int i, int j, const double4& pi, const double4& pj, const StencilEntry& se, const double*, double) {
        if (i != cur) {
          cur = i;
          o = off[i];
          for (int q = 0; q < part; ++q) o += countp[(size_t)q * natoms + i];
          a = perm[i];
          wi[0] = wind[3 * a]; wi[1] = wind[3 * a + 1]; wi[2] = wind[3 * a + 2];
          xi[0] = X[3 * a]; xi[1] = X[3 * a + 1]; xi[2] = X[3 * a + 2];
        }
        if (o >= cap) {
          atomicOr(status, 8);
          ++o;
          return;
        }
        const int b = perm[j];
        const int wj[3] = {wind[3 * b], wind[3 * b + 1], wind[3 * b + 2]};
        int S[3];
        pair_image(g, se, pi, pj, wi, wj, S);
        // edge_displacement: X_j - X_i + Hz·S ((t1 + t2) + t3)
        double sh[3];
        xmatvec(g.Hz, (double)S[0], (double)S[1], (double)S[2], sh);
        ej[o] = j;
        eS[o] = make_int4(S[0], S[1], S[2], 0);
        ed[o] = make_double4(xadd(xsub(X[3 * b], xi[0]), sh[0]), xadd(xsub(X[3 * b + 1], xi[1]), sh[1]),
                             xadd(xsub(X[3 * b + 2], xi[2]), sh[2]), pj.w);
        ++o;
      },
      part, parts);
}

// Reverse edge of e = (i→j, S): the entry (j→i, -S) of j's list.  One warp
// per atom, a lane per edge; j's list is scanned four entries per step so
// that four loads are in flight.
__global__ void k_edge_rev(int n, const int* __restrict__ off, int cap, const int* __restrict__ ej,
                           const int4* __restrict__ eS, int* __restrict__ rev, int* __restrict__ status) {
  const int i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int e1 = min(off[i + 1], cap);
  for (int e = min(off[i], cap) + lane; e < e1; e += 32) {
    const int j = ej[e];
    const int4 s = eS[e];
    int found = -1;
    const int f1 = min(off[j + 1], cap);
    for (int f = min(off[j], cap); f < f1 && found < 0; f += 4) {
      int c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) c[u] = f + u < f1 ? ej[f + u] : -1;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (found < 0 && c[u] == i) {
          const int4 t = eS[f + u];
          if (t.x == -s.x && t.y == -s.y && t.z == -s.z) found = f + u;
        }
      }
    }
    if (found < 0) atomicOr(status, 4);
    rev[e] = found < 0 ? e : found;
  }
}

// F_k = Σ_{e ∈ out(k)} g_e - g_rev(e), written in original order.  Eight
// lanes per atom stride over its out-edges; their sums are combined by a
// fixed three-step shuffle tree, so the order of every addition is fixed.
constexpr int GATHER_LANES = 8;

__global__ void k_ace_gather(int n, const int* __restrict__ off, int cap, const int* __restrict__ rev,
                             const double* __restrict__ g, const int* __restrict__ perm, double* __restrict__ F) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = t / GATHER_LANES, q = t % GATHER_LANES;
  double f0 = 0, f1 = 0, f2 = 0;
  if (k < n) {
    const int e1 = min(off[k + 1], cap);
    for (int e = min(off[k], cap) + q; e < e1; e += GATHER_LANES) {
      const int r = rev[e];
      f0 += g[3 * (size_t)e] - g[3 * (size_t)r];
      f1 += g[3 * (size_t)e + 1] - g[3 * (size_t)r + 1];
      f2 += g[3 * (size_t)e + 2] - g[3 * (size_t)r + 2];
    }
  }
#pragma unroll
  for (int o = GATHER_LANES / 2; o > 0; o >>= 1) {
    f0 += __shfl_xor_sync(0xffffffffu, f0, o);
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
  }
  if (k < n && q == 0) {
    const int o = perm[k];
    F[3 * o] = f0;
    F[3 * o + 1] = f1;
    F[3 * o + 2] = f2;
  }
}

// Site energies in original order.
__global__ void k_site_energies(int n, const double* __restrict__ site_out, const int* __restrict__ perm,
                                double* __restrict__ Esite) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) Esite[perm[s]] = site_out[10 * (size_t)s];
}

__global__ void k_mask_sites(int n, int n_owned, const int* __restrict__ perm, double* __restrict__ site_out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * 10) return;
  if (perm[k / 10] >= n_owned) site_out[k] = 0.0;
}

void mask_unowned_sites(pfw_ws* ws, double* site_out, int n) {
  if (ws->n_owned < 0 || ws->n_owned >= n || n == 0) return;
  k_mask_sites<<<grid_for((int64_t)n * 10, 256), 256, 0, ws->stream>>>(n, ws->n_owned, ws->perm.as<int>(), site_out);
  ws->launches += 1;
}

__global__ void k_iota(int n, int* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k <= n) out[k] = k;
}

// Per-system totals of a batch: the units of system s, summed in unit order
// (deterministic), give E[s], W[9s..9s+8] and the fitting features.
__global__ void k_system_reduce(int nsys, const int* __restrict__ sys_units, const double* __restrict__ unit_out,
                                const double* __restrict__ unit_feat, int nfeat, double* __restrict__ E,
                                double* __restrict__ W, double* __restrict__ feat) {
  const int s = blockIdx.x;
  if (s >= nsys) return;
  const int u0 = sys_units[s], u1 = sys_units[s + 1];
  const int ncol = 10 + (feat ? nfeat : 0);
  for (int k = threadIdx.x; k < ncol; k += blockDim.x) {
    double acc = 0.0;
    if (k < 10)
      for (int u = u0; u < u1; ++u) acc += unit_out[10 * (size_t)u + k];
    else
      for (int u = u0; u < u1; ++u) acc += unit_feat[(size_t)nfeat * u + (k - 10)];
    if (k == 0) {
      if (E) E[s] = acc;
    } else if (k < 10) {
      if (W) W[9 * (size_t)s + k - 1] = acc;
    } else {
      feat[(size_t)nfeat * s + k - 10] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
template <class T>
static T* upload(DevBuf& b, const T* src, size_t count, cudaStream_t st) {
  T* d = static_cast<T*>(b.ensure(sizeof(T) * std::max<size_t>(count, 1)));
  if (count) PFW_CUDA(cudaMemcpyAsync(d, src, sizeof(T) * count, cudaMemcpyHostToDevice, st));
  return d;
}

static RadialDev upload_family(const pfw_radial_family& f, int nz, DevBuf& len, DevBuf& nodes, DevBuf& coeff,
                               DevBuf& coeff32, DevBuf& tr, DevBuf& pw, DevBuf& ek, DevBuf& ev, cudaStream_t st) {
  if (f.nchannels < 0 || f.nknots < 2) throw Error(PFW_EINVAL, "invalid radial family shape");
  const int np = nz * nz;
  for (int k = 0; k < np; ++k) {
    if (f.lengths[k] < 2 || f.lengths[k] > f.nknots) throw Error(PFW_EINVAL, "invalid spline node count");
    const int kind = f.envelope_kind[k];
    if (kind < 1 || kind > 3) throw Error(PFW_EINVAL, "unsupported radial envelope");
    if (f.powers[2 * k] <= 0 || f.powers[2 * k + 1] < f.powers[2 * k]) throw Error(PFW_EINVAL, "invalid Agnesi transform");
    // read_radial's node rule (ACE/resolved.jl:80-81): -1 = first < ... < last = 1
    const double* nd = f.nodes + (size_t)k * f.nknots;
    bool sorted = nd[0] == -1.0 && nd[f.lengths[k] - 1] == 1.0;
    for (int i = 1; i < f.lengths[k]; ++i) sorted = sorted && nd[i] > nd[i - 1];
    if (!sorted) throw Error(PFW_EINVAL, "spline nodes must increase from -1 to 1");
  }
  RadialDev d;
  d.nch = f.nchannels;
  d.nknots = f.nknots;
  d.nz = nz;
  d.lengths = upload(len, f.lengths, np, st);
  d.nodes = upload(nodes, f.nodes, (size_t)np * f.nknots, st);
  const size_t ncoeff = (size_t)np * (f.nknots - 1) * f.nchannels * 4;
  d.coeff = upload(coeff, f.coeff, ncoeff, st);
  {
    std::vector<float> c32(std::max<size_t>(ncoeff, 1));
    for (size_t i = 0; i < ncoeff; ++i) c32[i] = (float)f.coeff[i];
    d.coeff32 = upload(coeff32, c32.data(), c32.size(), st);
    PFW_CUDA(cudaStreamSynchronize(st));  // the staging vector goes out of scope
  }
  d.transform = upload(tr, f.transform, (size_t)np * 6, st);
  d.powers = upload(pw, f.powers, (size_t)np * 2, st);
  d.env_kind = upload(ek, f.envelope_kind, np, st);
  d.env = upload(ev, f.envelope, (size_t)np * 5, st);
  return d;
}

static void release_graph(AceDevice* a) {
  if (a->graph_exec) cudaGraphExecDestroy(a->graph_exec);
  if (a->graph) cudaGraphDestroy(a->graph);
  a->graph_exec = nullptr;
  a->graph = nullptr;
  a->graph_key = GraphKey{};
}

static void free_device(AceDevice* a) {
  if (!a) return;
  release_graph(a);
  DevBuf* bufs[] = {&a->r_len, &a->r_nodes, &a->r_coeff, &a->r_tr, &a->r_pow, &a->r_envk, &a->r_env,
                    &a->q_len, &a->q_nodes, &a->q_coeff, &a->q_tr, &a->q_pow, &a->q_envk, &a->q_env,
                    &a->density, &a->dn_off, &a->dn, &a->dm_off, &a->dm, &a->prods, &a->term_off, &a->terms,
                    &a->weights, &a->weights32, &a->r_coeff32, &a->q_coeff32, &a->wpair, &a->ref, &a->pair_ok, &a->Fnorm, &a->crow_off, &a->crow_k, &a->crow_val,
                    &a->edge_count, &a->edge_countp, &a->edge_off, &a->edge_j, &a->edge_d, &a->edge_S, &a->edge_rev, &a->edge_g,
                    &a->site_out, &a->site_E_orig, &a->status, &a->unit_begin, &a->unit_out,
                    &a->batch_units, &a->batch_sys_units, &a->batch_out, &a->batch_feat, &a->design_G,
                    &a->design_order};
  for (auto* b : bufs) b->release();
  delete a;
}

void ace_free(pfw_ws* ws) {
  free_device(ws->ace);
  ws->ace = nullptr;
}

static void fill_model(pfw_ws* ws, AceDevice* a, const pfw_ace_tables* t);

// Validated device copy of packed ACE tables (pack_model, ACE/adaptation.jl:78-98).
static AceDevice* load_model(pfw_ws* ws, const pfw_ace_tables* t) {
  if (t->nz < 1 || t->nz > 16) throw Error(PFW_EINVAL, "ACE models support 1 to 16 species channels");
  if (t->lmax < 0 || t->lmax > ACE_LMAX) throw Error(PFW_EINVAL, "ACE lmax must be in 0..6");
  if (t->angular_kind != 0 && t->angular_kind != 1)
    throw Error(PFW_EINVAL, "angular kind must be 0 (real spherical) or 1 (real solid)");
  if (t->radial.nchannels < 1) throw Error(PFW_EINVAL, "empty radial basis");
  if (!(std::isfinite(t->cutoff) && t->cutoff > 0)) throw Error(PFW_EINVAL, "invalid ACE cutoff");
  if (t->ndensity < 1 || t->ndensity > 65534 || t->nproducts < 1 || t->nproducts > 65535)
    throw Error(PFW_EINVAL, "ACE basis size out of range (density <= 65534, products <= 65535)");
  AceDevice* a = new AceDevice();
  try {
    fill_model(ws, a, t);
  } catch (...) {
    free_device(a);
    throw;
  }
  return a;
}

void ace_load(pfw_ws* ws, const pfw_ace_tables* t) {
  AceDevice* a = load_model(ws, t);
  ace_free(ws);
  ws->ace = a;
}

static void fill_model(pfw_ws* ws, AceDevice* a, const pfw_ace_tables* t) {
  cudaStream_t st = ws->stream;
  const int nz = t->nz;
  a->nz = nz;
  a->lmax = t->lmax;
  a->solid = t->angular_kind;
  a->nY = (t->lmax + 1) * (t->lmax + 1);
  a->nR = t->radial.nchannels;
  a->nQ = t->pair.nchannels;
  a->D = t->ndensity;
  a->P = t->nproducts;
  a->nB = t->nbasis;
  a->cutoff = t->cutoff;
  a->R = upload_family(t->radial, nz, a->r_len, a->r_nodes, a->r_coeff, a->r_coeff32, a->r_tr, a->r_pow, a->r_envk,
                       a->r_env, st);
  if (a->nQ > 0)
    a->Q = upload_family(t->pair, nz, a->q_len, a->q_nodes, a->q_coeff, a->q_coeff32, a->q_tr, a->q_pow, a->q_envk,
                         a->q_env, st);
  else
    a->Q = a->R;
  // density tables, grouped by radial channel and by harmonic
  std::vector<int2> dens(a->D);
  for (int k = 0; k < a->D; ++k) {
    const int n = t->density[2 * k], m = t->density[2 * k + 1];
    if (n < 0 || n >= a->nR || m < 0 || m >= a->nY) throw Error(PFW_EINVAL, "invalid density indices");
    dens[k] = make_int2(n, m);
  }
  upload(a->density, dens.data(), dens.size(), st);
  std::vector<int> dn_off(a->nR + 1, 0), dm_off(a->nY + 1, 0);
  for (auto& d : dens) {
    dn_off[d.x + 1]++;
    dm_off[d.y + 1]++;
  }
  for (int k = 0; k < a->nR; ++k) dn_off[k + 1] += dn_off[k];
  for (int k = 0; k < a->nY; ++k) dm_off[k + 1] += dm_off[k];
  std::vector<int2> dn(a->D), dm(a->D);
  {
    std::vector<int> fn(dn_off.begin(), dn_off.end() - 1), fm(dm_off.begin(), dm_off.end() - 1);
    for (int k = 0; k < a->D; ++k) {
      dn[fn[dens[k].x]++] = make_int2(k, dens[k].y);
      dm[fm[dens[k].y]++] = make_int2(k, dens[k].x);
    }
  }
  upload(a->dn_off, dn_off.data(), dn_off.size(), st);
  upload(a->dn, dn.data(), dn.size(), st);
  upload(a->dm_off, dm_off.data(), dm_off.size(), st);
  upload(a->dm, dm.data(), dm.size(), st);
  // products (≤ 4 factors, sentinel D) and the adjoint terms of each density:
  // one term per occurrence of a in product k, holding the other factors
  const int* poff = t->product_offsets;
  if (poff[0] != 0) throw Error(PFW_EINVAL, "product offsets must start at 0");
  const unsigned short SENT = (unsigned short)a->D;
  std::vector<ushort4> prods(a->P);
  std::vector<std::vector<ushort4>> per(a->D);
  for (int k = 0; k < a->P; ++k) {
    const int nu = poff[k + 1] - poff[k];
    if (nu < 1) throw Error(PFW_EINVAL, "empty ACE product");
    if (nu > 4) throw Error(PFW_EINVAL, "ACE correlation order above 4 is not supported");
    a->max_order = std::max(a->max_order, nu);
    unsigned short f[4] = {SENT, SENT, SENT, SENT};
    for (int q = 0; q < nu; ++q) {
      const int v = t->product_factors[poff[k] + q];
      if (v < 0 || v >= a->D) throw Error(PFW_EINVAL, "invalid product indices");
      f[q] = (unsigned short)v;
    }
    prods[k] = make_ushort4(f[0], f[1], f[2], f[3]);
    for (int q = 0; q < nu; ++q) {
      unsigned short o[3] = {SENT, SENT, SENT};
      int c = 0;
      for (int u = 0; u < nu; ++u)
        if (u != q) o[c++] = f[u];
      per[f[q]].push_back(make_ushort4((unsigned short)k, o[0], o[1], o[2]));
    }
  }
  std::vector<int> toff(a->D + 1, 0);
  std::vector<ushort4> terms;
  for (int d = 0; d < a->D; ++d) {
    toff[d + 1] = toff[d] + (int)per[d].size();
    terms.insert(terms.end(), per[d].begin(), per[d].end());
  }
  a->T = (int)terms.size();
  upload(a->prods, prods.data(), prods.size(), st);
  upload(a->term_off, toff.data(), toff.size(), st);
  upload(a->terms, terms.data(), terms.size(), st);
  // precontracted weights w[z][k] = Σ_b C[b,k]·WB[z][b] (ACE/cpu.jl:265-268) and
  // the coupling by invariant row (fitting features B = C·P)
  std::vector<double> wts((size_t)nz * a->P, 0.0);
  std::vector<int> roff(a->nB + 1, 0);
  for (int e = 0; e < t->ncoupling; ++e) {
    const int r = t->coupling_rows[e], c = t->coupling_cols[e];
    if (r < 0 || r >= a->nB || c < 0 || c >= a->P) throw Error(PFW_EINVAL, "invalid coupling entry");
    roff[r + 1]++;
    for (int z = 0; z < nz; ++z) wts[(size_t)z * a->P + c] += t->coupling_vals[e] * t->WB[(size_t)z * a->nB + r];
  }
  for (int b = 0; b < a->nB; ++b) roff[b + 1] += roff[b];
  std::vector<int> rk(t->ncoupling);
  std::vector<double> rv(t->ncoupling);
  {
    std::vector<int> fill(roff.begin(), roff.end() - 1);
    for (int e = 0; e < t->ncoupling; ++e) {
      const int q = fill[t->coupling_rows[e]]++;
      rk[q] = t->coupling_cols[e];
      rv[q] = t->coupling_vals[e];
    }
  }
  upload(a->weights, wts.data(), wts.size(), st);
  const std::vector<float> w32(wts.begin(), wts.end());  // alive until the synchronisation below
  upload(a->weights32, w32.data(), w32.size(), st);
  upload(a->crow_off, roff.data(), roff.size(), st);
  upload(a->crow_k, rk.data(), rk.size(), st);
  upload(a->crow_val, rv.data(), rv.size(), st);
  upload(a->wpair, t->Wpair, (size_t)nz * a->nQ, st);
  upload(a->ref, t->reference, nz, st);
  std::vector<int> pok(nz);
  for (int z = 0; z < nz; ++z) pok[z] = t->pair_allowed[z] ? 1 : 0;
  upload(a->pair_ok, pok.data(), pok.size(), st);
  // BlockAngular normalisation F[l,0] = sqrt((2l+1)/2π), F[l,m] = -F[l,m-1]/sqrt((l+m)(l+1-m))
  const int L = a->lmax;
  std::vector<double> F((L + 1) * (L + 1), 0.0);
  const double twopi = 6.283185307179586;
  for (int l = 0; l <= L; ++l) {
    F[l * (L + 1)] = std::sqrt((double)(2 * l + 1) / twopi);
    for (int m = 1; m <= l; ++m) F[l * (L + 1) + m] = -F[l * (L + 1) + m - 1] / std::sqrt((double)((l + m) * (l + 1 - m)));
  }
  upload(a->Fnorm, F.data(), F.size(), st);
  PFW_CUDA(cudaStreamSynchronize(st));
}

static AceTables tables_of(AceDevice* a) {
  AceTables p;
  p.R = a->R;
  p.Q = a->Q;
  p.nz = a->nz;
  p.nY = a->nY;
  p.nR = a->nR;
  p.nQ = a->nQ;
  p.D = a->D;
  p.P = a->P;
  p.T = a->T;
  p.nB = a->nB;
  p.prods = a->prods.as<ushort4>();
  p.term_off = a->term_off.as<int>();
  p.terms = a->terms.as<ushort4>();
  p.density = a->density.as<int2>();
  p.dn_off = a->dn_off.as<int>();
  p.dn = a->dn.as<int2>();
  p.dm_off = a->dm_off.as<int>();
  p.dm = a->dm.as<int2>();
  p.weights = a->weights.as<double>();
  p.weights32 = a->weights32.as<float>();
  p.crow_off = a->crow_off.as<int>();
  p.crow_k = a->crow_k.as<int>();
  p.crow_val = a->crow_val.as<double>();
  p.wpair = a->wpair.as<double>();
  p.ref = a->ref.as<double>();
  p.pair_ok = a->pair_ok.as<int>();
  p.Fnorm = a->Fnorm.as<double>();
  p.solid = a->solid;
  return p;
}

// Largest working set that fits (or the tuned schedule): site groups of ACE_GROUP
// threads per CTA and edges per chunk.
static AceLayout choose_layout(const AceTables& p, int device, int chunk, int groups, int feat) {
  int optin = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  const size_t limit = (size_t)optin;
  // tables staged in shared memory first; models whose adjoint terms (then
  // products) do not fit read them from global memory instead
  const int gtabs[] = {0, 1, 3};
  if (chunk > 0) {
    for (int gt : gtabs) {
      AceLayout lay;
      lay.make(p, chunk, groups, feat, 0, gt);
      if (lay.total <= limit) return lay;
    }
    if (!feat) throw Error(PFW_EINVAL, "ACE schedule does not fit in shared memory");
  }
  const int cand128[][2] = {{32, 2}, {16, 3}, {16, 2}, {32, 1}, {16, 1}, {8, 1}};
  const int cand64[][2] = {{16, 6}, {16, 4}, {8, 8}, {16, 3}, {8, 4}, {16, 2}, {8, 2}, {8, 1}};
  const int (*cand)[2] = ACE_GROUP == 128 ? cand128 : cand64;
  const int ncand = ACE_GROUP == 128 ? 6 : 8;
  for (int k = 0; k < ncand; ++k)  // the largest working set that fits, tables staged where they fit
    for (int gt : gtabs) {
      AceLayout lay;
      lay.make(p, cand[k][0], cand[k][1], feat, 0, gt);
      if (lay.total <= limit) return lay;
    }
  throw Error(PFW_EINVAL, "ACE model too large for the site kernel's shared memory");
}

void ace_set_schedule(pfw_ws* ws, int chunk, int groups) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  if (chunk == 0 && groups == 0) {
    a->sched_chunk = a->sched_groups = 0;
    release_graph(a);
    return;
  }
  if (!(chunk == 8 || chunk == 16 || chunk == 32) || chunk > ACE_MAX_CHUNK || groups < 1 || groups > ACE_MAX_GROUPS)
    throw Error(PFW_EINVAL, "ACE schedule: chunk 8, 16 or 32 (at most a quarter of a site group's threads) and "
                            "groups 1.." + std::to_string(ACE_MAX_GROUPS));
  choose_layout(tables_of(a), ws->opt.device, chunk, groups, 0);  // validates the fit
  a->sched_chunk = chunk;
  a->sched_groups = groups;
  release_graph(a);
}

struct SiteLaunch {
  int nunits;
  const int* unit_begin;
  const int* unit_sites;  // non-null: unit u is the single site unit_sites[u]
  int cap;
  const int* off;
  const double4* ed;
  const double4* pos;
  double* g;
  double* unit_out;
  double* unit_feat;
  int want_grad;
  int* status;
  SurParams sur;
};

template <int L, class T, int SUR>
static void launch_sites(const AceTables& p, const AceLayout& lay, const SiteLaunch& s, cudaStream_t st, int device) {
  auto kern = k_ace_sites<L, T, SUR>;
  PFW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay.total));
  int sms = 0, per_sm = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  PFW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ACE_GROUP * lay.G, lay.total));
  per_sm = std::max(per_sm, 1);
  const int blocks = std::max(1, std::min(sms * per_sm, (s.nunits + lay.G - 1) / lay.G));
  kern<<<blocks, ACE_GROUP * lay.G, lay.total, st>>>(p, lay, s.sur, s.nunits, s.unit_begin, s.unit_sites, s.cap, s.off,
                                                     s.ed, s.pos, s.g, s.unit_out, s.unit_feat, s.want_grad, s.status);
}

template <class T, int SUR = 0>
static void dispatch_sites(int lmax, const AceTables& p, const AceLayout& lay, const SiteLaunch& s, cudaStream_t st,
                           int device) {
  switch (lmax) {
    case 0: launch_sites<0, T, SUR>(p, lay, s, st, device); break;
    case 1: launch_sites<1, T, SUR>(p, lay, s, st, device); break;
    case 2: launch_sites<2, T, SUR>(p, lay, s, st, device); break;
    case 3: launch_sites<3, T, SUR>(p, lay, s, st, device); break;
    case 4: launch_sites<4, T, SUR>(p, lay, s, st, device); break;
    case 5: launch_sites<5, T, SUR>(p, lay, s, st, device); break;
    default: launch_sites<6, T, SUR>(p, lay, s, st, device); break;
  }
}

static bool shift_mode(const Prepared& P) {
  for (auto& g : P.sys)
    if (g.minimum_image && !g.fast_shift) return false;
  return true;
}

// Stencil parts per home cell for the environment kernels: enough warps to
// fill the GPU when the cells are few (at most 3 parts of the 27 entries).
static int edge_parts(const Prepared& P) {
  const int want = 148 * 16;
  return std::max(1, std::min(3, (want + std::max(P.ncells, 1) - 1) / std::max(P.ncells, 1)));
}

// count + scan of the environments (no host synchronisation)
static void edges_count_launch(pfw_ws* ws, AceDevice* a) {
  const Prepared& P = ws->prep;
  cudaStream_t st = ws->stream;
  const int n = P.n;
  const int parts = edge_parts(P);
  int* count = a->edge_count.as<int>();
  int* countp = static_cast<int*>(a->edge_countp.ensure(sizeof(int) * (size_t)std::max(n, 1) * std::max(parts - 1, 1)));
  PFW_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * std::max(n, 1), st));
  if (parts > 1) PFW_CUDA(cudaMemsetAsync(countp, 0, sizeof(int) * (size_t)n * (parts - 1), st));
  const dim3 grid(grid_for((int64_t)P.ncells * parts, 4)), block(128);
  if (P.ncells > 0) {
    if (shift_mode(P))
      k_edge_count<0><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(),
                                              ws->cell_start.as<int>(), ws->pos.as<double4>(), P.ncells, parts, n,
                                              count, countp);
    else
      k_edge_count<1><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(),
                                              ws->cell_start.as<int>(), ws->pos.as<double4>(), P.ncells, parts, n,
                                              count, countp);
    ws->launches += 1;
  }
  a->edge_parts = parts;
  exclusive_scan_i32(ws, count, a->edge_off.as<int>(), n);
}

// fill + reverse index up to the buffer capacity (no host synchronisation)
static void edges_fill_launch(pfw_ws* ws, AceDevice* a) {
  const Prepared& P = ws->prep;
  cudaStream_t st = ws->stream;
  const int n = P.n;
  const int parts = a->edge_parts;
  const dim3 grid(grid_for((int64_t)P.ncells * parts, 4)), block(128);
  int* status = a->status.as<int>();
  const int* countp = a->edge_countp.as<int>();
  if (P.ncells > 0 && a->cap > 0) {
    if (shift_mode(P))
      k_edge_fill<0><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                             ws->pos.as<double4>(), ws->perm.as<int>(), ws->wind.as<int>(),
                                             ws->X.as<double>(), P.ncells, parts, n, countp, a->edge_off.as<int>(),
                                             a->cap, a->edge_j.as<int>(), a->edge_S.as<int4>(), a->edge_d.as<double4>(),
                                             status);
    else
      k_edge_fill<1><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                             ws->pos.as<double4>(), ws->perm.as<int>(), ws->wind.as<int>(),
                                             ws->X.as<double>(), P.ncells, parts, n, countp, a->edge_off.as<int>(),
                                             a->cap, a->edge_j.as<int>(), a->edge_S.as<int4>(), a->edge_d.as<double4>(),
                                             status);
    k_edge_rev<<<grid_for(n, 4), 128, 0, st>>>(n, a->edge_off.as<int>(), a->cap, a->edge_j.as<int>(),
                                               a->edge_S.as<int4>(), a->edge_rev.as<int>(), status);
    ws->launches += 2;
  }
}

static void ensure_edge_buffers(AceDevice* a, int cap) {
  a->cap = cap;
  a->edge_j.ensure(sizeof(int) * std::max(cap, 1));
  a->edge_S.ensure(sizeof(int4) * std::max(cap, 1));
  a->edge_d.ensure(sizeof(double4) * std::max(cap, 1));
  a->edge_rev.ensure(sizeof(int) * std::max(cap, 1));
  a->edge_g.ensure(sizeof(double) * 3 * std::max(cap, 1));
}

// Eager environments: count, read the total back, size the buffers, fill.
static void build_edges(pfw_ws* ws, AceDevice* a) {
  const int n = ws->prep.n;
  a->edge_count.ensure(sizeof(int) * std::max(n, 1));
  a->edge_off.ensure(sizeof(int) * (n + 1));
  a->status.ensure(sizeof(int) * 4);
  edges_count_launch(ws, a);
  int total = 0;
  PFW_CUDA(cudaMemcpyAsync(&total, a->edge_off.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, ws->stream));
  PFW_CUDA(cudaStreamSynchronize(ws->stream));
  a->nedges = total;
  ensure_edge_buffers(a, total);
  edges_fill_launch(ws, a);
}

// Site kernel, force gather and the per-unit outputs (no host synchronisation).
static void sites_launch(pfw_ws* ws, AceDevice* a, uint32_t req, int nunits, const int* unit_begin,
                         double* unit_out, double* unit_feat, const AceLayout& lay, double* F_dev) {
  cudaStream_t st = ws->stream;
  const int n = ws->prep.n;
  const bool want_grad = (req & (PFW_REQ_FORCES | PFW_REQ_VIRIAL)) != 0;
  const AceTables p = tables_of(a);
  SiteLaunch s{};
  s.nunits = nunits;
  s.unit_begin = unit_begin;
  s.unit_sites = nullptr;
  s.cap = a->cap;
  s.off = a->edge_off.as<int>();
  s.ed = a->edge_d.as<double4>();
  s.pos = ws->pos.as<double4>();
  s.g = a->edge_g.as<double>();
  s.unit_out = unit_out;
  s.unit_feat = unit_feat;
  s.want_grad = want_grad;
  s.status = a->status.as<int>();
  ws->stage_begin(1);
  if (nunits > 0) {
    if (ws->opt.precision == PFW_PRECISION_MIXED) dispatch_sites<float>(a->lmax, p, lay, s, st, ws->opt.device);
    else dispatch_sites<double>(a->lmax, p, lay, s, st, ws->opt.device);
    ws->launches += 1;
  }
  ws->stage_end(1);
  ws->stage_begin(2);
  if (F_dev && n > 0) {
    if (want_grad) {
      k_ace_gather<<<grid_for((int64_t)n * GATHER_LANES, 128), 128, 0, st>>>(n, a->edge_off.as<int>(), a->cap, a->edge_rev.as<int>(), s.g,
                                                     ws->perm.as<int>(), F_dev);
      ws->launches += 1;
    } else {
      PFW_CUDA(cudaMemsetAsync(F_dev, 0, sizeof(double) * 3 * n, st));
    }
  }
}

static void ace_check(pfw_ws* ws, AceDevice* a) {
  int hs[4];
  PFW_CUDA(cudaMemcpyAsync(hs, a->status.ptr, sizeof(hs), cudaMemcpyDeviceToHost, ws->stream));
  PFW_CUDA(cudaStreamSynchronize(ws->stream));
  PFW_CUDA(cudaGetLastError());
  if (hs[0] & 2) throw Error(PFW_EDOMAIN, "coincident physical atoms have undefined harmonics / pair envelope");
  if (hs[0] & 8) throw Error(PFW_ECAPACITY, "neighbour environments outgrew the planned capacity; re-plan");
  if (hs[0] & 4) throw Error(PFW_EINVAL, "internal: reverse edge not found");
  if (hs[0] & 16) throw Error(PFW_ETIMEDOUT, "a tensor-core wait of the surrogate MLP ran out");
}

void ace_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  check_species(ws, a->nz, "ACE model has no element channel for a species");
  cudaStream_t st = ws->stream;
  ws->prep.valid = false;
  ws->stage_begin(3);
  ws->stage_begin(0);
  prepare(ws, a->cutoff);
  ws->stage_end(0);
  a->status.ensure(sizeof(int) * 4);
  PFW_CUDA(cudaMemsetAsync(a->status.ptr, 0, sizeof(int) * 4, st));
  build_edges(ws, a);
  ws->stage_end(3);
  const int n = ws->prep.n;
  a->n = n;
  // one unit per site: unit_out holds the site partials
  int* ub = static_cast<int*>(a->unit_begin.ensure(sizeof(int) * (n + 1)));
  a->unit_out.ensure(sizeof(double) * 10 * std::max(n, 1));
  double* Esite = static_cast<double*>(a->site_E_orig.ensure(sizeof(double) * std::max(n, 1)));
  k_iota<<<grid_for(n + 1, 256), 256, 0, st>>>(n, ub);
  ws->launches += 1;
  const AceLayout lay = choose_layout(tables_of(a), ws->opt.device, a->sched_chunk, a->sched_groups, 0);
  sites_launch(ws, a, req, n, ub, a->unit_out.as<double>(), nullptr, lay, F_dev);
  double* E = E_dev ? E_dev : static_cast<double*>(ws->out_E.ensure(sizeof(double)));
  double* W = W_dev ? W_dev : static_cast<double*>(ws->out_W.ensure(sizeof(double) * 9));
  if (n > 0) {
    k_site_energies<<<grid_for(n, 256), 256, 0, st>>>(n, a->unit_out.as<double>(), ws->perm.as<int>(), Esite);
    ws->launches += 1;
  }
  mask_unowned_sites(ws, a->unit_out.as<double>(), n);
  reduce_site_parts(ws, a->unit_out.as<double>(), n, E, W);
  ws->stage_end(2);
  a->evaluated = true;
  ace_check(ws, a);
}

int ace_feature_count(pfw_ws* ws) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  return a->nz * (a->nB + a->nQ);
}

// Sites per work unit of a batch: small enough that large systems spread over
// many site groups, large enough that a unit's feature partials stay few.
#ifndef PFW_BATCH_UNIT_SITES
#define PFW_BATCH_UNIT_SITES 8
#endif
constexpr int BATCH_UNIT_SITES = PFW_BATCH_UNIT_SITES;

// Work units of the current batch.  In sorted order the sites of system s
// are [atom_begin_s, atom_begin_s + natoms_s) (its cells follow those of
// system s-1), so the units depend only on the atom counts.
static void plan_units(pfw_ws* ws, AceDevice* a) {
  if (a->batch_version == ws->geometry_version) return;
  auto& ub = a->h_batch_units;
  auto& su = a->h_batch_sys_units;
  ub.clear();
  su.clear();
  for (const auto& hs : ws->systems) {
    su.push_back((int)ub.size());
    for (int k = 0; k < hs.natoms; k += BATCH_UNIT_SITES) ub.push_back(hs.atom_begin + k);
  }
  su.push_back((int)ub.size());
  a->batch_nunits = (int)ub.size();
  ub.push_back(ws->n);
  upload(a->batch_units, ub.data(), ub.size(), ws->stream);
  upload(a->batch_sys_units, su.data(), su.size(), ws->stream);
  a->batch_version = ws->geometry_version;
}

// Site kernel, force gather and per-system totals of a planned batch
// (device work only; capturable).
static void batch_launch(pfw_ws* ws, AceDevice* a, uint32_t req, const AceLayout& lay, double* E_dev,
                         double* F_dev, double* W_dev, double* feat_dev) {
  const int nsys = (int)ws->systems.size(), nu = a->batch_nunits;
  const int nfeat = a->nz * (a->nB + a->nQ);
  double* feat_part = feat_dev ? a->batch_feat.as<double>() : nullptr;
  sites_launch(ws, a, req, nu, a->batch_units.as<int>(), a->batch_out.as<double>(), feat_part, lay, F_dev);
  k_system_reduce<<<nsys, 128, 0, ws->stream>>>(nsys, a->batch_sys_units.as<int>(), a->batch_out.as<double>(),
                                                 feat_part, nfeat, E_dev, W_dev, feat_dev);
  ws->launches += 1;
}

// Batch of systems.  Eager: plan, build, evaluate.
void ace_evaluate_batch(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev, double* feat_dev) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  check_species(ws, a->nz, "ACE model has no element channel for a species");
  cudaStream_t st = ws->stream;
  ws->prep.valid = false;
  prepare(ws, a->cutoff);
  a->status.ensure(sizeof(int) * 4);
  PFW_CUDA(cudaMemsetAsync(a->status.ptr, 0, sizeof(int) * 4, st));
  build_edges(ws, a);
  a->n = ws->prep.n;
  plan_units(ws, a);
  const size_t nu = std::max(a->batch_nunits, 1);
  a->batch_out.ensure(sizeof(double) * 10 * nu);
  if (feat_dev) a->batch_feat.ensure(sizeof(double) * (size_t)ace_feature_count(ws) * nu);
  const AceLayout lay = choose_layout(tables_of(a), ws->opt.device, a->sched_chunk, a->sched_groups, feat_dev != nullptr);
  batch_launch(ws, a, req, lay, E_dev, F_dev, W_dev, feat_dev);
  ws->stage_end(2);
  ace_check(ws, a);
}

// Batch evaluation replayed from a CUDA graph.  The first call (or a call
// after the batch, model, schedule or outputs changed) plans with an eager
// run, sizes the environment buffers with 25 % headroom and captures the
// device-only sequence — cell-list build, environments, site kernel, force
// gather, per-system outputs — on the workspace stream; later calls launch
// the graph.  Positions may change between replays (pfw_batch_update_positions):
// an environment that outgrows the headroom raises PFW_ECAPACITY at the next
// pfw_batch_graph_sync.
void ace_batch_graph(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev, double* feat_dev) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  GraphKey key;
  key.geometry_version = ws->geometry_version;
  key.alloc_epoch = g_alloc_epoch.load();
  key.E = E_dev;
  key.F = F_dev;
  key.W = W_dev;
  key.feat = feat_dev;
  key.req = req;
  key.chunk = a->sched_chunk;
  key.groups = a->sched_groups;
  key.precision = ws->opt.precision;
  cudaStream_t st = ws->stream;
  const auto& ps = ws->prep.sys;
  const bool same_plan = a->graph_sys.size() == ps.size() &&
                         (ps.empty() || std::memcmp(a->graph_sys.data(), ps.data(), sizeof(SysGeom) * ps.size()) == 0);
  if (!a->graph_exec || !(a->graph_key == key) || !same_plan) {
    release_graph(a);
    for (const auto& hs : ws->systems)
      if (!hs.pbc[0] || !hs.pbc[1] || !hs.pbc[2])
        throw Error(PFW_EINVAL, "graph batches require fully periodic systems");
    ace_evaluate_batch(ws, req, E_dev, F_dev, W_dev, feat_dev);  // plan and validate
    ensure_edge_buffers(a, (int)std::min<int64_t>((int64_t)(a->nedges * 1.25) + 4096, INT32_MAX / 4));
    const bool feat = feat_dev != nullptr;
    const AceLayout lay = choose_layout(tables_of(a), ws->opt.device, a->sched_chunk, a->sched_groups, feat);
    const bool diag = ws->diag;
    ws->diag = false;
    const uint64_t launches0 = ws->launches;
    PFW_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      PFW_CUDA(cudaMemsetAsync(a->status.ptr, 0, sizeof(int) * 4, st));
      prepare_launch(ws, true);
      edges_count_launch(ws, a);
      edges_fill_launch(ws, a);
      batch_launch(ws, a, req, lay, E_dev, F_dev, W_dev, feat_dev);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      ws->diag = diag;
      throw;
    }
    PFW_CUDA(cudaStreamEndCapture(st, &a->graph));
    ws->diag = diag;
    a->graph_kernels = ws->launches - launches0;
    ws->launches = launches0;
    PFW_CUDA(cudaGraphInstantiate(&a->graph_exec, a->graph, 0));
    a->graph_key = key;
    a->graph_key.alloc_epoch = g_alloc_epoch.load();  // after the planning run's allocations
    a->graph_sys = ws->prep.sys;
  }
  PFW_CUDA(cudaGraphLaunch(a->graph_exec, st));
  ws->launches += a->graph_kernels;  // kernels replayed by the graph
}

void ace_batch_graph_sync(pfw_ws* ws) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  prepare_check(ws);
  try {
    ace_check(ws, a);
  } catch (const Error& e) {
    if (e.code == PFW_ECAPACITY) release_graph(a);  // the next launch re-plans
    throw;
  }
}

// ---------------------------------------------------------------------------
// design rows (design_matrix_impl, ACE/fitting.jl:18-67)
// ---------------------------------------------------------------------------
// The adjoint terms are never read; products staged where they fit.
static AceLayout choose_design_layout(const AceTables& p, int device) {
  int optin = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  const int cand[][2] = {{16, 4}, {16, 2}, {8, 4}, {8, 2}, {8, 1}};
  for (auto& c : cand) {
    if (c[0] > ACE_MAX_CHUNK || c[1] > ACE_DESIGN_MAX_GROUPS) continue;
    for (int gt : {1, 3}) {
      AceLayout lay;
      lay.make(p, c[0], c[1], 0, 0, gt, 1);
      if (lay.total <= (size_t)optin) return lay;
    }
  }
  throw Error(PFW_EINVAL, "ACE model too large for the design kernel's shared memory");
}

template <int L>
static void launch_design(const AceTables& p, const AceLayout& lay, int nsys, const SysGeom* sysv, AceDevice* a,
                          const pfw_ws* ws, double* A_dev, int64_t ld, double* base_dev) {
  auto kern = k_ace_design<L>;
  PFW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay.total));
  int sms = 0, per_sm = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws->opt.device));
  PFW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ACE_GROUP * lay.G, lay.total));
  per_sm = std::max(per_sm, 1);
  // column slices per system so that small batches still fill every group
  const int slots = sms * per_sm * lay.G;
  const int nslice = nsys >= slots ? 1 : std::max(1, std::min((slots + nsys - 1) / nsys, (p.nB + ACE_GROUP - 1) / ACE_GROUP));
  const int blocks = std::max(1, std::min(sms * per_sm, (nsys * nslice + lay.G - 1) / lay.G));
  // one row of product factor gradients per site group
  double4* gs = static_cast<double4*>(a->design_G.ensure(sizeof(double4) * (size_t)blocks * lay.G * p.P));
  // systems by decreasing atom count, handed out by a counter
  std::vector<int> order(nsys);
  for (int s = 0; s < nsys; ++s) order[s] = s;
  const auto& ps = ws->prep.sys;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return ps[x].natoms > ps[y].natoms; });
  int* dorder = static_cast<int*>(a->design_order.ensure(sizeof(int) * (nsys + 1)));
  PFW_CUDA(cudaMemcpyAsync(dorder, order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, ws->stream));
  PFW_CUDA(cudaMemsetAsync(dorder + nsys, 0, sizeof(int), ws->stream));
  kern<<<blocks, ACE_GROUP * lay.G, lay.total, ws->stream>>>(
      p, lay, nsys, sysv, a->cap, a->edge_off.as<int>(), a->edge_j.as<int>(), a->edge_d.as<double4>(),
      ws->pos.as<double4>(), ws->perm.as<int>(), gs, dorder, dorder + nsys, nslice, A_dev, ld, base_dev,
      a->status.as<int>());
}

void ace_design_shape(pfw_ws* ws, int64_t* rows, int64_t* cols) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  if (rows) *rows = 10 * (int64_t)ws->systems.size() + 3 * (int64_t)ws->n;
  if (cols) *cols = (int64_t)a->nz * (a->nB + a->nQ);
}

void ace_design_matrix(pfw_ws* ws, double* A_dev, int64_t ld, int64_t rows_capacity, double* base_dev) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  check_species(ws, a->nz, "ACE model has no element channel for a species");
  if (a->nQ > 4 * ACE_GROUP) throw Error(PFW_EINVAL, "design rows support at most 256 pair channels");
  int64_t rows = 0, cols = 0;
  ace_design_shape(ws, &rows, &cols);
  if (!A_dev) throw Error(PFW_EINVAL, "null design matrix");
  if (ld < cols || rows_capacity < rows) throw Error(PFW_ESHAPE, "design matrix buffer too small");
  cudaStream_t st = ws->stream;
  ws->prep.valid = false;
  prepare(ws, a->cutoff);
  a->status.ensure(sizeof(int) * 4);
  PFW_CUDA(cudaMemsetAsync(a->status.ptr, 0, sizeof(int) * 4, st));
  build_edges(ws, a);
  a->n = ws->prep.n;
  const int nsys = (int)ws->prep.sys.size();
  const AceTables p = tables_of(a);
  const AceLayout lay = choose_design_layout(p, ws->opt.device);
  // the rows arrive zeroed; the kernel only adds
  PFW_CUDA(cudaMemset2DAsync(A_dev, sizeof(double) * ld, 0, sizeof(double) * cols, rows, st));
  if (nsys > 0) {
    const SysGeom* sysv = ws->sysgeom.as<SysGeom>();
    switch (a->lmax) {
      case 0: launch_design<0>(p, lay, nsys, sysv, a, ws, A_dev, ld, base_dev); break;
      case 1: launch_design<1>(p, lay, nsys, sysv, a, ws, A_dev, ld, base_dev); break;
      case 2: launch_design<2>(p, lay, nsys, sysv, a, ws, A_dev, ld, base_dev); break;
      case 3: launch_design<3>(p, lay, nsys, sysv, a, ws, A_dev, ld, base_dev); break;
      case 4: launch_design<4>(p, lay, nsys, sysv, a, ws, A_dev, ld, base_dev); break;
      case 5: launch_design<5>(p, lay, nsys, sysv, a, ws, A_dev, ld, base_dev); break;
      default: launch_design<6>(p, lay, nsys, sysv, a, ws, A_dev, ld, base_dev); break;
    }
    ws->launches += 1;
  }
  a->evaluated = false;
  ace_check(ws, a);
}

void ace_site_energies(pfw_ws* ws, double* host) {
  AceDevice* a = ws->ace;
  if (!a || !a->evaluated) throw Error(PFW_ESTATE, "no ACE evaluation to report");
  if (!host) throw Error(PFW_EINVAL, "null output");
  PFW_CUDA(cudaMemcpyAsync(host, a->site_E_orig.ptr, sizeof(double) * a->n, cudaMemcpyDeviceToHost, ws->stream));
  PFW_CUDA(cudaStreamSynchronize(ws->stream));
}

// FP64 FMA throughput: 8 independent dependency chains per thread.
__global__ void k_fp64_probe(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; ++it)
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 1.2345) out[0] = s;  // keep the chains live
}

double probe_fp64(pfw_ws* ws) {
  int sms = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws->opt.device));
  double* out = static_cast<double*>(ws->out_E.ensure(sizeof(double)));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  PFW_CUDA(cudaEventCreate(&e0));
  PFW_CUDA(cudaEventCreate(&e1));
  k_fp64_probe<<<blocks, threads, 0, ws->stream>>>(out, 64, 0.999999, 1e-7);  // warm-up
  PFW_CUDA(cudaEventRecord(e0, ws->stream));
  k_fp64_probe<<<blocks, threads, 0, ws->stream>>>(out, iters, 0.999999, 1e-7);
  PFW_CUDA(cudaEventRecord(e1, ws->stream));
  PFW_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  PFW_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ws->launches += 2;
  const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  return flops / (ms * 1e-3) / 1e12;
}

// ---------------------------------------------------------------------------
// learned per-atom surrogate with gated ACE fallback
// ---------------------------------------------------------------------------
// The reference has no GPU surrogate; its closest analogue is the CPU
// invariant head ACEFeatureEnergy (ACE/feature_energy.jl:1-86).  Here a
// restricted ACE model (the low-order invariants and pair sums) produces 64
// features per site inside the site kernel, an ensemble of BF16-weight MLPs
// gives the site energy and dE/dfeature, and the ACE pullback turns that into
// edge gradients.  Sites whose features leave the training range, or whose
// ensemble disagrees by more than tau, are re-evaluated with the full ACE
// model on the same environments.
struct SurDevice {
  AceDevice* fm = nullptr;  // the feature model (restricted ACE tables)
  int nin = 0, H = 0, M = 0, nz = 0;
  float tau = 0.f;
  bool has_mlp = false;
  DevBuf W1, W2, w3, b1, b2, b3, xm, xs, xlo, xhi, ym, ys, ccol_off, ccol_b, ccol_val;
  DevBuf flags, fb_count, fb_list, fb_out, site_A, site_feat, site_df, site_e, feat_out, zlist, zcount;
  int64_t last_fallback = -1, last_sites = 0;
};

void sur_free(pfw_ws* ws) {
  SurDevice* d = ws->sur;
  if (!d) return;
  free_device(d->fm);
  DevBuf* bufs[] = {&d->W1, &d->W2, &d->w3, &d->b1, &d->b2, &d->b3, &d->xm, &d->xs, &d->xlo, &d->xhi, &d->ym,
                    &d->ys, &d->ccol_off, &d->ccol_b, &d->ccol_val, &d->flags, &d->fb_count, &d->fb_list,
                    &d->fb_out, &d->site_A, &d->site_feat, &d->site_df, &d->site_e, &d->feat_out, &d->zlist,
                    &d->zcount};
  for (auto* b : bufs) b->release();
  delete d;
  ws->sur = nullptr;
}

constexpr int SUR_MAXW = 64;   // MLP kernel: nin, hidden <= 64

void sur_load(pfw_ws* ws, const pfw_ace_tables* t, const pfw_mlp_params* mp) {
  if (t->nbasis + t->pair.nchannels < 1) throw Error(PFW_EINVAL, "feature model has no features");
  const int nin = t->nbasis + t->pair.nchannels;
  if (mp) {
    if (mp->nz != t->nz || mp->nin != nin) throw Error(PFW_ESHAPE, "MLP input shape does not match the feature model");
    if (mp->members < 1 || mp->members > 4) throw Error(PFW_EINVAL, "ensemble of 1 to 4 members");
    if (mp->hidden < 1 || mp->hidden > SUR_MAXW || nin > SUR_MAXW)
      throw Error(PFW_EINVAL, "the surrogate MLP supports up to 64 inputs and 64 hidden units");
    if (!mp->W1 || !mp->b1 || !mp->W2 || !mp->b2 || !mp->w3 || !mp->b3 || !mp->x_mean || !mp->x_std ||
        !mp->x_lo || !mp->x_hi || !mp->y_mean || !mp->y_std)
      throw Error(PFW_EINVAL, "MLP parameter arrays are required");
    for (size_t k = 0; k < (size_t)mp->nz * nin; ++k)
      if (!(mp->x_std[k] > 0.0) || !std::isfinite(mp->x_mean[k]))
        throw Error(PFW_EINVAL, "feature standardisation must be finite with positive scales");
  }
  AceDevice* fm = load_model(ws, t);
  SurDevice* d = new SurDevice();
  d->fm = fm;
  try {
    cudaStream_t st = ws->stream;
    d->nin = nin;
    d->nz = t->nz;
    // coupling by product column: w_k = Σ_b C[b,k] dE/dB_b
    std::vector<int> coff(t->nproducts + 1, 0);
    for (int e = 0; e < t->ncoupling; ++e) coff[t->coupling_cols[e] + 1]++;
    for (int k = 0; k < t->nproducts; ++k) coff[k + 1] += coff[k];
    std::vector<int> cb(t->ncoupling);
    std::vector<double> cv(t->ncoupling);
    {
      std::vector<int> fill(coff.begin(), coff.end() - 1);
      for (int e = 0; e < t->ncoupling; ++e) {
        const int q = fill[t->coupling_cols[e]]++;
        cb[q] = t->coupling_rows[e];
        cv[q] = t->coupling_vals[e];
      }
    }
    upload(d->ccol_off, coff.data(), coff.size(), st);
    upload(d->ccol_b, cb.data(), cb.size(), st);
    upload(d->ccol_val, cv.data(), cv.size(), st);
    if (mp) {
      const int nz = mp->nz, M = mp->members, H = mp->hidden;
      d->M = M;
      d->H = H;
      d->tau = (float)mp->tau;
      upload(d->W1, mp->W1, (size_t)nz * M * H * nin, st);
      upload(d->W2, mp->W2, (size_t)nz * M * H * H, st);
      upload(d->w3, mp->w3, (size_t)nz * M * H, st);
      upload(d->b1, mp->b1, (size_t)nz * M * H, st);
      upload(d->b2, mp->b2, (size_t)nz * M * H, st);
      upload(d->b3, mp->b3, (size_t)nz * M, st);
      upload(d->xm, mp->x_mean, (size_t)nz * nin, st);
      upload(d->xs, mp->x_std, (size_t)nz * nin, st);
      upload(d->xlo, mp->x_lo, (size_t)nz * nin, st);
      upload(d->xhi, mp->x_hi, (size_t)nz * nin, st);
      upload(d->ym, mp->y_mean, nz, st);
      upload(d->ys, mp->y_std, nz, st);
      d->has_mlp = true;
    }
    PFW_CUDA(cudaStreamSynchronize(st));
  } catch (...) {
    free_device(d->fm);
    delete d;
    throw;
  }
  sur_free(ws);
  ws->sur = d;
}

static AceLayout choose_sur_layout(const AceTables& p, int device, int pass) {
  int optin = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  const int cand[][2] = {{32, 4}, {32, 3}, {16, 8}, {16, 6}, {16, 4}, {32, 2}, {16, 2}, {16, 1}, {8, 1}};
  for (auto& c : cand) {
    if (c[0] > ACE_MAX_CHUNK || c[1] > ACE_MAX_GROUPS) continue;
    for (int gt : {0, 1, 3}) {
      AceLayout lay;
      lay.make(p, c[0], c[1], 0, pass, gt);
      if (lay.total <= (size_t)optin) return lay;
    }
  }
  throw Error(PFW_EINVAL, "surrogate feature model too large for the site kernel's shared memory");
}

// Sites of each species (lists in any order; every site's result is
// independent of its position in the list).
__global__ void k_species_lists(int n, int nz, const double4* __restrict__ pos, int* __restrict__ count,
                                int* __restrict__ list) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int z = min(max((int)pos[s].w, 0), nz - 1);
  list[(size_t)z * n + atomicAdd(count + z, 1)] = s;
}

static void sur_prepare(pfw_ws* ws, SurDevice* d) {
  AceDevice* a = d->fm;
  cudaStream_t st = ws->stream;
  ws->prep.valid = false;
  prepare(ws, a->cutoff);
  a->status.ensure(sizeof(int) * 4);
  PFW_CUDA(cudaMemsetAsync(a->status.ptr, 0, sizeof(int) * 4, st));
  build_edges(ws, a);
  const int n = ws->prep.n;
  a->n = n;
  int* ub = static_cast<int*>(a->unit_begin.ensure(sizeof(int) * (n + 1)));
  a->unit_out.ensure(sizeof(double) * 10 * std::max(n, 1));
  k_iota<<<grid_for(n + 1, 256), 256, 0, st>>>(n, ub);
  ws->launches += 1;
}

static SiteLaunch sur_launch(pfw_ws* ws, SurDevice* d, int n, bool want_grad) {
  AceDevice* a = d->fm;
  SiteLaunch s{};
  s.nunits = n;
  s.unit_begin = a->unit_begin.as<int>();
  s.cap = a->cap;
  s.off = a->edge_off.as<int>();
  s.ed = a->edge_d.as<double4>();
  s.pos = ws->pos.as<double4>();
  s.g = a->edge_g.as<double>();
  s.unit_out = a->unit_out.as<double>();
  s.want_grad = want_grad;
  s.status = a->status.as<int>();
  SurParams& sp = s.sur;
  sp.nin = d->nin;
  sp.H = d->H;
  sp.M = d->M;
  sp.W1 = d->W1.as<unsigned short>();
  sp.W2 = d->W2.as<unsigned short>();
  sp.w3 = d->w3.as<unsigned short>();
  sp.b1 = d->b1.as<float>();
  sp.b2 = d->b2.as<float>();
  sp.b3 = d->b3.as<float>();
  sp.x_mean = d->xm.as<double>();
  sp.x_std = d->xs.as<double>();
  sp.x_lo = d->xlo.as<float>();
  sp.x_hi = d->xhi.as<float>();
  sp.y_mean = d->ym.as<double>();
  sp.y_std = d->ys.as<double>();
  sp.tau = d->tau;
  sp.ccol_off = d->ccol_off.as<int>();
  sp.ccol_b = d->ccol_b.as<int>();
  sp.ccol_val = d->ccol_val.as<double>();
  const size_t nn = std::max(n, 1);
  sp.flags = static_cast<int*>(d->flags.ensure(sizeof(int) * nn));
  sp.site_A = static_cast<double*>(d->site_A.ensure(sizeof(double) * nn * a->D));
  sp.site_feat = static_cast<double*>(d->site_feat.ensure(sizeof(double) * nn * d->nin));
  sp.site_df = static_cast<double*>(d->site_df.ensure(sizeof(double) * nn * d->nin));
  sp.site_e = static_cast<double*>(d->site_e.ensure(sizeof(double) * nn));
  return s;
}

// Feature pass: A-basis and own-species features of every site.
static void sur_feature_pass(pfw_ws* ws, SurDevice* d, const SiteLaunch& s) {
  AceDevice* a = d->fm;
  const AceTables p = tables_of(a);
  if (s.nunits > 0) {
    const AceLayout lay = choose_sur_layout(p, ws->opt.device, 1);
    if (ws->opt.precision == PFW_PRECISION_MIXED) dispatch_sites<float, 1>(a->lmax, p, lay, s, ws->stream, ws->opt.device);
    else dispatch_sites<double, 1>(a->lmax, p, lay, s, ws->stream, ws->opt.device);
    ws->launches += 1;
  }
}

// Per-site features in original order: out[o*nin + i].
__global__ void k_permute_rows(int n, int w, const double* __restrict__ in, const int* __restrict__ perm,
                               double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * w) return;
  const int s = k / w, i = k - s * w;
  out[(size_t)perm[s] * w + i] = in[k];
}

void sur_features(pfw_ws* ws, double* out_dev) {
  SurDevice* d = ws->sur;
  if (!d) throw Error(PFW_ESTATE, "no surrogate feature model loaded");
  check_species(ws, d->nz, "feature model has no element channel for a species");
  sur_prepare(ws, d);
  const int n = ws->prep.n;
  SiteLaunch s = sur_launch(ws, d, n, false);
  sur_feature_pass(ws, d, s);
  if (n > 0) {
    k_permute_rows<<<grid_for((int64_t)n * d->nin, 256), 256, 0, ws->stream>>>(n, d->nin, s.sur.site_feat,
                                                                               ws->perm.as<int>(), out_dev);
    ws->launches += 1;
  }
  ace_check(ws, d->fm);
}

__global__ void k_flag_list(int n, const int* __restrict__ flags, const int* __restrict__ pos_excl,
                            int* __restrict__ list) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n && flags[s]) list[pos_excl[s]] = s;
}

__global__ void k_scatter_sites(int count, const int* __restrict__ list, const double* __restrict__ fb_out,
                                double* __restrict__ site_out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count * 10) return;
  const int u = k / 10, c = k - u * 10;
  site_out[10 * (size_t)list[u] + c] = fb_out[10 * (size_t)u + c];
}

void sur_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev) {
  SurDevice* d = ws->sur;
  AceDevice* full = ws->ace;
  if (!d || !d->has_mlp) throw Error(PFW_ESTATE, "no surrogate (feature model and MLP) loaded");
  if (!full) throw Error(PFW_ESTATE, "the surrogate falls back to the ACE model: load it first");
  if (full->cutoff != d->fm->cutoff || full->nz != d->nz)
    throw Error(PFW_EINVAL, "surrogate feature model and ACE model differ in cutoff or species");
  check_species(ws, d->nz, "feature model has no element channel for a species");
  // a mixed workspace runs the two site passes (and any fallback sites) in FP32
  AceDevice* a = d->fm;
  cudaStream_t st = ws->stream;
  ws->stage_begin(3);
  ws->stage_begin(0);
  sur_prepare(ws, d);
  ws->stage_end(0);
  ws->stage_end(3);
  const int n = ws->prep.n;
  const bool want_grad = (req & (PFW_REQ_FORCES | PFW_REQ_VIRIAL)) != 0;
  const AceTables p = tables_of(a);
  ws->stage_begin(1);
  SiteLaunch s = sur_launch(ws, d, n, false);
  // 1. features and A-basis of every site
  sur_feature_pass(ws, d, s);
  // 2. the MLP ensemble per species, tiles of 64 sites
  int* zc = static_cast<int*>(d->zcount.ensure(sizeof(int) * d->nz));
  int* zl = static_cast<int*>(d->zlist.ensure(sizeof(int) * (size_t)std::max(n, 1) * d->nz));
  PFW_CUDA(cudaMemsetAsync(zc, 0, sizeof(int) * d->nz, st));
  if (n > 0) {
    k_species_lists<<<grid_for(n, 256), 256, 0, st>>>(n, d->nz, ws->pos.as<double4>(), zc, zl);
    const size_t smem = tc_mlp_smem();
    PFW_CUDA(cudaFuncSetAttribute(k_sur_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_sur_mlp_tc<<<dim3(grid_for(n, TC_TILE), d->nz), 256, smem, st>>>(s.sur, n, zc, zl, a->status.as<int>());
    ws->launches += 2;
  }
  // 3. pullback with the per-site weights
  s.want_grad = want_grad;
  if (n > 0) {
    const AceLayout lay = choose_sur_layout(p, ws->opt.device, 2);
    if (ws->opt.precision == PFW_PRECISION_MIXED) dispatch_sites<float, 2>(a->lmax, p, lay, s, st, ws->opt.device);
    else dispatch_sites<double, 2>(a->lmax, p, lay, s, st, ws->opt.device);
    ws->launches += 1;
  }
  // fallback: the flagged sites with the full model on the same environments
  int* flags = s.sur.flags;
  int* pos_excl = static_cast<int*>(d->fb_count.ensure(sizeof(int) * (n + 1)));
  exclusive_scan_i32(ws, flags, pos_excl, n);
  int count = 0;
  PFW_CUDA(cudaMemcpyAsync(&count, pos_excl + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaStreamSynchronize(st));
  d->last_fallback = count;
  d->last_sites = n;
  if (count > 0) {
    int* list = static_cast<int*>(d->fb_list.ensure(sizeof(int) * count));
    double* fb_out = static_cast<double*>(d->fb_out.ensure(sizeof(double) * 10 * count));
    k_flag_list<<<grid_for(n, 256), 256, 0, st>>>(n, flags, pos_excl, list);
    const AceTables pf = tables_of(full);
    const AceLayout lf = choose_layout(pf, ws->opt.device, full->sched_chunk, full->sched_groups, 0);
    SiteLaunch f = s;
    f.sur = SurParams{};
    f.nunits = count;
    f.unit_begin = nullptr;
    f.unit_sites = list;
    f.unit_out = fb_out;
    if (ws->opt.precision == PFW_PRECISION_MIXED) dispatch_sites<float, 0>(full->lmax, pf, lf, f, st, ws->opt.device);
    else dispatch_sites<double, 0>(full->lmax, pf, lf, f, st, ws->opt.device);
    k_scatter_sites<<<grid_for((int64_t)count * 10, 256), 256, 0, st>>>(count, list, fb_out, a->unit_out.as<double>());
    ws->launches += 3;
  }
  ws->stage_end(1);
  ws->stage_begin(2);
  if (F_dev && n > 0) {
    if (want_grad) {
      k_ace_gather<<<grid_for((int64_t)n * GATHER_LANES, 128), 128, 0, st>>>(n, a->edge_off.as<int>(), a->cap, a->edge_rev.as<int>(),
                                                     a->edge_g.as<double>(), ws->perm.as<int>(), F_dev);
      ws->launches += 1;
    } else {
      PFW_CUDA(cudaMemsetAsync(F_dev, 0, sizeof(double) * 3 * n, st));
    }
  }
  double* Esite = static_cast<double*>(a->site_E_orig.ensure(sizeof(double) * std::max(n, 1)));
  if (n > 0) {
    k_site_energies<<<grid_for(n, 256), 256, 0, st>>>(n, a->unit_out.as<double>(), ws->perm.as<int>(), Esite);
    ws->launches += 1;
  }
  double* E = E_dev ? E_dev : static_cast<double*>(ws->out_E.ensure(sizeof(double)));
  double* W = W_dev ? W_dev : static_cast<double*>(ws->out_W.ensure(sizeof(double) * 9));
  mask_unowned_sites(ws, a->unit_out.as<double>(), n);
  reduce_site_parts(ws, a->unit_out.as<double>(), n, E, W);
  ws->stage_end(2);
  a->evaluated = true;
  ace_check(ws, a);
}

// site_df[s] = dEdx[perm[s]] (sorted order), site energies zero.
__global__ void k_gather_site_df(int n, int w, const double* __restrict__ dEdx, const int* __restrict__ perm,
                                 double* __restrict__ site_df, double* __restrict__ site_e) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * w) return;
  const int s = k / w, i = k - s * w;
  site_df[k] = dEdx[(size_t)perm[s] * w + i];
  if (i == 0) site_e[s] = 0.0;
}

// Forces of a per-site dE/dfeature field through the feature model: the
// feature pass (A-basis of the current geometry), then the surrogate's
// pullback pass with the given field and the reverse-edge force gather.
void sur_pullback(pfw_ws* ws, const double* dEdx_dev, double* F_dev) {
  SurDevice* d = ws->sur;
  if (!d) throw Error(PFW_ESTATE, "no surrogate feature model loaded");
  if (!dEdx_dev || !F_dev) throw Error(PFW_EINVAL, "feature gradients and force output required");
  if (ws->opt.precision != PFW_PRECISION_FP64) throw Error(PFW_EINVAL, "the surrogate path runs in the FP64 workspace");
  check_species(ws, d->nz, "feature model has no element channel for a species");
  sur_prepare(ws, d);
  AceDevice* a = d->fm;
  const int n = ws->prep.n;
  cudaStream_t st = ws->stream;
  SiteLaunch s = sur_launch(ws, d, n, false);
  sur_feature_pass(ws, d, s);
  if (n > 0) {
    k_gather_site_df<<<grid_for((int64_t)n * d->nin, 256), 256, 0, st>>>(n, d->nin, dEdx_dev, ws->perm.as<int>(),
                                                                          s.sur.site_df, s.sur.site_e);
    s.want_grad = true;
    const AceTables p = tables_of(a);
    dispatch_sites<double, 2>(a->lmax, p, choose_sur_layout(p, ws->opt.device, 2), s, st, ws->opt.device);
    k_ace_gather<<<grid_for((int64_t)n * GATHER_LANES, 128), 128, 0, st>>>(n, a->edge_off.as<int>(), a->cap, a->edge_rev.as<int>(),
                                                   a->edge_g.as<double>(), ws->perm.as<int>(), F_dev);
    ws->launches += 3;
  }
  ace_check(ws, a);
}

void sur_stats(pfw_ws* ws, int64_t* fallback, int64_t* sites) {
  SurDevice* d = ws->sur;
  if (!d) throw Error(PFW_ESTATE, "no surrogate loaded");
  if (fallback) *fallback = d->last_fallback;
  if (sites) *sites = d->last_sites;
}

int sur_feature_width(pfw_ws* ws) {
  if (!ws->sur) throw Error(PFW_ESTATE, "no surrogate feature model loaded");
  return ws->sur->nin;
}

void sur_site_energies(pfw_ws* ws, double* host) {
  SurDevice* d = ws->sur;
  if (!d || !d->fm->evaluated) throw Error(PFW_ESTATE, "no surrogate evaluation to report");
  PFW_CUDA(cudaMemcpyAsync(host, d->fm->site_E_orig.ptr, sizeof(double) * d->fm->n, cudaMemcpyDeviceToHost,
                           ws->stream));
  PFW_CUDA(cudaStreamSynchronize(ws->stream));
}

}  // namespace pfw
