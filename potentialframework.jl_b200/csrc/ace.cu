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
//   k_ace_site    one CTA per site, edges in chunks of 32:
//                   radial splines and harmonics → A-basis A[a] = Σ_j R[j,n_a]Y[j,m_a]
//                   products P_k and adjoints dA (division-free, per-density
//                   term lists), site energy
//                   T1[j,n] = Σ dA·Y, T2[j,m] = Σ dA·R, then per-edge gradient
//                   g_j = r̂(Σ_n dR·T1 + Σ Wpair·dQ) + Σ_m ∇Y·T2
//   k_ace_gather  F_k = Σ_{e∈out(k)} g_e - g_{rev(e)}  (reduce_site!,
//                 NeighbourList/execution.jl:256-273, without a racing scatter)
//   k_ace_reduce  E and the 3×3 virial from per-site partials
#include <algorithm>
#include <cmath>
#include <vector>

#include "ace_math.cuh"
#include "pfw_internal.h"
#include "traverse.cuh"

namespace pfw {

constexpr int ACE_THREADS = 128;
constexpr int ACE_CHUNK = 32;

struct AceDevice {
  int nz = 0, lmax = 0, nY = 0, nR = 0, nQ = 0, D = 0, P = 0, nB = 0, max_order = 0;
  double cutoff = 0;
  RadialDev R{}, Q{};
  DevBuf r_len, r_nodes, r_coeff, r_tr, r_pow, r_envk, r_env;
  DevBuf q_len, q_nodes, q_coeff, q_tr, q_pow, q_envk, q_env;
  DevBuf density, dn_off, dn, dm_off, dm, prod_off, prod_fac, term_off, term, weights, wpair, ref, pair_ok, Fnorm;
  DevBuf c_rows, c_cols, c_vals;
  int ncoupling = 0;
  // per evaluation
  DevBuf edge_count, edge_off, edge_j, edge_d, edge_S, edge_rev, edge_g, site_out, site_E_orig, status;
  int64_t nedges = 0;
  int n = 0;
  bool evaluated = false;
};

struct AceParams {
  RadialDev R, Q;
  int nz, lmax, nY, nR, nQ, D, P;
  const int2* density;   // [D] (n, m)
  const int* dn_off;     // [nR+1] densities by radial channel
  const int2* dn;        //   (a, m)
  const int* dm_off;     // [nY+1] densities by harmonic
  const int2* dm;        //   (a, n)
  const int* prod_off;   // [P+1]
  const int* prod_fac;   // factors
  const int* term_off;   // [D+1] occurrences of each density in products
  const int2* term;      //   (k, position)
  const double* weights; // [nz][P]
  const double* wpair;   // [nz][nQ]
  const double* ref;     // [nz]
  const int* pair_ok;    // [nz]
  const double* Fnorm;   // [(L+1)^2]
};

// ---------------------------------------------------------------------------
// environments
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(128)
    k_edge_count(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
                 const double4* __restrict__ pos, int ncells, int* __restrict__ count) {
  __shared__ WarpStage stage[4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * 4 + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  int cur = -1, cnt = 0;
  warp_traverse_cell<MODE>(g, cell, cell_start, pos, stage[warp], lane,
                           [&](int i, int, const double4&, const double4&, const StencilEntry&, const double*, double) {
                             if (i != cur) {
                               if (cur >= 0) count[cur] = cnt;
                               cur = i;
                               cnt = 0;
                             }
                             ++cnt;
                           });
  if (cur >= 0) count[cur] = cnt;
}

template <int MODE>
__global__ void __launch_bounds__(128)
    k_edge_fill(const SysGeom* __restrict__ sysv, const int* __restrict__ cell_sys, const int* __restrict__ cell_start,
                const double4* __restrict__ pos, const int* __restrict__ perm, const int* __restrict__ wind,
                const double* __restrict__ X, int ncells, const int* __restrict__ off, int* __restrict__ ej,
                int4* __restrict__ eS, double4* __restrict__ ed) {
  __shared__ WarpStage stage[4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * 4 + warp;
  if (cell >= ncells) return;
  const SysGeom& g = sysv[cell_sys[cell]];
  int cur = -1, o = 0, a = 0;
  int wi[3] = {0, 0, 0};
  double xi[3] = {0, 0, 0};
  warp_traverse_cell<MODE>(g, cell, cell_start, pos, stage[warp], lane,
                           [&](int i, int j, const double4& pi, const double4& pj, const StencilEntry& se,
                               const double*, double) {
                             if (i != cur) {
                               cur = i;
                               o = off[i];
                               a = perm[i];
                               wi[0] = wind[3 * a]; wi[1] = wind[3 * a + 1]; wi[2] = wind[3 * a + 2];
                               xi[0] = X[3 * a]; xi[1] = X[3 * a + 1]; xi[2] = X[3 * a + 2];
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
                           });
}

// Reverse edge of e = (i→j, S): the entry (j→i, -S) of j's list.
__global__ void k_edge_rev(int n, const int* __restrict__ off, const int* __restrict__ ej, const int4* __restrict__ eS,
                           int* __restrict__ rev, int* __restrict__ status) {
  const int i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  for (int e = off[i] + lane; e < off[i + 1]; e += 32) {
    const int j = ej[e];
    const int4 s = eS[e];
    int found = -1;
    for (int f = off[j]; f < off[j + 1]; ++f) {
      if (ej[f] == i) {
        const int4 t = eS[f];
        if (t.x == -s.x && t.y == -s.y && t.z == -s.z) {
          found = f;
          break;
        }
      }
    }
    if (found < 0) atomicOr(status, 4);
    rev[e] = found < 0 ? e : found;
  }
}

// ---------------------------------------------------------------------------
// site kernel
// ---------------------------------------------------------------------------
struct SiteSmem {
  double *A, *dA, *Y, *dY, *R, *dR, *T1, *T2, *eu, *ee, *ede, *edu, *dq, *er, *ed, *red;
  int *ek0, *epidx;
  static size_t bytes(int D, int nY, int nR) {
    size_t d = 2 * (size_t)D + (size_t)ACE_CHUNK * (nY + 3 * nY + 3 * nR + nY) + ACE_CHUNK * (7 + 3) + ACE_THREADS * 10;
    return d * sizeof(double) + 2 * ACE_CHUNK * sizeof(int);
  }
  __device__ void carve(double* base, int D, int nY, int nR) {
    double* p = base;
    A = p; p += D;
    dA = p; p += D;
    Y = p; p += ACE_CHUNK * nY;
    dY = p; p += ACE_CHUNK * nY * 3;
    R = p; p += ACE_CHUNK * nR;
    dR = p; p += ACE_CHUNK * nR;
    T1 = p; p += ACE_CHUNK * nR;
    T2 = p; p += ACE_CHUNK * nY;
    eu = p; p += ACE_CHUNK;
    ee = p; p += ACE_CHUNK;
    ede = p; p += ACE_CHUNK;
    edu = p; p += ACE_CHUNK;
    dq = p; p += ACE_CHUNK;
    er = p; p += ACE_CHUNK;
    ed = p; p += 3 * ACE_CHUNK + ACE_CHUNK;  // + spare
    red = p; p += ACE_THREADS * 10;
    ek0 = reinterpret_cast<int*>(p);
    epidx = ek0 + ACE_CHUNK;
  }
};

template <int L>
__device__ __forceinline__ int lmax_of(int runtime) {
  return L >= 0 ? L : runtime;
}

// Per-edge set-up of one chunk (thread t < nc): geometry, radial interval and
// envelope, pair term, harmonics (values, and gradients when Grad).
template <int L, bool Grad>
__device__ __forceinline__ void chunk_edges(const AceParams& p, SiteSmem& S, const double4* __restrict__ edge_d, int e0,
                                            int nc, int iz, double& e_acc, int* status) {
  const int t = threadIdx.x;
  if (t >= nc) return;
  const double4 d = edge_d[e0 + t];
  const int zj = min(max((int)d.w, 0), p.nz - 1);
  const int pidx = iz * p.nz + zj;
  const double r = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
  if (!(r > 0.0)) atomicOr(status, 2);
  const double rr = r > 0.0 ? r : 1.0;
  S.er[t] = rr;
  S.ed[3 * t] = d.x;
  S.ed[3 * t + 1] = d.y;
  S.ed[3 * t + 2] = d.z;
  const EdgeRadial<double> er = edge_radial<double>(p.R, pidx, rr);
  S.ek0[t] = er.k0;
  S.epidx[t] = pidx;
  S.eu[t] = er.u;
  S.ee[t] = er.e;
  S.ede[t] = er.de;
  S.edu[t] = er.du;
  // pair radials: energy Σ_n Wpair[n]·Q_n, or gradient factor Σ_n Wpair[n]·dQ_n/dr
  double qe = 0.0, qd = 0.0;
  if (p.pair_ok[zj] && p.nQ > 0) {
    const EdgeRadial<double> eq = edge_radial<double>(p.Q, pidx, rr);
    if (!eq.ok) atomicOr(status, 2);
    const double* wp = p.wpair + (size_t)iz * p.nQ;
    for (int n = 0; n < p.nQ; ++n) {
      double v, dv;
      channel_ed(channel_coeff(p.Q, pidx, eq.k0, n), eq, v, dv);
      qe += v * wp[n];
      qd += wp[n] * dv;
    }
  }
  if (!Grad) e_acc += qe;
  S.dq[t] = qd;
  const int nY = p.nY;
  double* Yt = S.Y + t * nY;
  double* dYt = S.dY + t * nY * 3;
  harmonics<double, Grad, L>(p.Fnorm, rr, d.x, d.y, d.z, [&](int idx, const Jet<double, Grad>& j) {
    Yt[idx] = j.v;
    if constexpr (Grad) {
      dYt[3 * idx] = j.gx;
      dYt[3 * idx + 1] = j.gy;
      dYt[3 * idx + 2] = j.gz;
    }
  });
}

template <int L>
__global__ void __launch_bounds__(ACE_THREADS)
    k_ace_site(AceParams p, int nsites, const int* __restrict__ edge_off, const double4* __restrict__ edge_d,
               const double4* __restrict__ pos, double* __restrict__ edge_g, double* __restrict__ site_out,
               int want_grad, int* __restrict__ status) {
  extern __shared__ double smem_raw[];
  SiteSmem S;
  S.carve(smem_raw, p.D, p.nY, p.nR);
  const int s = blockIdx.x;
  if (s >= nsites) return;
  const int tid = threadIdx.x;
  const int iz = min(max((int)pos[s].w, 0), p.nz - 1);
  const int eb = edge_off[s], E = edge_off[s + 1] - eb;
  const int D = p.D, nY = p.nY, nR = p.nR, P = p.P;
  double e_acc = 0.0;
  for (int a = tid; a < D; a += ACE_THREADS) S.A[a] = 0.0;
  // ---- A-basis -------------------------------------------------------
  for (int c0 = 0; c0 < E; c0 += ACE_CHUNK) {
    const int nc = min(ACE_CHUNK, E - c0);
    __syncthreads();
    chunk_edges<L, false>(p, S, edge_d, eb + c0, nc, iz, e_acc, status);
    __syncthreads();
    for (int idx = tid; idx < nc * nR; idx += ACE_THREADS) {
      const int t = idx / nR, n = idx - t * nR;
      const double* c = channel_coeff(p.R, S.epidx[t], S.ek0[t], n);
      const double u = S.eu[t];
      S.R[t * nR + n] = S.ee[t] * (((c[3] * u + c[2]) * u + c[1]) * u + c[0]);
    }
    __syncthreads();
    for (int a = tid; a < D; a += ACE_THREADS) {
      const int2 nm = p.density[a];
      double acc = S.A[a];
      for (int t = 0; t < nc; ++t) acc += S.R[t * nR + nm.x] * S.Y[t * nY + nm.y];
      S.A[a] = acc;
    }
  }
  __syncthreads();
  // ---- products, site energy and adjoints ------------------------------
  const double* w = p.weights + (size_t)iz * P;
  for (int k = tid; k < P; k += ACE_THREADS) {
    double pk = 1.0;
    for (int f = p.prod_off[k]; f < p.prod_off[k + 1]; ++f) pk *= S.A[p.prod_fac[f]];
    e_acc += w[k] * pk;
  }
  for (int a = tid; a < D; a += ACE_THREADS) {
    double acc = 0.0;
    for (int q = p.term_off[a]; q < p.term_off[a + 1]; ++q) {
      const int2 kt = p.term[q];
      double v = w[kt.x];
      const int f0 = p.prod_off[kt.x], f1 = p.prod_off[kt.x + 1];
      for (int f = f0; f < f1; ++f)
        if (f - f0 != kt.y) v *= S.A[p.prod_fac[f]];
      acc += v;
    }
    S.dA[a] = acc;
  }
  double wv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  // ---- pullback ---------------------------------------------------------
  if (want_grad) {
    for (int c0 = 0; c0 < E; c0 += ACE_CHUNK) {
      const int nc = min(ACE_CHUNK, E - c0);
      __syncthreads();
      double dummy = 0.0;
      chunk_edges<L, true>(p, S, edge_d, eb + c0, nc, iz, dummy, status);
      __syncthreads();
      for (int idx = tid; idx < nc * nR; idx += ACE_THREADS) {
        const int t = idx / nR, n = idx - t * nR;
        EdgeRadial<double> er;
        er.u = S.eu[t];
        er.e = S.ee[t];
        er.de = S.ede[t];
        er.du = S.edu[t];
        double v, dv;
        channel_ed(channel_coeff(p.R, S.epidx[t], S.ek0[t], n), er, v, dv);
        S.R[t * nR + n] = v;
        S.dR[t * nR + n] = dv;
      }
      __syncthreads();
      for (int idx = tid; idx < nc * nR; idx += ACE_THREADS) {
        const int t = idx / nR, n = idx - t * nR;
        double acc = 0.0;
        for (int q = p.dn_off[n]; q < p.dn_off[n + 1]; ++q) {
          const int2 am = p.dn[q];
          acc += S.dA[am.x] * S.Y[t * nY + am.y];
        }
        S.T1[t * nR + n] = acc;
      }
      for (int idx = tid; idx < nc * nY; idx += ACE_THREADS) {
        const int t = idx / nY, m = idx - t * nY;
        double acc = 0.0;
        for (int q = p.dm_off[m]; q < p.dm_off[m + 1]; ++q) {
          const int2 an = p.dm[q];
          acc += S.dA[an.x] * S.R[t * nR + an.y];
        }
        S.T2[t * nY + m] = acc;
      }
      __syncthreads();
      {
        const int t = tid >> 2, q = tid & 3;  // 4 threads per edge
        double s1 = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        if (t < nc) {
          for (int n = q; n < nR; n += 4) s1 += S.dR[t * nR + n] * S.T1[t * nR + n];
          for (int m = q; m < nY; m += 4) {
            const double t2 = S.T2[t * nY + m];
            gx += S.dY[(t * nY + m) * 3] * t2;
            gy += S.dY[(t * nY + m) * 3 + 1] * t2;
            gz += S.dY[(t * nY + m) * 3 + 2] * t2;
          }
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
          s1 += __shfl_xor_sync(0xffffffffu, s1, o);
          gx += __shfl_xor_sync(0xffffffffu, gx, o);
          gy += __shfl_xor_sync(0xffffffffu, gy, o);
          gz += __shfl_xor_sync(0xffffffffu, gz, o);
        }
        if (t < nc && q == 0) {
          const double r = S.er[t];
          const double dx = S.ed[3 * t], dy = S.ed[3 * t + 1], dz = S.ed[3 * t + 2];
          const double radial = (s1 + S.dq[t]) / r;
          const double g0 = radial * dx + gx, g1 = radial * dy + gy, g2 = radial * dz + gz;
          double* ge = edge_g + 3 * (size_t)(eb + c0 + t);
          ge[0] = g0;
          ge[1] = g1;
          ge[2] = g2;
          const double dd[3] = {dx, dy, dz}, gg[3] = {g0, g1, g2};
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int a = 0; a < 3; ++a) wv[a + 3 * b] -= dd[a] * gg[b];
        }
      }
    }
  }
  // ---- site energy and virial partials -----------------------------------
  __syncthreads();
  double* red = S.red;
  red[tid] = e_acc;
#pragma unroll
  for (int k = 0; k < 9; ++k) red[(k + 1) * ACE_THREADS + tid] = wv[k];
  __syncthreads();
  for (int st = ACE_THREADS / 2; st > 0; st >>= 1) {
    if (tid < st)
      for (int k = 0; k < 10; ++k) red[k * ACE_THREADS + tid] += red[k * ACE_THREADS + tid + st];
    __syncthreads();
  }
  if (tid < 10) site_out[10 * (size_t)s + tid] = red[tid * ACE_THREADS] + (tid == 0 ? p.ref[iz] : 0.0);
}

// F_k = Σ_{e ∈ out(k)} g_e - g_rev(e), written in original order.
__global__ void k_ace_gather(int n, const int* __restrict__ off, const int* __restrict__ rev,
                             const double* __restrict__ g, const int* __restrict__ perm, double* __restrict__ F) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double f0 = 0, f1 = 0, f2 = 0;
  for (int e = off[k]; e < off[k + 1]; ++e) {
    const int r = rev[e];
    f0 += g[3 * (size_t)e] - g[3 * (size_t)r];
    f1 += g[3 * (size_t)e + 1] - g[3 * (size_t)r + 1];
    f2 += g[3 * (size_t)e + 2] - g[3 * (size_t)r + 2];
  }
  const int o = perm[k];
  F[3 * o] = f0;
  F[3 * o + 1] = f1;
  F[3 * o + 2] = f2;
}

// Per-site [E, W(9)] → totals; site energies in original order.
__global__ void k_ace_reduce(int n, const double* __restrict__ site_out, const int* __restrict__ perm,
                             double* __restrict__ E, double* __restrict__ W, double* __restrict__ Esite) {
  __shared__ double sh[10][256];
  Kahan acc[10];
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 10; ++k) acc[k].add(site_out[10 * (size_t)s + k]);
    if (Esite) Esite[perm[s]] = site_out[10 * (size_t)s];
  }
#pragma unroll
  for (int k = 0; k < 10; ++k) sh[k][threadIdx.x] = acc[k].s - acc[k].c;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
#pragma unroll
      for (int k = 0; k < 10; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (E) E[0] = sh[0][0];
    if (W)
      for (int k = 0; k < 9; ++k) W[k] = sh[k + 1][0];
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
                               DevBuf& tr, DevBuf& pw, DevBuf& ek, DevBuf& ev, cudaStream_t st) {
  if (f.nchannels < 0 || f.nknots < 2) throw Error(PFW_EINVAL, "invalid radial family shape");
  const int np = nz * nz;
  for (int k = 0; k < np; ++k) {
    if (f.lengths[k] < 2 || f.lengths[k] > f.nknots) throw Error(PFW_EINVAL, "invalid spline node count");
    const int kind = f.envelope_kind[k];
    if (kind < 1 || kind > 3) throw Error(PFW_EINVAL, "unsupported radial envelope");
    if (f.powers[2 * k] <= 0 || f.powers[2 * k + 1] < f.powers[2 * k]) throw Error(PFW_EINVAL, "invalid Agnesi transform");
  }
  RadialDev d;
  d.nch = f.nchannels;
  d.nknots = f.nknots;
  d.nz = nz;
  d.lengths = upload(len, f.lengths, np, st);
  d.nodes = upload(nodes, f.nodes, (size_t)np * f.nknots, st);
  d.coeff = upload(coeff, f.coeff, (size_t)np * (f.nknots - 1) * f.nchannels * 4, st);
  d.transform = upload(tr, f.transform, (size_t)np * 6, st);
  d.powers = upload(pw, f.powers, (size_t)np * 2, st);
  d.env_kind = upload(ek, f.envelope_kind, np, st);
  d.env = upload(ev, f.envelope, (size_t)np * 5, st);
  return d;
}

void ace_free(pfw_ws* ws) {
  if (!ws->ace) return;
  AceDevice* a = ws->ace;
  DevBuf* bufs[] = {&a->r_len, &a->r_nodes, &a->r_coeff, &a->r_tr, &a->r_pow, &a->r_envk, &a->r_env,
                    &a->q_len, &a->q_nodes, &a->q_coeff, &a->q_tr, &a->q_pow, &a->q_envk, &a->q_env,
                    &a->density, &a->dn_off, &a->dn, &a->dm_off, &a->dm, &a->prod_off, &a->prod_fac,
                    &a->term_off, &a->term, &a->weights, &a->wpair, &a->ref, &a->pair_ok, &a->Fnorm,
                    &a->c_rows, &a->c_cols, &a->c_vals, &a->edge_count, &a->edge_off, &a->edge_j, &a->edge_d,
                    &a->edge_S, &a->edge_rev, &a->edge_g, &a->site_out, &a->site_E_orig, &a->status};
  for (auto* b : bufs) b->release();
  delete a;
  ws->ace = nullptr;
}

void ace_load(pfw_ws* ws, const pfw_ace_tables* t) {
  if (t->nz < 1 || t->nz > 16) throw Error(PFW_EINVAL, "ACE models support 1 to 16 species channels");
  if (t->lmax < 0 || t->lmax > ACE_LMAX) throw Error(PFW_EINVAL, "ACE lmax must be in 0..6");
  if (t->radial.nchannels < 1) throw Error(PFW_EINVAL, "empty radial basis");
  if (!(std::isfinite(t->cutoff) && t->cutoff > 0)) throw Error(PFW_EINVAL, "invalid ACE cutoff");
  ace_free(ws);
  AceDevice* a = new AceDevice();
  ws->ace = a;
  cudaStream_t st = ws->stream;
  const int nz = t->nz;
  a->nz = nz;
  a->lmax = t->lmax;
  a->nY = (t->lmax + 1) * (t->lmax + 1);
  a->nR = t->radial.nchannels;
  a->nQ = t->pair.nchannels;
  a->D = t->ndensity;
  a->P = t->nproducts;
  a->nB = t->nbasis;
  a->cutoff = t->cutoff;
  a->R = upload_family(t->radial, nz, a->r_len, a->r_nodes, a->r_coeff, a->r_tr, a->r_pow, a->r_envk, a->r_env, st);
  if (a->nQ > 0)
    a->Q = upload_family(t->pair, nz, a->q_len, a->q_nodes, a->q_coeff, a->q_tr, a->q_pow, a->q_envk, a->q_env, st);
  else
    a->Q = a->R;
  // density tables
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
  // products and per-density occurrence lists
  std::vector<int> poff(t->product_offsets, t->product_offsets + a->P + 1);
  if (poff[0] != 0) throw Error(PFW_EINVAL, "product offsets must start at 0");
  std::vector<int> pfac(t->product_factors, t->product_factors + poff[a->P]);
  std::vector<int> toff(a->D + 1, 0);
  for (int k = 0; k < a->P; ++k) {
    if (poff[k + 1] <= poff[k]) throw Error(PFW_EINVAL, "empty ACE product");
    a->max_order = std::max(a->max_order, poff[k + 1] - poff[k]);
    for (int f = poff[k]; f < poff[k + 1]; ++f) {
      if (pfac[f] < 0 || pfac[f] >= a->D) throw Error(PFW_EINVAL, "invalid product indices");
      toff[pfac[f] + 1]++;
    }
  }
  for (int k = 0; k < a->D; ++k) toff[k + 1] += toff[k];
  std::vector<int2> term(toff[a->D]);
  {
    std::vector<int> fill(toff.begin(), toff.end() - 1);
    for (int k = 0; k < a->P; ++k)
      for (int f = poff[k]; f < poff[k + 1]; ++f) term[fill[pfac[f]]++] = make_int2(k, f - poff[k]);
  }
  upload(a->prod_off, poff.data(), poff.size(), st);
  upload(a->prod_fac, pfac.data(), pfac.size(), st);
  upload(a->term_off, toff.data(), toff.size(), st);
  upload(a->term, term.data(), term.size(), st);
  // precontracted weights w[z][k] = Σ_b C[b,k]·WB[z][b] (ACE/cpu.jl:265-268)
  std::vector<double> wts((size_t)nz * a->P, 0.0);
  for (int z = 0; z < nz; ++z)
    for (int e = 0; e < t->ncoupling; ++e) {
      const int r = t->coupling_rows[e], c = t->coupling_cols[e];
      if (r < 0 || r >= a->nB || c < 0 || c >= a->P) throw Error(PFW_EINVAL, "invalid coupling entry");
      wts[(size_t)z * a->P + c] += t->coupling_vals[e] * t->WB[(size_t)z * a->nB + r];
    }
  upload(a->weights, wts.data(), wts.size(), st);
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
  upload(a->c_rows, t->coupling_rows, t->ncoupling, st);
  upload(a->c_cols, t->coupling_cols, t->ncoupling, st);
  upload(a->c_vals, t->coupling_vals, t->ncoupling, st);
  a->ncoupling = t->ncoupling;
  PFW_CUDA(cudaStreamSynchronize(st));
}

static AceParams params_of(AceDevice* a) {
  AceParams p;
  p.R = a->R;
  p.Q = a->Q;
  p.nz = a->nz;
  p.lmax = a->lmax;
  p.nY = a->nY;
  p.nR = a->nR;
  p.nQ = a->nQ;
  p.D = a->D;
  p.P = a->P;
  p.density = a->density.as<int2>();
  p.dn_off = a->dn_off.as<int>();
  p.dn = a->dn.as<int2>();
  p.dm_off = a->dm_off.as<int>();
  p.dm = a->dm.as<int2>();
  p.prod_off = a->prod_off.as<int>();
  p.prod_fac = a->prod_fac.as<int>();
  p.term_off = a->term_off.as<int>();
  p.term = a->term.as<int2>();
  p.weights = a->weights.as<double>();
  p.wpair = a->wpair.as<double>();
  p.ref = a->ref.as<double>();
  p.pair_ok = a->pair_ok.as<int>();
  p.Fnorm = a->Fnorm.as<double>();
  return p;
}

template <int L>
static void launch_site(const AceParams& p, int n, size_t smem, cudaStream_t st, const int* off, const double4* ed,
                        const double4* pos, double* g, double* out, int want_grad, int* status) {
  PFW_CUDA(cudaFuncSetAttribute(k_ace_site<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_ace_site<L><<<n, ACE_THREADS, smem, st>>>(p, n, off, ed, pos, g, out, want_grad, status);
}

// Build the directed environments of the current geometry (sorted centres).
static void build_edges(pfw_ws* ws, AceDevice* a) {
  const Prepared& P = ws->prep;
  cudaStream_t st = ws->stream;
  const int n = P.n;
  int* count = static_cast<int*>(a->edge_count.ensure(sizeof(int) * std::max(n, 1)));
  int* off = static_cast<int*>(a->edge_off.ensure(sizeof(int) * (n + 1)));
  PFW_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * std::max(n, 1), st));
  bool shift = true;
  for (auto& g : P.sys)
    if (g.minimum_image && !g.fast_shift) shift = false;
  const dim3 grid(grid_for(P.ncells, 4)), block(128);
  if (P.ncells > 0) {
    if (shift) k_edge_count<0><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(),
                                                          ws->cell_start.as<int>(), ws->pos.as<double4>(), P.ncells, count);
    else k_edge_count<1><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(),
                                                   ws->cell_start.as<int>(), ws->pos.as<double4>(), P.ncells, count);
    ws->launches += 1;
  }
  exclusive_scan_i32(ws, count, off, n);
  int total = 0;
  PFW_CUDA(cudaMemcpyAsync(&total, off + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaStreamSynchronize(st));
  a->nedges = total;
  int* ej = static_cast<int*>(a->edge_j.ensure(sizeof(int) * std::max(total, 1)));
  int4* eS = static_cast<int4*>(a->edge_S.ensure(sizeof(int4) * std::max(total, 1)));
  double4* ed = static_cast<double4*>(a->edge_d.ensure(sizeof(double4) * std::max(total, 1)));
  int* rev = static_cast<int*>(a->edge_rev.ensure(sizeof(int) * std::max(total, 1)));
  int* status = static_cast<int*>(a->status.ensure(sizeof(int) * 4));
  if (P.ncells > 0 && total > 0) {
    if (shift)
      k_edge_fill<0><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                             ws->pos.as<double4>(), ws->perm.as<int>(), ws->wind.as<int>(),
                                             ws->X.as<double>(), P.ncells, off, ej, eS, ed);
    else
      k_edge_fill<1><<<grid, block, 0, st>>>(ws->sysgeom.as<SysGeom>(), ws->cell_sys.as<int>(), ws->cell_start.as<int>(),
                                             ws->pos.as<double4>(), ws->perm.as<int>(), ws->wind.as<int>(),
                                             ws->X.as<double>(), P.ncells, off, ej, eS, ed);
    k_edge_rev<<<grid_for(n, 4), 128, 0, st>>>(n, off, ej, eS, rev, status);
    ws->launches += 2;
  }
}

void ace_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev) {
  AceDevice* a = ws->ace;
  if (!a) throw Error(PFW_ESTATE, "no ACE model loaded");
  if (ws->max_species >= a->nz) throw Error(PFW_EINVAL, "ACE model has no element channel for a species");
  cudaStream_t st = ws->stream;
  ws->prep.valid = false;
  ws->stage_begin(3);
  ws->stage_begin(0);
  prepare(ws, a->cutoff);
  ws->stage_end(0);
  int* status = static_cast<int*>(a->status.ensure(sizeof(int) * 4));
  PFW_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * 4, st));
  build_edges(ws, a);
  ws->stage_end(3);
  const int n = ws->prep.n;
  a->n = n;
  const bool want_grad = (req & (PFW_REQ_FORCES | PFW_REQ_VIRIAL)) != 0;
  double* g = static_cast<double*>(a->edge_g.ensure(sizeof(double) * 3 * std::max<int64_t>(a->nedges, 1)));
  double* out = static_cast<double*>(a->site_out.ensure(sizeof(double) * 10 * std::max(n, 1)));
  double* Esite = static_cast<double*>(a->site_E_orig.ensure(sizeof(double) * std::max(n, 1)));
  const AceParams p = params_of(a);
  const size_t smem = SiteSmem::bytes(a->D, a->nY, a->nR);
  if (smem > 200 * 1024) throw Error(PFW_EINVAL, "ACE model too large for the site kernel's shared memory");
  ws->stage_begin(1);
  if (n > 0) {
    const int* off = a->edge_off.as<int>();
    const double4* ed = a->edge_d.as<double4>();
    const double4* pos = ws->pos.as<double4>();
    switch (a->lmax) {
      case 0: launch_site<0>(p, n, smem, st, off, ed, pos, g, out, want_grad, status); break;
      case 1: launch_site<1>(p, n, smem, st, off, ed, pos, g, out, want_grad, status); break;
      case 2: launch_site<2>(p, n, smem, st, off, ed, pos, g, out, want_grad, status); break;
      case 3: launch_site<3>(p, n, smem, st, off, ed, pos, g, out, want_grad, status); break;
      case 4: launch_site<4>(p, n, smem, st, off, ed, pos, g, out, want_grad, status); break;
      case 5: launch_site<5>(p, n, smem, st, off, ed, pos, g, out, want_grad, status); break;
      default: launch_site<6>(p, n, smem, st, off, ed, pos, g, out, want_grad, status); break;
    }
    ws->launches += 1;
  }
  ws->stage_end(1);
  ws->stage_begin(2);
  if (F_dev && n > 0) {
    if (want_grad) {
      k_ace_gather<<<grid_for(n, 128), 128, 0, st>>>(n, a->edge_off.as<int>(), a->edge_rev.as<int>(), g,
                                                     ws->perm.as<int>(), F_dev);
      ws->launches += 1;
    } else {
      PFW_CUDA(cudaMemsetAsync(F_dev, 0, sizeof(double) * 3 * n, st));
    }
  }
  double* E = E_dev ? E_dev : static_cast<double*>(ws->out_E.ensure(sizeof(double)));
  double* W = W_dev ? W_dev : static_cast<double*>(ws->out_W.ensure(sizeof(double) * 9));
  k_ace_reduce<<<1, 256, 0, st>>>(n, out, ws->perm.as<int>(), E, W, Esite);
  ws->launches += 1;
  ws->stage_end(2);
  a->evaluated = true;
  int hs[4];
  PFW_CUDA(cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaStreamSynchronize(st));
  PFW_CUDA(cudaGetLastError());
  if (hs[0] & 2) throw Error(PFW_EDOMAIN, "coincident physical atoms have undefined harmonics / pair envelope");
  if (hs[0] & 4) throw Error(PFW_EINVAL, "internal: reverse edge not found");
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

}  // namespace pfw
