// ace_site.cuh — the persistent ACE site kernel.
//
// One CTA per SM slot holds the model's product, adjoint-term and density
// tables in shared memory (loaded once; the precontracted weights are read
// through L1; a model whose product or term tables do not fit leaves them in
// global memory, read through L1), and
// runs G groups of ACE_GROUP (64) threads; each group evaluates one site at a time
// (sites strided over the grid), with its own A/dA vectors and an edge-chunk
// working set of CH edges:
//
//   pass 1 (per chunk)  radial spline values R[t,n], harmonics Y[t,m], pair
//                       energy; A[a] += Σ_t R[t,n_a]·Y[t,m_a]
//   products            P_k = Π A (≤ 4 factors, missing factors point at the
//                       sentinel A[D] = 1), E_i = ref + Σ w_k P_k + pair;
//                       dA[a] = Σ_{terms of a} w_k Π(other factors)
//   pass 2 (per chunk)  R, dR/dr, Y, ∇Y; T1[t,n] = Σ dA·Y, T2[t,m] = Σ dA·R;
//                       g_t = r̂ (Σ_n dR·T1 + Σ Wpair·dQ) + Σ_m ∇Y·T2
//
// Arithmetic type T is double for the plain path and float for the mixed
// form (energies and the virial are accumulated in double either way).
#pragma once
#include "ace_math.cuh"

namespace pfw {

// Threads per site group and site groups per CTA (512 threads per CTA).
#ifndef PFW_ACE_GROUP
#define PFW_ACE_GROUP 64
#endif
constexpr int ACE_GROUP = PFW_ACE_GROUP;
constexpr int ACE_MAX_GROUPS = 512 / ACE_GROUP;
constexpr int ACE_MAX_CHUNK = ACE_GROUP / 4;  // at least four threads per edge of a chunk
static_assert(ACE_GROUP == 64 || ACE_GROUP == 128, "site groups of 64 or 128 threads");

struct AceTables {
  RadialDev R, Q;
  int nz, nY, nR, nQ, D, P, T;    // T: number of adjoint terms
  const ushort4* prods;           // [P] factor indices, D = sentinel
  const int* term_off;            // [D+1]
  const ushort4* terms;           // [T] (k, other factors)
  const int2* density;            // [D] (n, m)
  const int* dn_off;              // [nR+1]
  const int2* dn;                 // [D] (a, m)
  const int* dm_off;              // [nY+1]
  const int2* dm;                 // [D] (a, n)
  const double* weights;          // [nz][P]
  const float* weights32;         // the same in FP32 (mixed-form adjoints)
  int nB;                         // invariants (fitting features)
  const int* crow_off;            // [nB+1] coupling rows (CSR)
  const int* crow_k;              // product of each stored entry
  const double* crow_val;         //   and its value
  const double* wpair;            // [nz][nQ]
  const double* ref;              // [nz]
  const int* pair_ok;             // [nz]
  const double* Fnorm;            // [(L+1)^2]
  int solid;                      // 1: real solid harmonics r^l·Y_lm
};

// Learned per-atom surrogate: an ensemble of M MLPs per centre species,
// nin → H → H → 1 with SiLU, BF16 weights (FP32 arithmetic), on the
// standardised low-order invariants of a restricted ACE model (its nB
// invariants B = C·P, then its nQ pair sums).  The site kernel runs twice
// around the batched MLP (k_sur_mlp): pass 1 stores every site's A-basis and
// features, pass 2 turns dE/dfeature into per-site product and pair weights
// and runs the ACE pullback with them.
struct SurParams {
  int nin, H, M;
  const unsigned short* W1;   // [nz][M][H][nin]  (BF16 bits)
  const unsigned short* W2;   // [nz][M][H][H]
  const unsigned short* w3;   // [nz][M][H]
  const float *b1, *b2;       // [nz][M][H]
  const float* b3;            // [nz][M]
  const double *x_mean, *x_std;  // [nz][nin] standardisation (double: features can sit far from zero)
  const float *x_lo, *x_hi;      // [nz][nin] standardised accepted range, margin included
  const double *y_mean, *y_std;  // [nz]
  float tau;                  // ensemble standard deviation gate (eV)
  const int* ccol_off;        // [P+1] restricted coupling by product (CSC)
  const int* ccol_b;
  const double* ccol_val;
  int* flags;                 // [n] per sorted site: 1 = outside the gate, evaluate with ACE
  double* site_A;             // [n][D] A-basis of each site (feature pass → pullback pass)
  double* site_feat;          // [n][nin] features of each site, own species block
  double* site_df;            // [n][nin] dE/dfeature (MLP pass)
  double* site_e;             // [n] MLP site energy without the reference energy
};

// shared-memory layout (byte offsets), computed identically on host and device
struct AceLayout {
  int CH, G;
  int RS, YS;  // odd row strides of the per-edge R and Y tables (bank-conflict padding)
  int feat;    // 1: per-unit fitting features are accumulated
  int nfeat;   // nz * (nB + nQ)
  int sur;     // surrogate pass: 1 features, 2 pullback with per-site weights
  int gtab;    // tables read from global memory (L1-cached) instead of staged:
               // bit 0 the adjoint terms, bit 1 the products (large models)
  size_t prods, terms, term_off, density, dn_off, dn, dm_off, dm, radp, tables_end;
  size_t group_bytes, total;
  // group-relative double offsets
  int A, dA, Y, dY, R, dR, T1, T2, esc, F, QV, WK, WQ, DD, QD, ints;
  __host__ __device__ static size_t align16(size_t v) { return (v + 15) & ~size_t(15); }
  __host__ __device__ void make(const AceTables& t, int ch, int g, int with_feat = 0, int sur_pass = 0,
                                int global_tables = 0, int design = 0) {
    CH = ch;
    G = g;
    sur = sur_pass;
    gtab = global_tables;
    feat = with_feat || sur == 1;
    nfeat = t.nz * (t.nB + t.nQ);
    size_t o = 0;
    prods = o; o = align16(o + ((gtab & 2) ? 0 : sizeof(ushort4) * t.P));
    terms = o; o = align16(o + ((gtab & 1) ? 0 : sizeof(ushort4) * t.T));
    term_off = o; o = align16(o + sizeof(int) * (t.D + 1));
    density = o; o = align16(o + sizeof(int2) * t.D);
    dn_off = o; o = align16(o + sizeof(int) * (t.nR + 1));
    dn = o; o = align16(o + sizeof(int2) * t.D);
    dm_off = o; o = align16(o + sizeof(int) * (t.nY + 1));
    dm = o; o = align16(o + sizeof(int2) * t.D);
    radp = o; o = align16(o + (design ? 0 : sizeof(double) * 2 * RADP_W * t.nz * t.nz));  // R and pair parameters
    tables_end = o;
    RS = t.nR | 1;
    YS = t.nY | 1;
    int d = 0;
    A = d; d += t.D + 1;
    dA = d; d += t.D + 1;
    Y = d; d += CH * YS;
    dY = d; d += CH * YS * 3;
    R = d; d += CH * RS;
    dR = d; d += CH * RS;
    T1 = d; d += CH * RS;
    T2 = d; d += CH * YS;
    esc = d; d += CH * 10 + 4 * 10;  // per-edge scalars, then warp partials
    F = d; d += feat ? nfeat : 0;     // unit feature accumulator
    QV = d; d += feat ? CH * t.nQ : 0;  // pair radial values of the chunk
    WK = d; d += sur == 2 ? t.P : 0;   // per-site product weights
    WQ = d; d += sur == 2 ? t.nQ : 0;  // per-site pair weights
    DD = d; d += design ? CH * (t.D + 1) * 3 : 0;  // design rows: ∂A_a/∂d of the chunk's edges (+ a zero row)
    QD = d; d += design ? CH * t.nQ * 2 : 0;  // design rows: pair values and d/dr
    ints = d; d += CH;               // 2 ints per edge
    group_bytes = align16(sizeof(double) * d);
    total = tables_end + group_bytes * G;
  }
};

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(ACE_GROUP) : "memory");
}

template <class T>
struct EdgeScalars {
  // per-edge values of the current chunk (index t): u, e, de, du, dq, r, dx, dy, dz
  double *u, *e, *de, *du, *dq, *r, *dx, *dy, *dz, *wred;
  int *k0, *pidx;
};

// Per-edge set-up of one chunk, ACE_GROUP / CH threads per edge (4 or 8;
// lt = tpe·t + q): q = 0 the R-family transform/interval/envelope (shared
// with the edge's other threads by shuffles), q = 1 the pair radials,
// harmonics split by azimuthal order m ≡ q (mod tpe), and the R channels
// n ≡ q (mod tpe)
// (values, and derivatives when Grad) — so no separate radial phase and
// barrier follow.
// Channels n ≡ q (mod tpe) of one radial family for one edge, NB channels'
// coefficients loaded before any is evaluated (independent loads in flight).
// on(n, v, dv) receives each channel's value and d/dr (dv unused without Grad).
template <class T, bool Grad, int NB, class On>
__device__ __forceinline__ void edge_channels(const RadialDev& f, int pidx, const EdgeRadial<T>& er, int q, int tpe,
                                              On&& on) {
  constexpr bool F32 = std::is_same<T, float>::value;
  const bool use32 = F32 && f.coeff32 != nullptr;  // the mixed form reads FP32 coefficients (one 16-B load)
  const size_t base = (((size_t)pidx * (f.nknots - 1) + er.k0) * f.nch) * 4;
  for (int n0 = q; n0 < f.nch; n0 += NB * tpe) {
    T c[NB][4];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int n = n0 + j * tpe;
      if (n < f.nch) {
        if (use32) {
          const float4 cf = __ldg(reinterpret_cast<const float4*>(f.coeff32 + base + 4 * (size_t)n));
          c[j][0] = (T)cf.x; c[j][1] = (T)cf.y; c[j][2] = (T)cf.z; c[j][3] = (T)cf.w;
        } else {
          const double2* cp = reinterpret_cast<const double2*>(f.coeff + base + 4 * (size_t)n);
          const double2 lo = __ldg(cp), hi = __ldg(cp + 1);
          c[j][0] = (T)lo.x; c[j][1] = (T)lo.y; c[j][2] = (T)hi.x; c[j][3] = (T)hi.y;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int n = n0 + j * tpe;
      if (n >= f.nch) break;
      const T c0 = c[j][0], c1 = c[j][1], c2 = c[j][2], c3 = c[j][3], u = er.u;
      const T v = ((c3 * u + c2) * u + c1) * u + c0;
      if constexpr (Grad) {
        const T dv = (T(3) * c3 * (u * u) + T(2) * c2 * u + c1);
        on(n, er.e * v, er.de * v + er.e * dv * er.du);
      } else {
        on(n, er.e * v, T(0));
      }
    }
  }
}

// Per-edge set-up of one chunk, ACE_GROUP / CH threads per edge (4 or 8;
// lt = tpe·t + q): q = 0 the R-family transform/interval/envelope, q = 1 the
// pair family's (both shared with the edge's other threads by shuffles),
// harmonics split by azimuthal order m ≡ q (mod tpe), the R and pair
// channels n ≡ q (mod tpe) (values, and derivatives when Grad); the pair
// energy and Σ Wpair·dQ/dr are summed over the edge's threads.
template <int L, class T, bool Grad>
__device__ __forceinline__ void ace_chunk_edges(const AceTables& p, double* gbase, const AceLayout& lay,
                                                const EdgeScalars<T>& es, const double4* __restrict__ edge_d, int e0,
                                                int nc, int iz, int lt, double& e_acc, int* status,
                                                const double* wq = nullptr, const double* radp = nullptr) {
  const int tpe = ACE_GROUP / lay.CH, tsh = 31 - __clz(tpe);
  const int t = lt >> tsh, q = lt & (tpe - 1);
  if (t >= nc) return;
  const double4 d = edge_d[e0 + t];
  const int zj = min(max((int)d.w, 0), p.nz - 1);
  const int pidx = iz * p.nz + zj;
  const T dx = (T)d.x, dy = (T)d.y, dz = (T)d.z;
  const T r0 = sqrt(dx * dx + dy * dy + dz * dz);
  const T r = r0 > T(0) ? r0 : T(1);
  const bool pair = p.nQ > 0 && p.pair_ok[zj];  // the same for all of the edge's threads
  EdgeRadial<T> er{}, eq{};
  // thread 0 of the edge sets up the R family, thread 1 the pair family: one
  // call with the family chosen per thread, so the two run side by side
  // rather than as two branches of the warp
  if (q == 0 || (q == 1 && pair)) {
    RadialDev fam = p.R;
    const double* famp = radp;
    if (q == 1) {
      fam = p.Q;
      famp = radp ? radp + RADP_W * p.nz * p.nz : nullptr;
    }
    const EdgeRadial<T> ex = edge_radial<T>(fam, pidx, r, famp);
    if (q == 0) er = ex;
    else eq = ex;
  }
  if (q == 0) {
    if (!(r0 > T(0))) atomicOr(status, 2);
    es.r[t] = r;
    es.dx[t] = dx;
    es.dy[t] = dy;
    es.dz[t] = dz;
    es.k0[t] = er.k0;
    es.pidx[t] = pidx;
    es.u[t] = er.u;
    es.e[t] = er.e;
    es.de[t] = er.de;
    es.du[t] = er.du;
  } else if (q == 1 && pair) {
    if (!eq.ok) atomicOr(status, 2);
  }
  // the radial set-ups from the edge's first two threads (the tpe threads of
  // an edge are consecutive lanes of one warp, all inside or all outside nc)
  const int lane = lt & 31;
  const int src = lane & ~(tpe - 1);
  const unsigned seg = ((1u << tpe) - 1u) << src;
  er.k0 = __shfl_sync(seg, er.k0, src);
  er.u = __shfl_sync(seg, er.u, src);
  er.e = __shfl_sync(seg, er.e, src);
  if constexpr (Grad) {
    er.de = __shfl_sync(seg, er.de, src);
    er.du = __shfl_sync(seg, er.du, src);
  }
  // the chunk tables hold T: FP64 for the plain path, FP32 for the mixed form
  T* Rt = reinterpret_cast<T*>(gbase + lay.R) + t * lay.RS;
  T* dRt = reinterpret_cast<T*>(gbase + lay.dR) + t * lay.RS;
  edge_channels<T, Grad, 1>(p.R, pidx, er, q, tpe, [&](int n, T v, T dv) {
    Rt[n] = v;
    if constexpr (Grad) dRt[n] = dv;
  });
  if (p.nQ > 0) {
    double* qv = (!Grad && lay.feat) ? gbase + lay.QV + t * p.nQ : nullptr;
    double qe = 0.0;
    T qd = T(0);
    if (pair) {
      eq.k0 = __shfl_sync(seg, eq.k0, src + 1);
      eq.u = __shfl_sync(seg, eq.u, src + 1);
      eq.e = __shfl_sync(seg, eq.e, src + 1);
      if constexpr (Grad) {
        eq.de = __shfl_sync(seg, eq.de, src + 1);
        eq.du = __shfl_sync(seg, eq.du, src + 1);
      }
      const double* wp = wq ? wq : p.wpair + (size_t)iz * p.nQ;
      edge_channels<T, Grad, 1>(p.Q, pidx, eq, q, tpe, [&](int n, T v, T dv) {
        qe += (double)v * wp[n];
        if constexpr (Grad) qd += (T)wp[n] * dv;
        if (qv) qv[n] = v;
      });
    } else if (qv) {
      for (int n = q; n < p.nQ; n += tpe) qv[n] = 0.0;
    }
    for (int o = 1; o < tpe; o <<= 1) {
      qe += __shfl_xor_sync(seg, qe, o);
      qd += __shfl_xor_sync(seg, qd, o);
    }
    if (q == 0) {
      if (!Grad) e_acc += qe;
      es.dq[t] = qd;
    }
  } else if (q == 0) {
    es.dq[t] = T(0);
  }
  // harmonics last: the radial set-ups are dead by now
  T* Yt = reinterpret_cast<T*>(gbase + lay.Y) + t * lay.YS;
  T* dYt = reinterpret_cast<T*>(gbase + lay.dY) + t * lay.YS * 3;
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    if ((m & (tpe - 1)) != q) continue;
    harmonics_m<T, Grad, L>(
        p.Fnorm, r, dx, dy, dz, m,
        [&](int idx, const Jet<T, Grad>& j) {
          Yt[idx] = j.v;
          if constexpr (Grad) {
            dYt[3 * idx] = j.gx;
            dYt[3 * idx + 1] = j.gy;
            dYt[3 * idx + 2] = j.gz;
          }
        },
        p.solid != 0);
  }
}

// Row sums of a CSR list (rows: off[r] .. off[r+1]) with the entries split
// evenly over the group's threads.  The ACE lists are stored by row and their
// lengths are very uneven (one density of the C3 model owns 265 of its 5,691
// adjoint terms), so a thread per row waits on the longest rows.  Each thread
// sums its contiguous share row by row (val(q) gives entry q; the sum is
// accumulated in Acc); a row split between threads is finished by the thread
// holding its first entry, which adds the later threads' partial sums in
// thread order — a fixed order, so the result is deterministic.  put(r, sum)
// receives every row that has entries, once.  scratch: 3·ACE_GROUP doubles
// that are free during the call; every thread of the group must call.
template <class Acc, class Val, class Put>
__device__ __forceinline__ void balanced_rows(int nrows, const int* __restrict__ off, double* __restrict__ scratch,
                                              int lt, int g, Val&& val, Put&& put) {
  const int Tn = off[nrows];
  double* plo = scratch;
  double* phi = scratch + ACE_GROUP;
  int* alo = reinterpret_cast<int*>(scratch + 2 * ACE_GROUP);
  int* ahi = alo + ACE_GROUP;
  const int q0 = (int)((int64_t)lt * Tn / ACE_GROUP), q1 = (int)((int64_t)(lt + 1) * Tn / ACE_GROUP);
  alo[lt] = q0 < q1 ? -1 : -2;  // -2: an empty share (fewer entries than threads), skipped when combining
  ahi[lt] = -1;
  group_sync(g);
  if (q0 < q1) {
    int lo = 0, hi = nrows - 1;  // the row of entry q0: the last r with off[r] <= q0
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (off[mid] <= q0) lo = mid;
      else hi = mid - 1;
    }
    int r = lo, q = q0;
    while (q < q1) {
      const int qe = min(off[r + 1], q1);
      const bool left = q == q0 && off[r] < q0;        // continues an earlier thread's share
      const bool right = qe == q1 && q1 < off[r + 1];  // continues into a later thread's share
      Acc acc = Acc(0);
      for (; q < qe; ++q) acc += val(q);
      if (left) {
        plo[lt] = (double)acc;
        alo[lt] = r;
      } else if (right) {
        phi[lt] = (double)acc;
        ahi[lt] = r;
      } else if (off[r + 1] > off[r]) {
        put(r, (double)acc);
      }
      ++r;
    }
  }
  group_sync(g);
  if (ahi[lt] >= 0) {
    const int r = ahi[lt];
    double acc = phi[lt];
    for (int t = lt + 1; t < ACE_GROUP && (alo[t] == r || alo[t] == -2); ++t)
      if (alo[t] == r) acc += plo[t];
    put(r, acc);
  }
}

// dA[a] = Σ_{terms (k, f1, f2, f3) of density a} w_k·A[f1]·A[f2]·A[f3], the
// terms balanced over the group's threads (densities without terms stay 0).
template <class T, class Wt>
__device__ __forceinline__ void adjoint_terms(int D, const int* __restrict__ toff, const ushort4* __restrict__ terms,
                                              const T* __restrict__ A, T* __restrict__ dA,
                                              double* __restrict__ scratch, int lt, int g, Wt&& wgt) {
  for (int a = lt; a < D; a += ACE_GROUP) dA[a] = T(0);
  balanced_rows<T>(
      D, toff, scratch, lt, g,
      [&](int q) {
        const ushort4 tm = terms[q];
        return (T)wgt(tm.x) * ((T)A[tm.y] * (T)A[tm.z] * (T)A[tm.w]);
      },
      [&](int a, double v) { dA[a] = (T)v; });
}

template <int L, class T, int SUR = 0>
__global__ void __launch_bounds__(ACE_MAX_GROUPS * ACE_GROUP)
    k_ace_sites(AceTables p, AceLayout lay, SurParams sp, int nunits, const int* __restrict__ unit_begin,
                const int* __restrict__ unit_sites, int cap,
                const int* __restrict__ edge_off, const double4* __restrict__ edge_d, const double4* __restrict__ pos,
                double* __restrict__ edge_g, double* __restrict__ unit_out, double* __restrict__ unit_feat,
                int want_grad, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  // ---- stage the model tables once per CTA ----
  ushort4* st_prods = reinterpret_cast<ushort4*>(smem + lay.prods);
  ushort4* st_terms = reinterpret_cast<ushort4*>(smem + lay.terms);
  const ushort4* s_prods = (lay.gtab & 2) ? p.prods : st_prods;
  const ushort4* s_terms = (lay.gtab & 1) ? p.terms : st_terms;
  int* s_toff = reinterpret_cast<int*>(smem + lay.term_off);
  int2* s_dens = reinterpret_cast<int2*>(smem + lay.density);
  int* s_dnoff = reinterpret_cast<int*>(smem + lay.dn_off);
  int2* s_dn = reinterpret_cast<int2*>(smem + lay.dn);
  int* s_dmoff = reinterpret_cast<int*>(smem + lay.dm_off);
  int2* s_dm = reinterpret_cast<int2*>(smem + lay.dm);
  if (!(lay.gtab & 2))
    for (int k = threadIdx.x; k < p.P; k += blockDim.x) st_prods[k] = p.prods[k];
  if (!(lay.gtab & 1))
    for (int k = threadIdx.x; k < p.T; k += blockDim.x) st_terms[k] = p.terms[k];
  for (int k = threadIdx.x; k <= p.D; k += blockDim.x) s_toff[k] = p.term_off[k];
  for (int k = threadIdx.x; k < p.D; k += blockDim.x) {
    s_dens[k] = p.density[k];
    s_dn[k] = p.dn[k];
    s_dm[k] = p.dm[k];
  }
  for (int k = threadIdx.x; k <= p.nR; k += blockDim.x) s_dnoff[k] = p.dn_off[k];
  for (int k = threadIdx.x; k <= p.nY; k += blockDim.x) s_dmoff[k] = p.dm_off[k];
  double* s_radp = reinterpret_cast<double*>(smem + lay.radp);
  stage_radial_params(p.R, s_radp, threadIdx.x, blockDim.x);
  if (p.nQ > 0) stage_radial_params(p.Q, s_radp + RADP_W * p.nz * p.nz, threadIdx.x, blockDim.x);
  __syncthreads();

  const int g = threadIdx.x / ACE_GROUP, lt = threadIdx.x % ACE_GROUP;
  if (g >= lay.G) return;
  double* gb = reinterpret_cast<double*>(smem + lay.tables_end + lay.group_bytes * g);
  // per-group tables in T (double-sized slots: the FP32 form uses the first half)
  T* A = reinterpret_cast<T*>(gb + lay.A);
  T* dA = reinterpret_cast<T*>(gb + lay.dA);
  T* Yc = reinterpret_cast<T*>(gb + lay.Y);
  T* dYc = reinterpret_cast<T*>(gb + lay.dY);
  T* Rc = reinterpret_cast<T*>(gb + lay.R);
  T* dRc = reinterpret_cast<T*>(gb + lay.dR);
  T* T1 = reinterpret_cast<T*>(gb + lay.T1);
  T* T2 = reinterpret_cast<T*>(gb + lay.T2);
  double* const chunk_scratch = gb + lay.Y;  // free between the passes
  EdgeScalars<T> es;
  const int CH = lay.CH;
  double* e0p = gb + lay.esc;
  es.u = e0p; es.e = e0p + CH; es.de = e0p + 2 * CH; es.du = e0p + 3 * CH; es.dq = e0p + 4 * CH;
  es.r = e0p + 5 * CH; es.dx = e0p + 6 * CH; es.dy = e0p + 7 * CH; es.dz = e0p + 8 * CH;
  es.wred = e0p + 10 * CH;
  es.k0 = reinterpret_cast<int*>(gb + lay.ints);
  es.pidx = es.k0 + CH;
  const int D = p.D, nY = p.nY, nR = p.nR, P = p.P, RS = lay.RS, YS = lay.YS;
  const int lane = lt & 31, wg = lt >> 5;

  double* Facc = gb + lay.F;
  const double* QVc = gb + lay.QV;
  for (int unit = blockIdx.x * lay.G + g; unit < nunits; unit += gridDim.x * lay.G) {
   double e_acc = 0.0;
   double wv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
   if (lay.feat) {
     group_sync(g);
     for (int k = lt; k < lay.nfeat; k += ACE_GROUP) Facc[k] = 0.0;
   }
   const int s_begin = unit_sites ? unit_sites[unit] : unit_begin[unit];
   const int s_end = unit_sites ? s_begin + 1 : unit_begin[unit + 1];
   for (int s = s_begin; s < s_end; ++s) {
    const int iz = min(max((int)pos[s].w, 0), p.nz - 1);
    const int eb = min(edge_off[s], cap), E = min(edge_off[s + 1], cap) - eb;
    if (lt == 0) e_acc += p.ref[iz];
    if (SUR == 1 && s > s_begin) {  // features are per site
      group_sync(g);
      for (int k = lt; k < lay.nfeat; k += ACE_GROUP) Facc[k] = 0.0;
    }
    group_sync(g);
    if (SUR == 2)  // the feature pass's A-basis
      for (int a = lt; a <= D; a += ACE_GROUP) A[a] = (a == D) ? T(1) : (T)sp.site_A[(size_t)s * D + a];
    else
      for (int a = lt; a <= D; a += ACE_GROUP) A[a] = (a == D) ? T(1) : T(0);
    // ---- pass 1: A-basis ----
    for (int c0 = 0; c0 < (SUR == 2 ? 0 : E); c0 += CH) {
      const int nc = min(CH, E - c0);
      group_sync(g);
      ace_chunk_edges<L, T, false>(p, gb, lay, es, edge_d, eb + c0, nc, iz, lt, e_acc, status, nullptr, s_radp);
      group_sync(g);
      if (lay.feat)  // Σ_j Q[j,n] of the centre's species block (fitting.jl:29)
        for (int n = lt; n < p.nQ; n += ACE_GROUP) {
          double acc = 0.0;
          for (int t = 0; t < nc; ++t) acc += QVc[t * p.nQ + n];
          Facc[p.nz * p.nB + iz * p.nQ + n] += acc;
        }
      for (int a = lt; a < D; a += ACE_GROUP) {
        const int2 nm = s_dens[a];
        T acc = (T)A[a];
        for (int t = 0; t < nc; ++t) acc += (T)Rc[t * RS + nm.x] * (T)Yc[t * YS + nm.y];
        A[a] = acc;
      }
    }
    group_sync(g);
    // ---- products, energy, adjoints ----
    const double* __restrict__ w = p.weights + (size_t)iz * P;
    if (!SUR)
      for (int k = lt; k < P; k += ACE_GROUP) {
        const ushort4 f = s_prods[k];
        e_acc += __ldg(w + k) * (double)((T)A[f.x] * (T)A[f.y] * (T)A[f.z] * (T)A[f.w]);
      }
    // the chunk tables (Y … T2) are free between the passes: balanced adjoints when they hold the scratch
    const bool balanced = lay.CH * (5 * lay.YS + 3 * lay.RS) >= 3 * ACE_GROUP;
    if (!SUR && want_grad) {
      if (balanced) {
        if constexpr (std::is_same<T, float>::value) {
          const float* w32 = p.weights32 + (size_t)iz * P;
          adjoint_terms<T>(D, s_toff, s_terms, A, dA, chunk_scratch, lt, g, [&](int k) { return __ldg(w32 + k); });
        } else {
          adjoint_terms<T>(D, s_toff, s_terms, A, dA, chunk_scratch, lt, g, [&](int k) { return __ldg(w + k); });
        }
      } else {
        for (int a = lt; a < D; a += ACE_GROUP) {
          T acc = T(0);
          for (int q = s_toff[a]; q < s_toff[a + 1]; ++q) {
            const ushort4 tm = s_terms[q];
            acc += (T)__ldg(w + tm.x) * ((T)A[tm.y] * (T)A[tm.z] * (T)A[tm.w]);
          }
          dA[a] = acc;
        }
      }
    }
    if (lay.feat && SUR != 2) {  // B = C·P of the centre's species block (fitting.jl:28)
      if (balanced) {
        group_sync(g);  // the adjoint's scratch is read by its combining threads until here
        balanced_rows<double>(
            p.nB, p.crow_off, chunk_scratch, lt, g,
            [&](int q) {
              const ushort4 f = s_prods[p.crow_k[q]];
              return p.crow_val[q] * (double)((T)A[f.x] * (T)A[f.y] * (T)A[f.z] * (T)A[f.w]);
            },
            [&](int b, double v) { Facc[iz * p.nB + b] += v; });
      } else {
        for (int b = lt; b < p.nB; b += ACE_GROUP) {
          double acc = 0.0;
          for (int q = p.crow_off[b]; q < p.crow_off[b + 1]; ++q) {
            const ushort4 f = s_prods[p.crow_k[q]];
            acc += p.crow_val[q] * (double)((T)A[f.x] * (T)A[f.y] * (T)A[f.z] * (T)A[f.w]);
          }
          Facc[iz * p.nB + b] += acc;
        }
      }
    }
    const double* wq = nullptr;
    if constexpr (SUR == 1) {
      // ---- surrogate feature pass: keep A and the own-species features ----
      group_sync(g);
      const int nB = p.nB, nQ = p.nQ, nin = nB + nQ;
      for (int a = lt; a < D; a += ACE_GROUP) sp.site_A[(size_t)s * D + a] = (double)A[a];
      for (int i = lt; i < nin; i += ACE_GROUP)
        sp.site_feat[(size_t)s * nin + i] = i < nB ? Facc[iz * nB + i] : Facc[p.nz * nB + iz * nQ + (i - nB)];
    }
    if constexpr (SUR == 2) {
      // ---- surrogate pullback: dE/dB through the coupling onto the products,
      //      dE/dQ onto the pair radials, then the ordinary adjoint ----
      const int nB = p.nB, nin = nB + p.nQ;
      const double* df = sp.site_df + (size_t)s * nin;
      double* wk = gb + lay.WK;
      double* wqs = gb + lay.WQ;
      for (int k = lt; k < P; k += ACE_GROUP) {
        double acc = 0.0;
        for (int q = sp.ccol_off[k]; q < sp.ccol_off[k + 1]; ++q) acc += sp.ccol_val[q] * df[sp.ccol_b[q]];
        wk[k] = acc;
      }
      for (int n = lt; n < p.nQ; n += ACE_GROUP) wqs[n] = df[nB + n];
      if (lt == 0) e_acc += sp.site_e[s];
      group_sync(g);
      wq = wqs;
      if (want_grad) {
        if (balanced) {
          adjoint_terms<T>(D, s_toff, s_terms, A, dA, chunk_scratch, lt, g, [&](int k) { return wk[k]; });
        } else {
          for (int a = lt; a < D; a += ACE_GROUP) {
            T acc = T(0);
            for (int q = s_toff[a]; q < s_toff[a + 1]; ++q) {
              const ushort4 tm = s_terms[q];
              acc += (T)wk[tm.x] * ((T)A[tm.y] * (T)A[tm.z] * (T)A[tm.w]);
            }
            dA[a] = acc;
          }
        }
      }
    }
    // ---- pass 2: pullback ----
    if (want_grad) {
      for (int c0 = 0; c0 < E; c0 += CH) {
        const int nc = min(CH, E - c0);
        group_sync(g);
        double dummy = 0.0;
        ace_chunk_edges<L, T, true>(p, gb, lay, es, edge_d, eb + c0, nc, iz, lt, dummy, status, wq, s_radp);
        group_sync(g);
        // T1[t, n] = Σ_{(a, m) of radial n} dA[a]·Y[t, m], T2[t, m] = Σ_{(a, n) of order m} dA[a]·R[t, n]:
        // a task is one column (n of T1, then m of T2) for up to four edges, so
        // the column's (a, ·) list and dA values are read once per four edges
        {
          constexpr int EB = 4;
          const int ncol = nR + nY, nblk = (nc + EB - 1) / EB;
          for (int task = lt; task < ncol * nblk; task += ACE_GROUP) {
            const int blk = task / ncol, col = task - blk * ncol;
            const int t0 = blk * EB, tn = min(EB, nc - t0);
            T acc[EB];
#pragma unroll
            for (int u = 0; u < EB; ++u) acc[u] = T(0);
            // T1 and T2 columns through one code path (the column's list, source
            // table and output chosen per thread), so a warp holding both kinds
            // does not run them as two branches
            const bool isT1 = col < nR;
            const int c = isT1 ? col : col - nR;
            const int* off = isT1 ? s_dnoff : s_dmoff;
            const int2* lst = isT1 ? s_dn : s_dm;
            const T* src = isT1 ? Yc : Rc;
            const int sst = isT1 ? YS : RS;
            T* dst = isT1 ? T1 : T2;
            const int dsto = isT1 ? RS : YS;
            for (int q = off[c]; q < off[c + 1]; ++q) {
              const int2 ai = lst[q];
              const T w = (T)dA[ai.x];
#pragma unroll
              for (int u = 0; u < EB; ++u)
                if (u < tn) acc[u] += w * (T)src[(t0 + u) * sst + ai.y];
            }
#pragma unroll
            for (int u = 0; u < EB; ++u)
              if (u < tn) dst[(t0 + u) * dsto + c] = acc[u];
          }
        }
        group_sync(g);
        // ACE_GROUP / CH threads per edge (4 or 8)
        const int tpe = ACE_GROUP / CH, tsh = 31 - __clz(tpe);
        const int t = lt >> tsh, q4 = lt & (tpe - 1);
        T s1 = T(0), gx = T(0), gy = T(0), gz = T(0);
        if (t < nc) {
          for (int n = q4; n < nR; n += tpe) s1 += (T)dRc[t * RS + n] * (T)T1[t * RS + n];
          for (int m = q4; m < nY; m += tpe) {
            const T t2 = (T)T2[t * YS + m];
            gx += (T)dYc[(t * YS + m) * 3] * t2;
            gy += (T)dYc[(t * YS + m) * 3 + 1] * t2;
            gz += (T)dYc[(t * YS + m) * 3 + 2] * t2;
          }
        }
        for (int o = 1; o < tpe; o <<= 1) {
          s1 += __shfl_xor_sync(0xffffffffu, s1, o);
          gx += __shfl_xor_sync(0xffffffffu, gx, o);
          gy += __shfl_xor_sync(0xffffffffu, gy, o);
          gz += __shfl_xor_sync(0xffffffffu, gz, o);
        }
        if (t < nc && q4 == 0) {
          const T r = (T)es.r[t];
          const T dx = (T)es.dx[t], dy = (T)es.dy[t], dz = (T)es.dz[t];
          const T radial = (s1 + (T)es.dq[t]) / r;
          const double g0 = (double)(radial * dx + gx), g1 = (double)(radial * dy + gy), g2 = (double)(radial * dz + gz);
          double* ge = edge_g + 3 * (size_t)(eb + c0 + t);
          ge[0] = g0;
          ge[1] = g1;
          ge[2] = g2;
          const double dd[3] = {(double)dx, (double)dy, (double)dz}, gg[3] = {g0, g1, g2};
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int a = 0; a < 3; ++a) wv[a + 3 * b] -= dd[a] * gg[b];
        }
      }
    }
   }  // sites of the unit
    // ---- unit energy and virial (warp shuffles, then 4 warp partials) ----
    double vals[10];
    vals[0] = e_acc;
#pragma unroll
    for (int k = 0; k < 9; ++k) vals[k + 1] = wv[k];
#pragma unroll
    for (int k = 0; k < 10; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) vals[k] += __shfl_xor_sync(0xffffffffu, vals[k], o);
    group_sync(g);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < 10; ++k) es.wred[wg * 10 + k] = vals[k];
    group_sync(g);
    if (lt < 10) {
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < ACE_GROUP / 32; ++w) v += es.wred[10 * w + lt];
      unit_out[10 * (size_t)unit + lt] = v;
    }
    if (lay.feat && unit_feat)
      for (int k = lt; k < lay.nfeat; k += ACE_GROUP) unit_feat[(size_t)lay.nfeat * unit + k] = Facc[k];
  }
}

}  // namespace pfw
