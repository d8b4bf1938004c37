// skin.cu — Verlet (skin) reuse of the pair neighbour list across calls.
//
// The reference rebuilds its cell topology on every evaluate! call; its GPU
// pair path keeps a skin list between calls (gpu_skin!, gpu_displacements!,
// NeighbourList/gpu.jl:404-549).  Here, with a skin s > 0 set, the first call
// builds the directed snapshot of all images within c + s (the neighbour
// snapshot kernels, with S relative to the ORIGINAL coordinates) and keeps it
// with a copy of the positions; later calls on the same structure (same atom
// count, cell and periodicity) measure the largest displacement since the
// build and, while it is at most s/2, evaluate only the listed pairs — every
// pair within c now was within c + s then:
//
//   k_pack_list  at a build: (j, S) → one int2 per entry, S as three 10-bit
//                offsets (|S| < 512, else the list path is not used)
//   k_max_disp   largest squared displacement (atomicMax on the FP64 bits)
//   k_pos4       positions and species as one double4 per atom
//   k_pair_list  8 lanes per atom stride over its list: d = (X_j - X_i) + H·S
//                with the exact-rounding intrinsics of the snapshot's R,
//                r² < c² selects the pairs, pair_term as the cell-list kernel;
//                forces written once per atom, E and W per atom
//
// The selected pairs are the reference's up to the rounding of d (the list
// path computes d from the original coordinates and the image shift, as the
// snapshot's R, rather than from wrapped coordinates): pairs within about
// one ulp of the cutoff can differ from the rebuild path.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pair_math.cuh"
#include "pfw_internal.h"

namespace pfw {

struct SkinState {
  bool valid = false;
  double cutoff = 0, built_skin = 0;
  int n = 0;
  double H[9] = {};
  uint8_t pbc[3] = {};
  int kind = -1;
  DevBuf off, j, S, list, Xref, dmax, pos4;
  int64_t builds = 0, reuses = 0;
};

void skin_free(pfw_ws* ws) {
  SkinState* s = ws->skin_state;
  if (!s) return;
  DevBuf* bufs[] = {&s->off, &s->j, &s->S, &s->list, &s->Xref, &s->dmax, &s->pos4};
  for (auto* b : bufs) b->release();
  delete s;
  ws->skin_state = nullptr;
}

// out[0]: the largest squared displacement; out[1] set when a species channel
// lies outside [0, limit) (device-uploaded species are only seen here on a
// reuse step).
__global__ void k_max_disp(int n, const double* __restrict__ X, const double* __restrict__ Xref,
                           const int* __restrict__ species, int limit, unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int z = species[i];
    if (z < 0 || z >= limit) out[1] = 1ull;
    const double dx = X[3 * i] - Xref[3 * i], dy = X[3 * i + 1] - Xref[3 * i + 1], dz = X[3 * i + 2] - Xref[3 * i + 2];
    const double d2 = dx * dx + dy * dy + dz * dz;
    m = (d2 > m || d2 != d2) ? (d2 != d2 ? INFINITY : d2) : m;  // a nonfinite position forces a rebuild
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

constexpr int SKIN_LANES = 8;  // lanes per atom
constexpr int SKIN_SBITS = 10;
constexpr int SKIN_SBIAS = 1 << (SKIN_SBITS - 1);

__global__ void k_pack_list(int64_t m, const int* __restrict__ j, const int* __restrict__ S, int2* __restrict__ out,
                            int* __restrict__ overflow) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
    unsigned packed = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int v = S[3 * q + a] + SKIN_SBIAS;
      if (v < 0 || v >= 2 * SKIN_SBIAS) atomicOr(overflow, 1);
      packed |= (unsigned)(v & (2 * SKIN_SBIAS - 1)) << (SKIN_SBITS * a);
    }
    out[q] = make_int2(j[q], (int)packed);
  }
}

__global__ void k_pos4(int n, const double* __restrict__ X, const int* __restrict__ species,
                       double4* __restrict__ pos4) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pos4[i] = make_double4(X[3 * i], X[3 * i + 1], X[3 * i + 2], (double)species[i]);
}

template <int KIND>
__global__ void __launch_bounds__(256)
    k_pair_list(int n, const int64_t* __restrict__ off, const int2* __restrict__ list,
                const double4* __restrict__ pos4, const double* __restrict__ Hz, double c2, PairParams prm,
                double* __restrict__ F, double* __restrict__ parts, unsigned long long* __restrict__ npairs) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) / SKIN_LANES;
  const int sub = threadIdx.x & (SKIN_LANES - 1);
  const unsigned grp = 0xffu << (threadIdx.x & 24);  // the 8 lanes of this atom
  if (i >= n) return;
  const double4 pi = pos4[i];
  const double xi = pi.x, yi = pi.y, zi = pi.z;
  double arow[4] = {0, 0, 0, 0};
  if (KIND == 0) {
    const int z = min(max((int)pi.w, 0), prm.nz - 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) arow[k] = k < prm.nz ? prm.A[z * prm.nz + k] : 0.0;
  }
  double fx = 0, fy = 0, fz = 0, e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long np = 0;
  const int64_t e1 = off[i + 1];
  const unsigned msk = 2 * SKIN_SBIAS - 1;
  auto visit = [&](const int2 ent, const double4 pj) {
    const unsigned pk = (unsigned)ent.y;
    double sh[3];
    xmatvec(Hz, (double)((int)(pk & msk) - SKIN_SBIAS), (double)((int)((pk >> SKIN_SBITS) & msk) - SKIN_SBIAS),
            (double)((int)((pk >> (2 * SKIN_SBITS)) & msk) - SKIN_SBIAS), sh);
    const double d0 = xadd(xsub(pj.x, xi), sh[0]);
    const double d1 = xadd(xsub(pj.y, yi), sh[1]);
    const double d2 = xadd(xsub(pj.z, zi), sh[2]);
    const double r2 = xr2(d0, d1, d2);
    if (!(r2 < c2)) return;
    ++np;
    double en, coef;
    const int zj = KIND == 0 ? min(max((int)pj.w, 0), 3) : 0;
    pair_term<KIND>(prm, arow[zj], r2, en, coef);
    const double gx = coef * d0, gy = coef * d1, gz = coef * d2;
    fx += gx; fy += gy; fz += gz;
    e += en;
    w[0] += d0 * gx; w[1] += d1 * gy; w[2] += d2 * gz;
    w[3] += d0 * gy; w[4] += d0 * gz; w[5] += d1 * gz;
  };
  // two entries per lane in flight: both list loads, then both position loads
  for (int64_t q = off[i] + sub; q < e1; q += 2 * SKIN_LANES) {
    const int64_t q2 = q + SKIN_LANES;
    const bool second = q2 < e1;
    const int2 ea = list[q];
    const int2 eb = second ? list[q2] : ea;
    const double4 pa = pos4[ea.x];
    const double4 pb = pos4[eb.x];
    visit(ea, pa);
    if (second) visit(eb, pb);
  }
  // fixed-order reduction over the atom's 8 lanes
#pragma unroll
  for (int o = SKIN_LANES / 2; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(grp, fx, o);
    fy += __shfl_xor_sync(grp, fy, o);
    fz += __shfl_xor_sync(grp, fz, o);
    e += __shfl_xor_sync(grp, e, o);
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] += __shfl_xor_sync(grp, w[k], o);
    np += __shfl_xor_sync(grp, np, o);
  }
  if (sub == 0) {
    if (prm.want_f) {
      F[3 * i] = fx;
      F[3 * i + 1] = fy;
      F[3 * i + 2] = fz;
    }
    const bool own = i < prm.n_owned;
    double* p = parts + 8 * (size_t)i;
    p[0] = own ? 0.5 * e : 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) p[1 + k] = own ? -0.5 * w[k] : 0.0;
    p[7] = 0.0;
    if (np) atomicAdd(npairs, np);
  }
}

bool skin_pair_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev) {
  if (!(ws->skin > 0.0) || ws->systems.size() != 1 || ws->opt.precision != PFW_PRECISION_FP64) return false;
  const PairModel& m = ws->pair;
  const pfw::HostSystem& hs = ws->systems[0];
  if (!ws->skin_state) ws->skin_state = new SkinState();
  SkinState& sk = *ws->skin_state;
  cudaStream_t st = ws->stream;
  const int n = ws->n;
  bool rebuild = !sk.valid || sk.cutoff != m.cutoff || sk.built_skin != ws->skin || sk.n != n ||
                 std::memcmp(sk.H, hs.H, sizeof(sk.H)) != 0 || std::memcmp(sk.pbc, hs.pbc, sizeof(sk.pbc)) != 0;
  unsigned long long* dm = static_cast<unsigned long long*>(sk.dmax.ensure(2 * sizeof(unsigned long long)));
  if (!rebuild && n > 0) {
    PFW_CUDA(cudaMemsetAsync(dm, 0, 2 * sizeof(unsigned long long), st));
    k_max_disp<<<std::min(grid_for(n, 256), 1184), 256, 0, st>>>(n, ws->X.as<double>(), sk.Xref.as<double>(),
                                                                  ws->species.as<int>(), ws->species_limit, dm);
    ws->launches += 1;
    unsigned long long bits[2] = {0, 0};
    PFW_CUDA(cudaMemcpyAsync(bits, dm, sizeof(bits), cudaMemcpyDeviceToHost, st));
    PFW_CUDA(cudaStreamSynchronize(st));
    if (bits[1])
      throw Error(PFW_EINVAL, "species channel outside the model's channels (must be >= 0 and < " +
                                  std::to_string(ws->species_limit) + ")");
    double d2;
    std::memcpy(&d2, &bits[0], sizeof(d2));
    if (!(2.0 * std::sqrt(d2) <= ws->skin)) rebuild = true;
  }
  if (rebuild) {
    sk.valid = false;
    const int64_t total = neighbour_build(ws, m.cutoff + ws->skin, false);
    if (total > (int64_t)INT32_MAX) throw Error(PFW_EINVAL, "skin list too large; lower the skin");
    std::swap(sk.off, ws->nb_offsets);
    std::swap(sk.j, ws->nb_j);
    std::swap(sk.S, ws->nb_S);
    ws->nb_total = -1;  // the snapshot buffers now belong to the skin list
    int2* lst = static_cast<int2*>(sk.list.ensure(sizeof(int2) * std::max<int64_t>(total, 1)));
    int* ovf = static_cast<int*>(sk.dmax.ensure(sizeof(unsigned long long)));
    PFW_CUDA(cudaMemsetAsync(ovf, 0, sizeof(int), st));
    if (total > 0) {
      k_pack_list<<<(int)std::min<int64_t>(grid_for(total, 256), 4096), 256, 0, st>>>(total, sk.j.as<int>(),
                                                                                        sk.S.as<int>(), lst, ovf);
      ws->launches += 1;
    }
    int hov = 0;
    PFW_CUDA(cudaMemcpyAsync(&hov, ovf, sizeof(int), cudaMemcpyDeviceToHost, st));
    PFW_CUDA(cudaStreamSynchronize(st));
    if (hov) return false;  // image shifts too large to pack: evaluate by rebuilding
    double* xr = static_cast<double*>(sk.Xref.ensure(sizeof(double) * 3 * std::max(n, 1)));
    if (n > 0) PFW_CUDA(cudaMemcpyAsync(xr, ws->X.ptr, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, st));
    sk.cutoff = m.cutoff;
    sk.built_skin = ws->skin;
    sk.n = n;
    std::memcpy(sk.H, hs.H, sizeof(sk.H));
    std::memcpy(sk.pbc, hs.pbc, sizeof(sk.pbc));
    sk.valid = true;
    sk.builds += 1;
  } else {
    sk.reuses += 1;
  }
  // the cell with open generators zeroed (the snapshot's S is 0 on open axes)
  double Hz[9];
  for (int b = 0; b < 3; ++b)
    for (int a = 0; a < 3; ++a) Hz[a + 3 * b] = hs.pbc[b] ? hs.H[a + 3 * b] : 0.0;
  double* dHz = static_cast<double*>(ws->minmax.ensure(sizeof(double) * 9));
  PFW_CUDA(cudaMemcpyAsync(dHz, Hz, sizeof(Hz), cudaMemcpyHostToDevice, st));
  const PairParams prm = make_pair_params(ws, req);
  double* parts = static_cast<double*>(ws->cellpart.ensure(sizeof(double) * 8 * std::max(n, 1)));
  unsigned long long* np = static_cast<unsigned long long*>(ws->counters.ensure(64)) + 4;
  PFW_CUDA(cudaMemsetAsync(np, 0, sizeof(unsigned long long), st));
  double* F = F_dev ? F_dev : static_cast<double*>(ws->out_F.ensure(sizeof(double) * 3 * std::max(n, 1)));
  ws->stage_begin(1);
  if (n > 0) {
    double4* p4 = static_cast<double4*>(sk.pos4.ensure(sizeof(double4) * n));
    k_pos4<<<grid_for(n, 256), 256, 0, st>>>(n, ws->X.as<double>(), ws->species.as<int>(), p4);
    const int grid = grid_for((int64_t)n * SKIN_LANES, 256);
    if (m.kind == 0)
      k_pair_list<0><<<grid, 256, 0, st>>>(n, sk.off.as<int64_t>(), sk.list.as<int2>(), p4, dHz, m.cutoff * m.cutoff,
                                           prm, F, parts, np);
    else
      k_pair_list<1><<<grid, 256, 0, st>>>(n, sk.off.as<int64_t>(), sk.list.as<int2>(), p4, dHz, m.cutoff * m.cutoff,
                                           prm, F, parts, np);
    ws->launches += 2;
  }
  ws->stage_end(1);
  double* E = E_dev ? E_dev : static_cast<double*>(ws->out_E.ensure(sizeof(double)));
  double* W = W_dev ? W_dev : static_cast<double*>(ws->out_W.ensure(sizeof(double) * 9));
  ws->stage_begin(2);
  reduce_pair_parts(ws, parts, n, 8, E, W);
  ws->stage_end(2);
  PFW_CUDA(cudaGetLastError());
  return true;
}

void skin_stats(pfw_ws* ws, int64_t* builds, int64_t* reuses) {
  const SkinState* s = ws->skin_state;
  if (builds) *builds = s ? s->builds : 0;
  if (reuses) *reuses = s ? s->reuses : 0;
}

}  // namespace pfw
