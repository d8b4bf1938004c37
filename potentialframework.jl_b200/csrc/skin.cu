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
//   k_max_disp   largest squared displacement (atomicMax on the FP64 bits)
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
  DevBuf off, j, S, Xref, dmax;
  int64_t builds = 0, reuses = 0;
};

void skin_free(pfw_ws* ws) {
  SkinState* s = ws->skin_state;
  if (!s) return;
  DevBuf* bufs[] = {&s->off, &s->j, &s->S, &s->Xref, &s->dmax};
  for (auto* b : bufs) b->release();
  delete s;
  ws->skin_state = nullptr;
}

__global__ void k_max_disp(int n, const double* __restrict__ X, const double* __restrict__ Xref,
                           unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double dx = X[3 * i] - Xref[3 * i], dy = X[3 * i + 1] - Xref[3 * i + 1], dz = X[3 * i + 2] - Xref[3 * i + 2];
    const double d2 = dx * dx + dy * dy + dz * dz;
    m = (d2 > m || d2 != d2) ? (d2 != d2 ? INFINITY : d2) : m;  // a nonfinite position forces a rebuild
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

constexpr int SKIN_LANES = 8;  // lanes per atom

template <int KIND>
__global__ void __launch_bounds__(256)
    k_pair_list(int n, const int64_t* __restrict__ off, const int* __restrict__ jl, const int* __restrict__ Sl,
                const double* __restrict__ X, const int* __restrict__ species, const double* __restrict__ Hz,
                double c2, PairParams prm, double* __restrict__ F, double* __restrict__ parts,
                unsigned long long* __restrict__ npairs) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) / SKIN_LANES;
  const int sub = threadIdx.x & (SKIN_LANES - 1);
  const unsigned grp = 0xffu << (threadIdx.x & 24);  // the 8 lanes of this atom
  if (i >= n) return;
  const double xi = X[3 * i], yi = X[3 * i + 1], zi = X[3 * i + 2];
  double arow[4] = {0, 0, 0, 0};
  if (KIND == 0) {
    const int z = min(max(species[i], 0), prm.nz - 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) arow[k] = k < prm.nz ? prm.A[z * prm.nz + k] : 0.0;
  }
  double fx = 0, fy = 0, fz = 0, e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long np = 0;
  const int64_t e1 = off[i + 1];
  for (int64_t q = off[i] + sub; q < e1; q += SKIN_LANES) {
    const int j = jl[q];
    double sh[3];
    xmatvec(Hz, (double)Sl[3 * q], (double)Sl[3 * q + 1], (double)Sl[3 * q + 2], sh);
    const double d0 = xadd(xsub(X[3 * j], xi), sh[0]);
    const double d1 = xadd(xsub(X[3 * j + 1], yi), sh[1]);
    const double d2 = xadd(xsub(X[3 * j + 2], zi), sh[2]);
    const double r2 = xr2(d0, d1, d2);
    if (!(r2 < c2)) continue;
    ++np;
    double en, coef;
    const int zj = KIND == 0 ? min(max(species[j], 0), 3) : 0;
    pair_term<KIND>(prm, arow[zj], r2, en, coef);
    const double gx = coef * d0, gy = coef * d1, gz = coef * d2;
    fx += gx; fy += gy; fz += gz;
    e += en;
    w[0] += d0 * gx; w[1] += d1 * gy; w[2] += d2 * gz;
    w[3] += d0 * gy; w[4] += d0 * gz; w[5] += d1 * gz;
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
  unsigned long long* dm = static_cast<unsigned long long*>(sk.dmax.ensure(sizeof(unsigned long long)));
  if (!rebuild && n > 0) {
    PFW_CUDA(cudaMemsetAsync(dm, 0, sizeof(unsigned long long), st));
    k_max_disp<<<std::min(grid_for(n, 256), 1184), 256, 0, st>>>(n, ws->X.as<double>(), sk.Xref.as<double>(), dm);
    ws->launches += 1;
    unsigned long long bits = 0;
    PFW_CUDA(cudaMemcpyAsync(&bits, dm, sizeof(bits), cudaMemcpyDeviceToHost, st));
    PFW_CUDA(cudaStreamSynchronize(st));
    double d2;
    std::memcpy(&d2, &bits, sizeof(d2));
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
    const int grid = grid_for((int64_t)n * SKIN_LANES, 256);
    if (m.kind == 0)
      k_pair_list<0><<<grid, 256, 0, st>>>(n, sk.off.as<int64_t>(), sk.j.as<int>(), sk.S.as<int>(), ws->X.as<double>(),
                                           ws->species.as<int>(), dHz, m.cutoff * m.cutoff, prm, F, parts, np);
    else
      k_pair_list<1><<<grid, 256, 0, st>>>(n, sk.off.as<int64_t>(), sk.j.as<int>(), sk.S.as<int>(), ws->X.as<double>(),
                                           ws->species.as<int>(), dHz, m.cutoff * m.cutoff, prm, F, parts, np);
    ws->launches += 1;
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
