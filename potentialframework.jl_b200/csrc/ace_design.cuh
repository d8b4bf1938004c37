// ace_design.cuh — dense energy/force/virial design rows of the ACE model
// (design_matrix_impl, ACE/fitting.jl:18-67) for a batch of systems.
//
// Rows of system s (stacked in system order, row base 10·s + 3·atom_begin_s):
//   0            energy:  Σ_i B_i into the invariant block of z_i, Σ_ij Q_j into
//                its pair block
//   1 + 3k + a   force component a of atom k (original order):
//                Σ_{e ∈ out(k)} ∂B_e − Σ_{e ∈ in(k)} ∂B_e
//   1 + 3n + a + 3b   virial (a, b): −Σ_e d_e[a] ∂B_e[b]
// Columns (row-major, leading dimension ld): WB block of species z at
// z·nB + b, Wpair block at nz·nB + z·nQ + q, i.e. vec(WB), vec(Wpair) in the
// reference's column order, so A·[vec(WB); vec(Wpair)] + baseline = [E; F; W].
//
// One site group (ACE_GROUP threads) per unit — a system and a slice of its
// invariants (small batches split each system's columns over several groups)
// — units taken largest system first by the next free group.  Within a unit
// thread lt owns the invariants b ≡ lt (mod ACE_GROUP) of the slice (column
// z·nB + b for sites of species z; the pair columns go with the first slice):
// every element of a column is updated by one thread only, in site order then
// edge order, as fire-and-forget reductions (the rows arrive zeroed), so the
// rows are deterministic and no update waits for a read.  Per site the group computes the A-basis
// (pass 1 of the site kernel) and each product's factor gradients
// G[k][s] = Π_{other factors} A (a global scratch row per group, read through
// L1); per chunk of edges it tabulates ∂A_a/∂d = ∂R_n/∂r Y_m d̂ + R_n ∇Y_m
// and the pair channels in shared memory; each owner then contracts its
// invariant's coupling entries:
//   ∂B_b/∂d_e = Σ_{(k,c) ∈ row b} c Σ_s G[k][s] ∂A_{f_s}/∂d_e
#pragma once
#include "ace_site.cuh"
#include "pfw_common.cuh"

namespace pfw {

constexpr int ACE_DESIGN_MAX_GROUPS = 4;  // the ∂A tables leave room for at most 4 groups

template <int L>
__global__ void __launch_bounds__(ACE_DESIGN_MAX_GROUPS * ACE_GROUP)
    k_ace_design(AceTables p, AceLayout lay, int nsys, const SysGeom* __restrict__ sysv, int cap,
                 const int* __restrict__ edge_off, const int* __restrict__ edge_j, const double4* __restrict__ edge_d,
                 const double4* __restrict__ pos, const int* __restrict__ perm, double4* __restrict__ gscratch,
                 const int* __restrict__ order, int* __restrict__ next_sys, int nslice, double* __restrict__ Aout,
                 int64_t ld, double* __restrict__ baseline, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  ushort4* st_prods = reinterpret_cast<ushort4*>(smem + lay.prods);
  int2* s_dens = reinterpret_cast<int2*>(smem + lay.density);
  const ushort4* s_prods = (lay.gtab & 2) ? p.prods : st_prods;
  if (!(lay.gtab & 2))
    for (int k = threadIdx.x; k < p.P; k += blockDim.x) st_prods[k] = p.prods[k];
  for (int k = threadIdx.x; k < p.D; k += blockDim.x) s_dens[k] = p.density[k];
  __syncthreads();

  const int g = threadIdx.x / ACE_GROUP, lt = threadIdx.x % ACE_GROUP;
  if (g >= lay.G) return;
  double* gb = reinterpret_cast<double*>(smem + lay.tables_end + lay.group_bytes * g);
  double* A = gb + lay.A;
  const double* Yc = gb + lay.Y;
  const double* dYc = gb + lay.dY;
  const double* Rc = gb + lay.R;
  const double* dRc = gb + lay.dR;
  double* DD = gb + lay.DD;  // [t][a][3]
  double* QD = gb + lay.QD;  // [t][q][2]
  EdgeScalars<double> es;
  const int CH = lay.CH;
  double* e0p = gb + lay.esc;
  es.u = e0p; es.e = e0p + CH; es.de = e0p + 2 * CH; es.du = e0p + 3 * CH; es.dq = e0p + 4 * CH;
  es.r = e0p + 5 * CH; es.dx = e0p + 6 * CH; es.dy = e0p + 7 * CH; es.dz = e0p + 8 * CH;
  es.wred = e0p + 10 * CH;
  es.k0 = reinterpret_cast<int*>(gb + lay.ints);
  es.pidx = es.k0 + CH;
  const int D = p.D, P = p.P, nB = p.nB, nQ = p.nQ, nz = p.nz, RS = lay.RS, YS = lay.YS;
  double4* Gk = gscratch + (size_t)(blockIdx.x * lay.G + g) * P;

  int* wslot = reinterpret_cast<int*>(es.wred);
  for (;;) {
    // systems largest first, each taken by the next free group
    group_sync(g);
    if (lt == 0) wslot[0] = atomicAdd(next_sys, 1);
    group_sync(g);
    const int ui = wslot[0];
    if (ui >= nsys * nslice) break;
    const int s = order[ui / nslice], slice = ui % nslice;
    // this unit's invariants b in [blo, bhi); the pair columns go with slice 0
    const int bw = (nB + nslice - 1) / nslice;
    const int blo = min(nB, slice * bw), bhi = min(nB, blo + bw);
    const bool pairs = slice == 0;
    const SysGeom& sg = sysv[s];
    const int b0 = sg.atom_begin, n = sg.natoms;
    const int64_t row0 = 10 * (int64_t)s + 3 * (int64_t)b0;
    const int64_t vrow = row0 + 1 + 3 * (int64_t)n;
    double base = 0.0;
    for (int i = b0; i < b0 + n; ++i) {
      const int iz = min(max((int)pos[i].w, 0), nz - 1);
      base += p.ref[iz];
      const int eb = min(edge_off[i], cap), E = min(edge_off[i + 1], cap) - eb;
      const int64_t own_row = row0 + 1 + 3 * (int64_t)(perm[i] - b0);
      group_sync(g);
      for (int a = lt; a <= D; a += ACE_GROUP) A[a] = (a == D) ? 1.0 : 0.0;
      // ---- pass 1: A-basis ----
      for (int c0 = 0; c0 < E; c0 += CH) {
        const int nc = min(CH, E - c0);
        group_sync(g);
        double dummy = 0.0;
        ace_chunk_edges<L, double, false>(p, gb, lay, es, edge_d, eb + c0, nc, iz, lt, dummy, status);
        group_sync(g);
        for (int a = lt; a < D; a += ACE_GROUP) {
          const int2 nm = s_dens[a];
          double acc = A[a];
          for (int t = 0; t < nc; ++t) acc += Rc[t * RS + nm.x] * Yc[t * YS + nm.y];
          A[a] = acc;
        }
      }
      group_sync(g);
      // ---- factor gradients of every product; energy row B = C·P ----
      for (int k = lt; k < P; k += ACE_GROUP) {
        const ushort4 f = s_prods[k];
        const double a0 = A[f.x], a1 = A[f.y], a2 = A[f.z], a3 = A[f.w];
        Gk[k] = make_double4(a1 * a2 * a3, a0 * a2 * a3, a0 * a1 * a3, a0 * a1 * a2);
      }
      const int cb0 = iz * nB, cq0 = nz * nB + iz * nQ;
      const int cb_first = cb0 + blo + lt, cb_end = cb0 + bhi;
      const int cq_first = pairs ? cq0 + lt : cq0 + nQ;
      for (int c = cb_first; c < cb_end; c += ACE_GROUP) {
        const int b = c - cb0;
        double acc = 0.0;
        for (int q = p.crow_off[b]; q < p.crow_off[b + 1]; ++q) {
          const ushort4 f = s_prods[p.crow_k[q]];
          acc += p.crow_val[q] * (A[f.x] * A[f.y] * A[f.z] * A[f.w]);
        }
        atomicAdd(Aout + row0 * ld + c, acc);
      }
      double qsum[4] = {0, 0, 0, 0};  // pair columns of this thread (nQ <= 4·ACE_GROUP)
      // ---- pass 2: derivative rows, chunk by chunk ----
      for (int c0 = 0; c0 < E; c0 += CH) {
        const int nc = min(CH, E - c0);
        group_sync(g);  // also orders the G rows before their first read
        double dummy = 0.0;
        ace_chunk_edges<L, double, true>(p, gb, lay, es, edge_d, eb + c0, nc, iz, lt, dummy, status);
        group_sync(g);
        // ∂A_a/∂d of the chunk's edges, zero for the sentinel factor a = D and
        // for the edges that pad the chunk to a multiple of four; the pair
        // channels, one thread per edge
        const int nc4 = (nc + 3) & ~3;
        for (int idx = lt; idx < nc4 * (D + 1); idx += ACE_GROUP) {
          const int t = idx / (D + 1), a = idx - t * (D + 1);
          double* o = DD + (size_t)idx * 3;
          if (t >= nc || a == D) {
            o[0] = o[1] = o[2] = 0.0;
            continue;
          }
          const int2 nm = s_dens[a];
          const double ir = 1.0 / es.r[t];
          const double y = Yc[t * YS + nm.y], rv = Rc[t * RS + nm.x];
          const double rad = dRc[t * RS + nm.x] * y * ir;
          const double* dy = dYc + (t * YS + nm.y) * 3;
          o[0] = rad * es.dx[t] + rv * dy[0];
          o[1] = rad * es.dy[t] + rv * dy[1];
          o[2] = rad * es.dz[t] + rv * dy[2];
        }
        if (lt < nc && nQ > 0) {
          const int t = lt;
          const double4 d4 = edge_d[eb + c0 + t];
          const int zj = min(max((int)d4.w, 0), nz - 1);
          double* o = QD + (size_t)t * nQ * 2;
          if (p.pair_ok[zj]) {
            const int pidx = iz * nz + zj;
            const EdgeRadial<double> eq = edge_radial<double>(p.Q, pidx, es.r[t]);
            for (int qn = 0; qn < nQ; ++qn) {
              double v, dv;
              channel_ed<double>(channel_coeff(p.Q, pidx, eq.k0, qn), eq, v, dv);
              o[2 * qn] = v;
              o[2 * qn + 1] = dv;
            }
          } else {
            for (int qn = 0; qn < 2 * nQ; ++qn) o[qn] = 0.0;
          }
        }
        group_sync(g);
        int dest[ACE_MAX_CHUNK];
#pragma unroll
        for (int t = 0; t < ACE_MAX_CHUNK; ++t)
          dest[t] = t < nc ? (int)(perm[edge_j[eb + c0 + t]] - b0) : 0;
        for (int c = cb_first; c < cb_end; c += ACE_GROUP) {
          const int b = c - cb0;
          const int q0 = p.crow_off[b], q1 = p.crow_off[b + 1];
          double own[3] = {0, 0, 0}, vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
          // four edges at a time: each coupling entry is loaded once for them,
          // and their twelve sums are independent
          for (int t0 = 0; t0 < nc; t0 += 4) {
            const int nt = min(4, nc - t0);
            double gx[4] = {0, 0, 0, 0}, gy[4] = {0, 0, 0, 0}, gz[4] = {0, 0, 0, 0};
            for (int q = q0; q < q1; ++q) {
              const int k = p.crow_k[q];
              const ushort4 f = s_prods[k];
              const double4 G4 = Gk[k];
              const double cv = p.crow_val[q];
              const int fs[4] = {f.x, f.y, f.z, f.w};
              const double gs[4] = {G4.x, G4.y, G4.z, G4.w};
#pragma unroll
              for (int u = 0; u < 4; ++u) {  // sentinel factors read the zero row
                const double w = cv * gs[u];
                const double* da = DD + ((size_t)t0 * (D + 1) + fs[u]) * 3;
#pragma unroll
                for (int tt = 0; tt < 4; ++tt) {
                  const double* dt = da + (size_t)tt * (D + 1) * 3;
                  gx[tt] += w * dt[0];
                  gy[tt] += w * dt[1];
                  gz[tt] += w * dt[2];
                }
              }
            }
#pragma unroll
            for (int tt = 0; tt < 4; ++tt) {
              if (tt >= nt) continue;
              const int t = t0 + tt;
              const double gsum[3] = {gx[tt], gy[tt], gz[tt]};
              const double dv[3] = {es.dx[t], es.dy[t], es.dz[t]};
              const int64_t dest_row = row0 + 1 + 3 * (int64_t)dest[t];
#pragma unroll
              for (int ax = 0; ax < 3; ++ax) {
                atomicAdd(Aout + (dest_row + ax) * ld + c, -gsum[ax]);
                own[ax] += gsum[ax];
              }
#pragma unroll
              for (int bb = 0; bb < 3; ++bb)
#pragma unroll
                for (int aa = 0; aa < 3; ++aa) vir[aa + 3 * bb] -= dv[aa] * gsum[bb];
            }
          }
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) atomicAdd(Aout + (own_row + ax) * ld + c, own[ax]);
#pragma unroll
          for (int k = 0; k < 9; ++k) atomicAdd(Aout + (vrow + k) * ld + c, vir[k]);
        }
        // pair columns: ∂(Σ_j Q_q)/∂d_e = Q_q'(r) d̂
        int slot = 0;
        for (int c = cq_first; c < cq0 + nQ; c += ACE_GROUP, ++slot) {
          const int qn = c - cq0;
          double own[3] = {0, 0, 0}, vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
          for (int t = 0; t < nc; ++t) {
            const double v = QD[((size_t)t * nQ + qn) * 2], dq = QD[((size_t)t * nQ + qn) * 2 + 1];
            qsum[slot] += v;
            const double dv[3] = {es.dx[t], es.dy[t], es.dz[t]};
            const double ir = 1.0 / es.r[t];
            const double gsum[3] = {dq * dv[0] * ir, dq * dv[1] * ir, dq * dv[2] * ir};
            const int64_t dest_row = row0 + 1 + 3 * (int64_t)dest[t];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
              atomicAdd(Aout + (dest_row + ax) * ld + c, -gsum[ax]);
              own[ax] += gsum[ax];
            }
#pragma unroll
            for (int bb = 0; bb < 3; ++bb)
#pragma unroll
              for (int aa = 0; aa < 3; ++aa) vir[aa + 3 * bb] -= dv[aa] * gsum[bb];
          }
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) atomicAdd(Aout + (own_row + ax) * ld + c, own[ax]);
#pragma unroll
          for (int k = 0; k < 9; ++k) atomicAdd(Aout + (vrow + k) * ld + c, vir[k]);
        }
      }
      int slot = 0;
      for (int c = cq_first; c < cq0 + nQ; c += ACE_GROUP, ++slot) atomicAdd(Aout + row0 * ld + c, qsum[slot]);
    }
    if (lt == 0 && baseline && slice == 0) baseline[s] = base;
  }
}

}  // namespace pfw
