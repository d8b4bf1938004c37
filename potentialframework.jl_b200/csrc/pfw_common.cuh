// pfw_common.cuh — shared device structures and exact-rounding geometry
// helpers of libpfw_b200.
//
// The neighbour SET must equal the reference's bit for bit, so every
// operation that decides it (wrap, fractional transform, key, displacement,
// r² < c²) is written with explicit round-to-nearest intrinsics
// (__dadd_rn/__dsub_rn/__dmul_rn/__ddiv_rn), which the compiler never fuses
// into FMAs, in the association order of NeighbourList/storage.jl:130-199 and
// geometry.jl:5-19.  Energy/force arithmetic elsewhere is free to contract.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pfw {

// Per-system geometry descriptor (one per system of a batch; one for a
// single evaluate!).  Built on the host by prepare_system() from the cell,
// pbc flags, cutoff and atom count, exactly as prepare! decides them.
struct SysGeom {
  double basis[9];      // column-major; identity on the minimum-image path
  double recip[9];      // inverse of basis
  double Hz[9];         // cell with open generators zeroed (ACE/environments.jl:20-25)
  double L[3];          // diagonal lengths (minimum-image path)
  double sizecell[3];   // bin width per axis (Å or fractional)
  double origin[3];     // bin origin (0 on periodic axes)
  double c, c2;         // cutoff and c*c
  int32_t dims[3];      // dense bins per axis (open axes: max key + 1)
  int32_t pdims[3];     // prepare!'s dims (1 on open axes): the wrap modulus
  int32_t radius[3];    // stencil half-width per axis
  int32_t pbc[3];
  int32_t minimum_image;  // 1: orthorhombic minimum image, 0: explicit images
  int32_t brute;          // all atoms of the system in one cell
  int32_t fast_shift;     // minimum image with every periodic dims >= 4: per-cell wrap
  int32_t atom_begin, natoms;  // original-order atom range of this system
  int32_t cell_begin, ncells;  // global cell range of this system
  int32_t pad;
};

// ---- exact geometry ------------------------------------------------------
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// Julia mod(x, y) for floats: rem then sign fix-up (rem is exact).
__device__ __forceinline__ double jl_mod(double x, double y) {
  double r = fmod(x, y);
  if (r == 0.0) return copysign(r, y);
  if ((r > 0.0) != (y > 0.0)) return xadd(r, y);
  return r;
}

// M·v with ((t1 + t2) + t3), M column-major.
__device__ __forceinline__ void xmatvec(const double* M, double v0, double v1, double v2, double out[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = xadd(xadd(xmul(M[a], v0), xmul(M[a + 3], v1)), xmul(M[a + 6], v2));
}

// r² = (dx² + dy²) + dz²
__device__ __forceinline__ double xr2(double dx, double dy, double dz) {
  return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
}

__device__ __forceinline__ int ifld(int a, int b) {
  int q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
  return q;
}
__device__ __forceinline__ int imod(int a, int b) {
  int r = a % b;
  if (r != 0 && ((r < 0) != (b < 0))) r += b;
  return r;
}

// Decoded stencil entry: neighbour cell (global index) and the displacement
// shift added to x_j - x_i.  For the minimum-image fast path the shift is the
// per-cell wrap -k·L (bit-identical to d - round(d/L)·L for every in-range
// pair when every periodic dims >= 4); for explicit images it is basis·s.
struct StencilEntry {
  int cell;        // global cell index, or -1 when the cell does not exist
  int s[3];        // integer image shift
  double sh[3];    // Cartesian shift
  bool zero;       // s == 0 (self pair must be excluded)
};

// Number of stencil offsets along axis a, and the offset of index t.
__device__ __forceinline__ int stencil_count(const SysGeom& g, int a) {
  if (g.minimum_image) {
    if (g.brute) return 1;
    if (!g.pbc[a]) return 3;
    return g.pdims[a] >= 3 ? 3 : g.pdims[a];  // dims 2: {0, 1}; dims 1: {0}
  }
  return 2 * g.radius[a] + 1;
}
__device__ __forceinline__ int stencil_offset(const SysGeom& g, int a, int t) {
  if (g.minimum_image) {
    if (g.brute) return 0;
    if (g.pbc[a] && g.pdims[a] < 3) return t;  // 0, 1
    return t - 1;
  }
  return t - g.radius[a];
}

// Resolve offset (o0,o1,o2) from the cell with key (k0,k1,k2) of system g.
__device__ __forceinline__ void stencil_entry(const SysGeom& g, const int key[3], const int off[3],
                                              StencilEntry& e) {
  int other[3];
  e.zero = true;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int v = key[a] + off[a];
    if (g.pbc[a]) {
      if (g.brute) {
        other[a] = 0;
        e.s[a] = off[a];
      } else {
        // other = mod(v, dims), s = fld(v, dims) without integer division:
        // |off| <= radius, so a few steps at most
        const int dm = g.pdims[a];
        int s = 0;
        while (v < 0) {
          v += dm;
          --s;
        }
        while (v >= dm) {
          v -= dm;
          ++s;
        }
        other[a] = v;
        e.s[a] = s;
      }
    } else {
      if (g.brute) v = 0;
      if (v < 0 || v >= g.dims[a]) {
        e.cell = -1;
        return;
      }
      other[a] = v;
      e.s[a] = 0;
    }
    if (e.s[a] != 0) e.zero = false;
  }
  e.cell = g.cell_begin + (other[0] * g.dims[1] + other[1]) * g.dims[2] + other[2];
  if (g.minimum_image) {
    // wrap shift -k·L with k = -s (only used when fast_shift is set)
#pragma unroll
    for (int a = 0; a < 3; ++a) e.sh[a] = g.pbc[a] ? xmul((double)e.s[a], g.L[a]) : 0.0;
  } else {
    xmatvec(g.basis, (double)e.s[0], (double)e.s[1], (double)e.s[2], e.sh);
  }
}

// Displacement of j from i for stencil entry e (wrapped sorted coordinates).
// Returns false when the pair is excluded (zero-shift self pair).
__device__ __forceinline__ void displacement(const SysGeom& g, const StencilEntry& e, double xi, double yi,
                                             double zi, double xj, double yj, double zj, double d[3]) {
  double dd[3] = {xsub(xj, xi), xsub(yj, yi), xsub(zj, zi)};
  if (g.minimum_image && !g.fast_shift) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
      d[a] = g.pbc[a] ? xsub(dd[a], xmul(rint(xdiv(dd[a], g.L[a])), g.L[a])) : dd[a];
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) d[a] = xadd(dd[a], e.sh[a]);
  }
}

// Kahan-compensated accumulator (FP64 energy/virial of the mixed form).
struct Kahan {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    double y = x - c;
    double t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

}  // namespace pfw
