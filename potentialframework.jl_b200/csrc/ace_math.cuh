// ace_math.cuh — per-edge ACE mathematics on the device: Agnesi transform,
// envelopes, cubic-spline radial channels with d/dr, and L2 real spherical
// harmonics with Cartesian gradients.
//
// Restates ACE/resolved.jl:156-179 (transformed, envelope),
// ACE/serial.jl:193-250 (envelope_derivative, radial_ed) and
// ACE/angular_blocks.jl:19-81 (BlockAngular recurrences with first-order
// jets) for one edge at a time.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

namespace pfw {

// One radial family on the device (layout of pfw_radial_family).
struct RadialDev {
  int nch, nknots, nz;
  const int* lengths;          // [nz*nz]
  const double* nodes;         // [nz*nz][nknots]
  const double* coeff;         // [nz*nz][nknots-1][nch][4]
  const float* coeff32;        // the same in FP32 for the mixed form (null: read coeff)
  const double* transform;     // [nz*nz][6]
  const int* powers;           // [nz*nz][2]
  const int* env_kind;         // [nz*nz]
  const double* env;           // [nz*nz][5]
};

template <class T>
__device__ __forceinline__ T ipow(T x, int n) {
  if (n == 0) return T(1);
  if (n < 0) {
    x = T(1) / x;
    n = -n;
  }
  T r = T(1);
  while (n) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}

// Per-edge transform, interval and envelope factors shared by every channel
// of a species pair: R_n = e·v_n(u), dR_n/dr = de·v_n(u) + e·v_n'(u)·du.
template <class T>
struct EdgeRadial {
  int k0;    // 0-based spline interval
  T u;       // position inside the interval
  T e, de;   // envelope and d/dr
  T du;      // du/dr = dx/dr / step
  bool ok;   // false: singular envelope at r = 0
};

// Per-pair parameters staged as 16 doubles: transform[6], p, q, envelope
// kind, envelope[5] (RADP_W; see stage_radial_params).
constexpr int RADP_W = 16;

// sp: the staged parameters of the family (shared memory), or null to read
// them from the family's global tables.
template <class T>
__device__ __forceinline__ EdgeRadial<T> edge_radial(const RadialDev& f, int pidx, T r, const double* sp = nullptr) {
  EdgeRadial<T> o;
  o.ok = true;
  const double* t;
  const double* ep;
  int p, q, kind;
  if (sp) {
    t = sp + RADP_W * pidx;
    p = (int)t[6];
    q = (int)t[7];
    kind = (int)t[8];
    ep = t + 9;
  } else {
    t = f.transform + 6 * pidx;
    p = f.powers[2 * pidx];
    q = f.powers[2 * pidx + 1];
    kind = f.env_kind[pidx];
    ep = f.env + 5 * pidx;
  }
  const T a = (T)t[0], rin = (T)t[1], r0 = (T)t[2], yin = (T)t[3], ycut = (T)t[4];
  const T s = (r - rin) / (r0 - rin);
  const int h = q - p;
  T y = r <= rin ? T(1) : T(1) / (T(1) + a * ipow(s, q) / (T(1) + ipow(s, h)));
  T x = T(-1) + T(2) * (y - yin) / (ycut - yin);
  x = x < T(-1) ? T(-1) : (x > T(1) ? T(1) : x);
  T dx;
  if (r <= rin || x <= T(-1) || x >= T(1)) {
    dx = 0;
  } else {
    const T den = T(1) + ipow(s, h);
    const T uu = ipow(s, q) / den;
    const T dd = (T(q) * ipow(s, q - 1) / den - (h == 0 ? T(0) : T(h) * ipow(s, q + h - 1) / (den * den))) / (r0 - rin);
    const T w = T(1) + a * uu;
    dx = T(-2) * a * dd / ((w * w) * (ycut - yin));
  }
  if (kind == 1) {  // PolyEnvelope2sX
    const T x1 = (T)ep[0], x2 = (T)ep[1], sc = (T)ep[4];
    const int p1 = (int)ep[2], p2 = (int)ep[3];
    if (x1 < x && x < x2) {
      o.e = sc * ipow(x - x1, p1) * ipow(x2 - x, p2);
      o.de = sc * (T(p1) * ipow(x - x1, p1 - 1) * ipow(x2 - x, p2) - T(p2) * ipow(x - x1, p1) * ipow(x2 - x, p2 - 1)) * dx;
    } else {
      o.e = 0;
      o.de = 0;
    }
  } else if (kind == 2) {  // ACE1_PolyEnvelope1sR: rcut, r0, p
    const T rc = (T)ep[0], rr0 = (T)ep[1];
    const int pp = (int)ep[2];
    if (r > rc) {
      o.e = 0;
      o.de = 0;
    } else {
      if (!(r > T(0))) o.ok = false;
      const T ss = r / rr0, sc = rc / rr0;
      o.e = ipow(ss, -pp) - ipow(sc, -pp) + T(pp) * ipow(sc, -pp - 1) * (ss - sc);
      o.de = T(pp) / rr0 * (ipow(rc / rr0, -pp - 1) - ipow(r / rr0, -pp - 1));
    }
  } else {  // 3: PolyEnvelope1sR: rcut, p
    const T rc = (T)ep[0];
    const int pp = (int)ep[1];
    if (r >= rc) {
      o.e = 0;
      o.de = 0;
    } else {
      if (!(r > T(0))) o.ok = false;
      const T ss = r / rc;
      o.e = (ipow(ss, -pp) - T(1)) * (T(1) - ss);
      o.de = (T(-pp) * ipow(ss, -pp - 1) * (T(1) - ss) - (ipow(ss, -pp) - T(1))) / rc;
    }
  }
  // searchsortedlast(nodes, x) clamped to [1, K-1] (1-based).  The nodes run
  // from -1 to 1 (checked at load); the interval of a uniform grid is the
  // first guess and the node values themselves settle it, so the count of
  // nodes <= x is exactly the bisection's, in one round of loads instead of
  // log2(K) dependent ones.
  const double* nd = f.nodes + (size_t)f.nknots * pidx;
  const int K = f.lengths[pidx];
  const T gd = (x + T(1)) * (T)(0.5 * (K - 1));
  int gi = gd >= T(0) ? (gd < (T)(K - 1) ? (int)gd : K - 1) : 0;  // NaN → 0
  while (gi + 1 < K && (T)nd[gi + 1] <= x) ++gi;
  while (gi >= 0 && (T)nd[gi] > x) --gi;
  const int lo = gi + 1;  // count of nodes <= x
  int k = lo < 1 ? 1 : (lo > K - 1 ? K - 1 : lo);
  o.k0 = k - 1;
  const T step = (T)nd[k] - (T)nd[k - 1];
  o.u = (x - (T)nd[k - 1]) / step;
  o.du = dx / step;
  return o;
}

// The per-pair parameters of a family in the RADP_W layout (block-strided copy).
__device__ __forceinline__ void stage_radial_params(const RadialDev& f, double* out, int tid, int nthreads) {
  const int np = f.nz * f.nz;
  for (int k = tid; k < np * RADP_W; k += nthreads) {
    const int pidx = k / RADP_W, j = k - pidx * RADP_W;
    double v = 0.0;
    if (j < 6) v = f.transform[6 * pidx + j];
    else if (j < 8) v = (double)f.powers[2 * pidx + (j - 6)];
    else if (j == 8) v = (double)f.env_kind[pidx];
    else if (j < 14) v = f.env[5 * pidx + (j - 9)];
    out[k] = v;
  }
}

// Channel n value and d/dr from the interval coefficients c[0..3].
template <class T>
__device__ __forceinline__ void channel_ed(const double* c, const EdgeRadial<T>& er, T& val, T& der) {
  const T c0 = (T)c[0], c1 = (T)c[1], c2 = (T)c[2], c3 = (T)c[3], u = er.u;
  const T v = ((c3 * u + c2) * u + c1) * u + c0;
  const T dv = (T(3) * c3 * (u * u) + T(2) * c2 * u + c1);
  val = er.e * v;
  der = er.de * v + er.e * dv * er.du;
}

__device__ __forceinline__ const double* channel_coeff(const RadialDev& f, int pidx, int k0, int n) {
  return f.coeff + (((size_t)pidx * (f.nknots - 1) + k0) * f.nch + n) * 4;
}

// First-order jet: value and Cartesian gradient (G = false: value only).
template <class T, bool G>
struct Jet {
  T v, gx, gy, gz;
};
template <class T, bool G>
__device__ __forceinline__ Jet<T, G> jmul(const Jet<T, G>& a, const Jet<T, G>& b) {
  if constexpr (G) return {a.v * b.v, a.gx * b.v + a.v * b.gx, a.gy * b.v + a.v * b.gy, a.gz * b.v + a.v * b.gz};
  else return {a.v * b.v, T(0), T(0), T(0)};
}
template <class T, bool G>
__device__ __forceinline__ Jet<T, G> jadd(const Jet<T, G>& a, const Jet<T, G>& b) {
  if constexpr (G) return {a.v + b.v, a.gx + b.gx, a.gy + b.gy, a.gz + b.gz};
  else return {a.v + b.v, T(0), T(0), T(0)};
}
template <class T, bool G>
__device__ __forceinline__ Jet<T, G> jsub(const Jet<T, G>& a, const Jet<T, G>& b) {
  if constexpr (G) return {a.v - b.v, a.gx - b.gx, a.gy - b.gy, a.gz - b.gz};
  else return {a.v - b.v, T(0), T(0), T(0)};
}
template <class T, bool G>
__device__ __forceinline__ Jet<T, G> jscale(T s, const Jet<T, G>& b) {
  if constexpr (G) return {s * b.v, s * b.gx, s * b.gy, s * b.gz};
  else return {s * b.v, T(0), T(0), T(0)};
}

constexpr int ACE_LMAX = 6;

// The harmonics of one azimuthal order m ≥ 0 (all l in m..L): the same
// recurrences as angular_blocks.jl:49-77 evaluated m-major, so each value is
// computed from the same operands by the same formula:
//   cos/sin(mφ):  c_{k+1} = c_k x - s_k y,  s_{k+1} = s_k x + c_k y  (c_0 → 1/√2 for m = 0)
//   Q_mm = -(2m-1) Q_{m-1,m-1},  Q_{m+1,m} = (2m+1) z Q_mm,
//   Q_lm = ((2l-1) z Q_{l-1,m} - (l+m-1) r² Q_{l-2,m}) / (l-m)
// emit(index, Jet) receives Y_lm at l*l+l+m and, for m > 0, Y_l,-m at l*l+l-m.
// solid: the same recurrences on the raw displacement (unit gradients), which
// gives the real solid harmonics r^l·Y_lm (BlockAngular solid=true,
// angular_blocks.jl:47-48).
template <class T, bool Grad, int L, class Emit>
__device__ __forceinline__ void harmonics_m(const double* __restrict__ F, T r, T dx, T dy, T dz, int m,
                                            Emit&& emit, bool solid = false) {
  using J = Jet<T, Grad>;
  const T ir = T(1) / r;
  J x, y, z;
  if (solid) {
    x = {dx, Grad ? T(1) : T(0), T(0), T(0)};
    y = {dy, T(0), Grad ? T(1) : T(0), T(0)};
    z = {dz, T(0), T(0), Grad ? T(1) : T(0)};
  } else {
    const T ux = dx * ir, uy = dy * ir, uz = dz * ir;
    x = {ux, Grad ? (T(1) - ux * ux) * ir : T(0), Grad ? (-ux * uy) * ir : T(0), Grad ? (-ux * uz) * ir : T(0)};
    y = {uy, Grad ? (-uy * ux) * ir : T(0), Grad ? (T(1) - uy * uy) * ir : T(0), Grad ? (-uy * uz) * ir : T(0)};
    z = {uz, Grad ? (-uz * ux) * ir : T(0), Grad ? (-uz * uy) * ir : T(0), Grad ? (T(1) - uz * uz) * ir : T(0)};
  }
  const J r2 = jadd(jadd(jmul(x, x), jmul(y, y)), jmul(z, z));
  J cs = {T(1), T(0), T(0), T(0)}, sn = {T(0), T(0), T(0), T(0)};
  J q = {T(1), T(0), T(0), T(0)};  // Q_kk along the diagonal
#pragma unroll
  for (int k = 1; k <= L; ++k) {
    if (k > m) break;
    const J c2 = jsub(jmul(cs, x), jmul(sn, y));
    const J s2 = jadd(jmul(sn, x), jmul(cs, y));
    cs = c2;
    sn = s2;
    q = jscale(T(-(2 * k - 1)), q);
  }
  if (m == 0) cs = {T(0.70710678118654752440), T(0), T(0), T(0)};
  J qm2 = q, qm1 = q;
#pragma unroll
  for (int l = 0; l <= L; ++l) {
    if (l < m) continue;
    J ql;
    if (l == m) {
      ql = q;
    } else if (l == m + 1) {
      ql = jscale(T(2 * m + 1), jmul(z, qm1));
    } else {
      const J a = jscale(T(2 * l - 1), jmul(z, qm1));
      const J b = jscale(T(l + m - 1), jmul(r2, qm2));
      ql = jscale(T(1) / T(l - m), jsub(a, b));
    }
    const T Fl = (T)F[l * (L + 1) + m];
    emit(l * l + l + m, jscale(Fl, jmul(ql, cs)));
    if (m > 0) emit(l * l + l - m, jscale(Fl, jmul(ql, sn)));
    qm2 = qm1;
    qm1 = ql;
  }
}

// BlockAngular harmonics of direction d (angular_blocks.jl:36-81).  Calls
// emit(index, Jet) for every component in l*l+l+m order; with Grad=false the
// gradients are not formed.  F: normalisation [(L+1)*(L+1)] as F[l*(L+1)+m].
template <class T, bool Grad, int L, class Emit>
__device__ __forceinline__ void harmonics(const double* __restrict__ F, T r, T dx, T dy, T dz, Emit&& emit) {
  static_assert(L >= 0 && L <= ACE_LMAX, "lmax out of range");
  const T ir = T(1) / r;
  const T ux = dx * ir, uy = dy * ir, uz = dz * ir;
  using J = Jet<T, Grad>;
  J x, y, z;
  x = {ux, Grad ? (T(1) - ux * ux) * ir : T(0), Grad ? (-ux * uy) * ir : T(0), Grad ? (-ux * uz) * ir : T(0)};
  y = {uy, Grad ? (-uy * ux) * ir : T(0), Grad ? (T(1) - uy * uy) * ir : T(0), Grad ? (-uy * uz) * ir : T(0)};
  z = {uz, Grad ? (-uz * ux) * ir : T(0), Grad ? (-uz * uy) * ir : T(0), Grad ? (T(1) - uz * uz) * ir : T(0)};
  const J r2 = jadd(jadd(jmul(x, x), jmul(y, y)), jmul(z, z));
  // cos/sin(mφ) jets
  J cs[ACE_LMAX + 1], sn[ACE_LMAX + 1];
  cs[0] = {T(1), T(0), T(0), T(0)};
  sn[0] = {T(0), T(0), T(0), T(0)};
#pragma unroll
  for (int m = 1; m <= L; ++m) {
    cs[m] = jsub(jmul(cs[m - 1], x), jmul(sn[m - 1], y));
    sn[m] = jadd(jmul(sn[m - 1], x), jmul(cs[m - 1], y));
  }
  const T inv_sqrt2 = T(0.70710678118654752440);
  cs[0] = {inv_sqrt2, T(0), T(0), T(0)};
  // associated-Legendre jets, rolling rows l-2, l-1, l
  J qm2[ACE_LMAX + 1], qm1[ACE_LMAX + 1], ql[ACE_LMAX + 1];
#pragma unroll
  for (int l = 0; l <= L; ++l) {
    if (l == 0) {
      ql[0] = {T(1), T(0), T(0), T(0)};
    } else {
      ql[l] = jscale(T(-(2 * l - 1)), qm1[l - 1]);
      ql[l - 1] = jscale(T(2 * l - 1), jmul(z, qm1[l - 1]));
#pragma unroll
      for (int m = 0; m <= l - 2; ++m) {
        const J a = jscale(T(2 * l - 1), jmul(z, qm1[m]));
        const J b = jscale(T(l + m - 1), jmul(r2, qm2[m]));
        const J c = jsub(a, b);
        const T il = T(1) / T(l - m);
        ql[m] = jscale(il, c);
      }
    }
#pragma unroll
    for (int m = 0; m <= l; ++m) {
      const T Fl = (T)F[l * (L + 1) + m];
      emit(l * l + l + m, jscale(Fl, jmul(ql[m], cs[m])));
      if (m > 0) emit(l * l + l - m, jscale(Fl, jmul(ql[m], sn[m])));
    }
#pragma unroll
    for (int m = 0; m <= l; ++m) {
      qm2[m] = qm1[m];
      qm1[m] = ql[m];
    }
  }
}

}  // namespace pfw
