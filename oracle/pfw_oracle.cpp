// pfw_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement (C++17, FP64) of PotentialFrameWork.jl's force-evaluation
// hot path, used as the parity oracle for libpfw_b200.so and as the timed
// "restated reference CPU algorithm" baseline.  It is never linked into, or
// called by, the product library.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it.
//
// Each function cites the reference file:line it restates.  Floating-point
// expressions keep the reference's association order and are compiled with
// -ffp-contract=off (the reference's Julia code is compiled without FMA
// contraction), so the geometry (wrap, displacement, cutoff test) is the same
// bit for bit as the reference's for the same inputs.
//
// Parity pins: tests/test_oracle_pins.py checks this file against the
// reference's saved 33-frame TiAl ACE oracle (data/ace_ref), the analytic
// known answers of test/runtests.jl and test/periodic_images.jl, and
// independent O(N²) brute-force image sums.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <numeric>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>
#include <atomic>
#include <functional>
#include <thread>

#include "../include/pfw_b200.h"

namespace pfo {

static thread_local std::string g_error;

// Dynamic parallel loop over [0, count) on nthreads host threads (the
// reference's Threads.@threads :dynamic loops).
static void parallel_for(int nthreads, int64_t count, const std::function<void(int64_t)>& fn) {
  if (nthreads <= 1 || count <= 1) {
    for (int64_t k = 0; k < count; ++k) fn(k);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  int nt = (int)std::min<int64_t>(nthreads, count);
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&] {
      for (int64_t k; (k = next.fetch_add(1)) < count;) fn(k);
    });
  for (auto& th : pool) th.join();
}

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ---------------------------------------------------------------------------
// Julia scalar semantics
// ---------------------------------------------------------------------------

// Julia mod(x, y) for floats: r = rem(x, y); fix sign to that of y.
static inline double jl_mod(double x, double y) {
  double r = std::fmod(x, y);
  if (r == 0.0) return std::copysign(r, y);
  if ((r > 0) != (y > 0)) return r + y;
  return r;
}
static inline int64_t jl_floor_int(double x) { return (int64_t)std::floor(x); }
static inline int64_t jl_fld(int64_t a, int64_t b) {
  int64_t q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) q -= 1;
  return q;
}
static inline int64_t jl_imod(int64_t a, int64_t b) {
  int64_t r = a % b;
  if (r != 0 && ((r < 0) != (b < 0))) r += b;
  return r;
}
// Julia round(x) — round half to even (default RoundNearest).
static inline double jl_round(double x) { return std::nearbyint(x); }

// integer power by repeated squaring (accurate to a few ulp; the reference's
// Float64^Int is compensated, the difference is at the 1e-16 relative level)
static inline double ipow(double x, int n) {
  if (n == 0) return 1.0;
  if (n < 0) { x = 1.0 / x; n = -n; }
  double r = 1.0;
  while (n) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}

// ---------------------------------------------------------------------------
// 3×3 helpers (column-major, columns = cell vectors)
// ---------------------------------------------------------------------------
using M3 = std::array<double, 9>;
static inline double& at(M3& m, int a, int b) { return m[a + 3 * b]; }
static inline double at(const M3& m, int a, int b) { return m[a + 3 * b]; }

// M·v with the sum ((t1 + t2) + t3), no contraction.
static inline void matvec(const M3& m, const double v[3], double out[3]) {
  for (int a = 0; a < 3; ++a) {
    double t = at(m, a, 0) * v[0];
    t = t + at(m, a, 1) * v[1];
    t = t + at(m, a, 2) * v[2];
    out[a] = t;
  }
}

// periodic_basis (NeighbourList/storage.jl:83-108): periodic generators kept,
// open axes completed with Gram-Schmidt of the Cartesian direction of largest
// residual.
static M3 periodic_basis(const M3& H, const bool pb[3]) {
  M3 B{};
  std::vector<std::array<double, 3>> orth;
  auto dot = [](const std::array<double, 3>& q, const std::array<double, 3>& v) {
    double s = q[0] * v[0];
    s = s + q[1] * v[1];
    s = s + q[2] * v[2];
    return s;
  };
  for (int a = 0; a < 3; ++a) {
    if (!pb[a]) continue;
    std::array<double, 3> v{at(H, 0, a), at(H, 1, a), at(H, 2, a)};
    for (double x : v)
      if (!std::isfinite(x)) throw Error(PFW_EINVAL, "periodic cell vectors must be finite");
    for (int c = 0; c < 3; ++c) at(B, c, a) = v[c];
    for (auto& q : orth) {
      double s = dot(q, v);
      for (int c = 0; c < 3; ++c) v[c] = v[c] - s * q[c];
    }
    double nrm = std::sqrt(dot(v, v));
    if (!(std::isfinite(nrm) && nrm > 0))
      throw Error(PFW_EINVAL, "periodic cell vectors must be linearly independent");
    for (int c = 0; c < 3; ++c) v[c] = v[c] / nrm;
    orth.push_back(v);
  }
  for (int a = 0; a < 3; ++a) {
    if (pb[a]) continue;
    std::array<std::array<double, 3>, 3> cand;
    for (int k = 0; k < 3; ++k) {
      std::array<double, 3> v{0, 0, 0};
      v[k] = 1.0;
      for (auto& q : orth) {
        double s = dot(q, v);
        for (int c = 0; c < 3; ++c) v[c] = v[c] - s * q[c];
      }
      cand[k] = v;
    }
    int best = 0;
    double bestn = -1;
    for (int k = 0; k < 3; ++k) {
      double s = dot(cand[k], cand[k]);
      if (s > bestn) { bestn = s; best = k; }  // argmax: first maximum
    }
    auto v = cand[best];
    double nrm = std::sqrt(dot(v, v));
    for (int c = 0; c < 3; ++c) v[c] = v[c] / nrm;
    for (int c = 0; c < 3; ++c) at(B, c, a) = v[c];
    orth.push_back(v);
  }
  return B;
}

// 3×3 inverse by the adjugate / cross-product formula: rows of the inverse are
// (b×c, c×a, a×b) / det, with columns a, b, c.
static M3 inv3(const M3& m) {
  const double* a = &m[0];
  const double* b = &m[3];
  const double* c = &m[6];
  double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
  double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
  double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  double det = a[0] * bc[0];
  det = det + a[1] * bc[1];
  det = det + a[2] * bc[2];
  M3 r{};
  for (int k = 0; k < 3; ++k) {
    at(r, 0, k) = bc[k] / det;
    at(r, 1, k) = ca[k] / det;
    at(r, 2, k) = ab[k] / det;
  }
  return r;
}

// ---------------------------------------------------------------------------
// prepare! (NeighbourList/storage.jl:130-241)
// ---------------------------------------------------------------------------
struct CellImage {
  int64_t cell;        // 0-based cell index in sorted-key order
  double shift[3];     // Cartesian basis·s (image path only)
  bool self;           // owns i==j only for s > 0 lexicographically
  int64_t lattice[3];  // s
};

struct Prepared {
  int64_t n = 0;
  double c = 0;
  bool pbc[3];
  bool minimum_image = true;
  bool brute = false;
  double L[3];
  M3 H, basis, reciprocal;
  std::vector<double> x, y, z;     // sorted, wrapped
  std::vector<int32_t> species;    // sorted
  std::vector<int64_t> p, inverse; // p[k] = original index of sorted atom k
  std::vector<std::array<int64_t, 3>> keys;  // per cell
  std::vector<std::pair<int64_t, int64_t>> ranges;  // [first, last] inclusive, per cell
  std::vector<std::vector<CellImage>> images;
  std::vector<std::vector<int64_t>> footprints;
  std::vector<std::vector<int64_t>> phases;
};

static void minimum_topology(Prepared& w, const int64_t dims[3],
                             std::map<std::array<int64_t, 3>, int64_t>& lookup) {
  // storage.jl:244-261
  for (int64_t i = 0; i < (int64_t)w.keys.size(); ++i) {
    auto& entries = w.images[i];
    if (w.brute) {
      entries.push_back(CellImage{i, {0, 0, 0}, false, {0, 0, 0}});
    } else {
      const auto& key = w.keys[i];
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int64_t off[3] = {dx, dy, dz};
            std::array<int64_t, 3> other;
            for (int a = 0; a < 3; ++a)
              other[a] = w.pbc[a] ? jl_imod(key[a] + off[a], dims[a]) : key[a] + off[a];
            auto it = lookup.find(other);
            if (it == lookup.end()) continue;
            int64_t j = it->second;
            if (j >= i) entries.push_back(CellImage{j, {0, 0, 0}, false, {0, 0, 0}});
          }
    }
    std::stable_sort(entries.begin(), entries.end(),
                     [](const CellImage& a, const CellImage& b) { return a.cell < b.cell; });
    entries.erase(std::unique(entries.begin(), entries.end(),
                              [](const CellImage& a, const CellImage& b) { return a.cell == b.cell; }),
                  entries.end());
  }
}

static void image_topology(Prepared& w, const double reach[3], const double sizecell[3],
                           const int64_t dims[3],
                           std::map<std::array<int64_t, 3>, int64_t>& lookup) {
  // storage.jl:265-283
  int64_t radius[3];
  for (int a = 0; a < 3; ++a)
    radius[a] = w.brute ? (w.pbc[a] ? (int64_t)std::ceil(reach[a]) : 0)
                        : std::max<int64_t>(1, (int64_t)std::ceil(reach[a] / sizecell[a]));
  for (int64_t i = 0; i < (int64_t)w.keys.size(); ++i) {
    auto& entries = w.images[i];
    const auto& key = w.keys[i];
    for (int64_t zz = -radius[2]; zz <= radius[2]; ++zz)
      for (int64_t yy = -radius[1]; yy <= radius[1]; ++yy)
        for (int64_t xx = -radius[0]; xx <= radius[0]; ++xx) {
          int64_t off[3] = {xx, yy, zz};
          int64_t j;
          if (w.brute) {
            j = i;
          } else {
            std::array<int64_t, 3> other;
            for (int a = 0; a < 3; ++a)
              other[a] = w.pbc[a] ? jl_imod(key[a] + off[a], dims[a]) : key[a] + off[a];
            auto it = lookup.find(other);
            if (it == lookup.end()) continue;
            j = it->second;
          }
          if (j < i) continue;
          CellImage e;
          e.cell = j;
          for (int a = 0; a < 3; ++a)
            e.lattice[a] = w.pbc[a] ? (w.brute ? off[a] : jl_fld(key[a] + off[a], dims[a])) : 0;
          double s[3] = {(double)e.lattice[0], (double)e.lattice[1], (double)e.lattice[2]};
          matvec(w.basis, s, e.shift);
          // self = shift > (0,0,0) in Julia's lexicographic tuple order
          const int64_t* l = e.lattice;
          e.self = (l[0] > 0) || (l[0] == 0 && (l[1] > 0 || (l[1] == 0 && l[2] > 0)));
          entries.push_back(e);
        }
  }
}

static void schedule(Prepared& w) {
  // pair_footprint! + schedule! (storage.jl:285-306): greedy colouring of
  // cell-task write footprints; phases run as barrier-separated parallel loops.
  int64_t ncell = (int64_t)w.keys.size();
  w.footprints.assign(ncell, {});
  for (int64_t i = 0; i < ncell; ++i) {
    std::vector<int64_t> fp{i};
    for (auto& e : w.images[i]) fp.push_back(e.cell);
    std::sort(fp.begin(), fp.end());
    fp.erase(std::unique(fp.begin(), fp.end()), fp.end());
    w.footprints[i] = fp;
  }
  std::vector<std::set<int64_t>> incidence(ncell);
  w.phases.clear();
  for (int64_t t = 0; t < ncell; ++t) {
    std::set<int64_t> forbidden;
    for (auto c : w.footprints[t]) forbidden.insert(incidence[c].begin(), incidence[c].end());
    int64_t color = 0;
    while (forbidden.count(color)) ++color;
    if (color >= (int64_t)w.phases.size()) w.phases.emplace_back();
    w.phases[color].push_back(t);
    for (auto c : w.footprints[t]) incidence[c].insert(color);
  }
}

static Prepared prepare(int64_t n, const double* X, const double* Hin, const uint8_t* pbcin,
                        const int32_t* species, double cutoff, int64_t brute_threshold,
                        bool with_schedule) {
  Prepared w;
  w.n = n;
  double c = cutoff;
  if (!(std::isfinite(c) && c > 0)) throw Error(PFW_EINVAL, "cutoff must be finite and positive (Å)");
  w.c = c;
  for (int k = 0; k < 9; ++k) w.H[k] = Hin[k];
  for (int a = 0; a < 3; ++a) w.pbc[a] = pbcin[a] != 0;
  bool axisaligned = true;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      if (a != b && at(w.H, a, b) != 0.0) axisaligned = false;
  for (int a = 0; a < 3; ++a) w.L[a] = at(w.H, a, a);
  bool anyp = w.pbc[0] || w.pbc[1] || w.pbc[2];
  bool mi = true;
  if (anyp) {
    mi = axisaligned;
    for (int a = 0; a < 3; ++a)
      if (w.pbc[a] && !(std::isfinite(w.L[a]) && w.L[a] > 2 * c)) mi = false;
  }
  w.minimum_image = mi;
  if (mi) {
    w.basis = M3{1, 0, 0, 0, 1, 0, 0, 0, 1};
    w.reciprocal = w.basis;
  } else {
    w.basis = periodic_basis(w.H, w.pbc);
    w.reciprocal = inv3(w.basis);
    for (double v : w.reciprocal)
      if (!std::isfinite(v)) throw Error(PFW_EINVAL, "periodic cell vectors must be linearly independent");
  }
  std::vector<double> coords[3], frac[3];
  for (int a = 0; a < 3; ++a) coords[a].resize(n);
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      double v = X[3 * i + a];
      if (!std::isfinite(v)) throw Error(PFW_EINVAL, "positions must be finite");
      coords[a][i] = (mi && w.pbc[a]) ? jl_mod(v, w.L[a]) : v;
    }
  if (!mi) {
    for (int a = 0; a < 3; ++a) frac[a].resize(n);
    for (int64_t i = 0; i < n; ++i) {
      double v[3] = {coords[0][i], coords[1][i], coords[2][i]}, f[3], r[3];
      matvec(w.reciprocal, v, f);
      for (int a = 0; a < 3; ++a) f[a] = w.pbc[a] ? jl_mod(f[a], 1.0) : f[a];
      matvec(w.basis, f, r);
      for (int a = 0; a < 3; ++a) { coords[a][i] = r[a]; frac[a][i] = f[a]; }
    }
  }
  w.brute = n <= brute_threshold;
  std::vector<double>* bin = mi ? coords : frac;
  double reach[3], extent[3], origin[3], sizecell[3];
  int64_t dims[3];
  for (int a = 0; a < 3; ++a) {
    if (mi) {
      reach[a] = c;
    } else {
      double s = at(w.reciprocal, a, 0) * at(w.reciprocal, a, 0);
      s = s + at(w.reciprocal, a, 1) * at(w.reciprocal, a, 1);
      s = s + at(w.reciprocal, a, 2) * at(w.reciprocal, a, 2);
      reach[a] = c * std::sqrt(s);
    }
    extent[a] = mi ? w.L[a] : 1.0;
    if (w.pbc[a] || n == 0) origin[a] = 0.0;
    else origin[a] = *std::min_element(bin[a].begin(), bin[a].end());
    dims[a] = w.pbc[a] ? std::max<int64_t>(1, jl_floor_int(extent[a] / reach[a])) : 1;
    sizecell[a] = w.pbc[a] ? extent[a] / (double)dims[a] : reach[a];
  }
  std::vector<std::array<int64_t, 3>> atomkeys(n);
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      if (w.brute) atomkeys[i][a] = 0;
      else if (w.pbc[a])
        atomkeys[i][a] = std::clamp<int64_t>(jl_floor_int(bin[a][i] / sizecell[a]), 0, dims[a] - 1);
      else
        atomkeys[i][a] = jl_floor_int((bin[a][i] - origin[a]) / sizecell[a]);
    }
  // sortperm! (Perm ordering: ties broken by index) — stable sort by key tuple
  w.p.resize(n);
  std::iota(w.p.begin(), w.p.end(), 0);
  std::stable_sort(w.p.begin(), w.p.end(),
                   [&](int64_t a, int64_t b) { return atomkeys[a] < atomkeys[b]; });
  w.inverse.resize(n);
  w.x.resize(n); w.y.resize(n); w.z.resize(n); w.species.resize(n);
  for (int64_t k = 0; k < n; ++k) {
    int64_t i = w.p[k];
    w.inverse[i] = k;
    w.x[k] = coords[0][i]; w.y[k] = coords[1][i]; w.z[k] = coords[2][i];
    w.species[k] = species ? species[i] : 0;
    const auto& key = atomkeys[i];
    if (w.keys.empty() || key != w.keys.back()) {
      w.keys.push_back(key);
      w.ranges.push_back({k, k});
    } else {
      w.ranges.back().second = k;
    }
  }
  std::map<std::array<int64_t, 3>, int64_t> lookup;
  for (int64_t i = 0; i < (int64_t)w.keys.size(); ++i) lookup[w.keys[i]] = i;
  w.images.assign(w.keys.size(), {});
  if (mi) minimum_topology(w, dims, lookup);
  else image_topology(w, reach, sizecell, dims, lookup);
  if (with_schedule) schedule(w);
  return w;
}

// geometry_lanes (NeighbourList/geometry.jl:5-19) for one lane: displacement
// of sorted atom j from sorted atom i, and whether r² < c².
static inline void lane_geometry(const Prepared& w, int64_t i, int64_t j, const CellImage& img,
                                 double d[3], bool& active) {
  double dd[3] = {w.x[j] - w.x[i], w.y[j] - w.y[i], w.z[j] - w.z[i]};
  if (w.minimum_image) {
    for (int a = 0; a < 3; ++a)
      d[a] = w.pbc[a] ? dd[a] - jl_round(dd[a] / w.L[a]) * w.L[a] : dd[a];
  } else {
    for (int a = 0; a < 3; ++a) d[a] = dd[a] + img.shift[a];
  }
  double r2 = d[0] * d[0];
  r2 = r2 + d[1] * d[1];
  r2 = r2 + d[2] * d[2];
  active = r2 < w.c * w.c;
}

// ---------------------------------------------------------------------------
// Pair models (PairPotentials/models.jl:138-176, lennard_jones.jl:5-33)
// ---------------------------------------------------------------------------
struct PairModel {
  int kind;  // 0 SmoothPair, 1 LJ
  int nz;
  std::vector<double> A;
  double eps, sigma, cutoff;
};

// energy and radial derivative dE/dr at distance r (from d).
static inline void pair_eval(const PairModel& m, int zi, int zj, double r, double& e, double& dedr) {
  if (m.kind == 0) {
    // PreparedSmooth: invc2 = inv(radius^2); q = 1 - r*r*invc2
    double a = m.A[zi * m.nz + zj];
    double invc2 = 1.0 / (m.cutoff * m.cutoff);
    double q = 1.0 - r * r * invc2;
    e = a * q * q * q;
    dedr = -6.0 * a * q * q * invc2 * r;
  } else {
    // LennardJonesRadial
    double ratio = m.sigma / r, ratio2 = ratio * ratio, q = ratio2 * ratio2 * ratio2;
    double rc = m.sigma / m.cutoff, qc2 = rc * rc, qc = qc2 * qc2 * qc2;
    e = 4.0 * m.eps * (q * q - q - qc * qc + qc);
    dedr = 24.0 * m.eps * (q - 2.0 * q * q) / r;
  }
}

// cell_task! (NeighbourList/execution.jl:173-217), lane by lane with width W
// (sum over lanes in lane order).  force is 3×n in sorted order.
static void cell_task(const Prepared& w, const PairModel& m, uint32_t req, int64_t task, int W,
                      std::vector<double>& force, double& e_out, double vir[9], int64_t& npairs) {
  double e = 0;
  double v[9] = {0};
  bool wantE = req & PFW_REQ_ENERGY, wantF = req & PFW_REQ_FORCES, wantV = req & PFW_REQ_VIRIAL;
  auto [first_i, last_i] = w.ranges[task];
  for (int64_t i = first_i; i <= last_i; ++i) {
    double central[3] = {0, 0, 0};
    for (const auto& img : w.images[task]) {
      auto [rf, rl] = w.ranges[img.cell];
      int64_t lo = std::max(rf, i + (img.self ? 0 : 1));
      for (int64_t j = lo; j <= rl; j += W) {
        double esum = 0, fs[3] = {0, 0, 0};
        double vlane[9] = {0};
        for (int k = 0; k < W; ++k) {
          int64_t jj = std::min(j + k, rl);
          bool structural = (j + k <= rl) && (jj > i || (img.self && jj == i));
          double d[3];
          bool active;
          lane_geometry(w, i, jj, img, d, active);
          active = active && structural;
          if (!active) continue;
          ++npairs;
          double r = d[0] * d[0];
          r = r + d[1] * d[1];
          r = r + d[2] * d[2];
          r = std::sqrt(r);
          double en, dedr;
          pair_eval(m, w.species[i], w.species[jj], r, en, dedr);
          esum += en;
          double coef = dedr / (r > 0 ? r : 1.0);
          double g[3] = {coef * d[0], coef * d[1], coef * d[2]};
          for (int a = 0; a < 3; ++a) fs[a] += g[a];
          if (wantF)
            for (int a = 0; a < 3; ++a) force[3 * jj + a] -= g[a];
          for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) vlane[a + 3 * b] += d[a] * g[b];
        }
        if (wantE) e += esum;
        if (wantF)
          for (int a = 0; a < 3; ++a) central[a] += fs[a];
        if (wantV)
          for (int k = 0; k < 9; ++k) v[k] -= vlane[k];
      }
    }
    if (wantF)
      for (int a = 0; a < 3; ++a) force[3 * i + a] += central[a];
  }
  e_out = e;
  for (int k = 0; k < 9; ++k) vir[k] = v[k];
}

// cell_task! again, with the W = 4 lanes as one SIMD vector of doubles (the
// reference's SIMD.jl Vec{4} lanes, geometry.jl:9-27): geometry, cutoff mask,
// safe geometry, pair function and gradient lane-parallel; lane sums and the
// per-lane force scatter in lane order as execution.jl:189-209.  Only the
// timed CPU baseline uses it (the checker runs the scalar cell_task).
typedef double v4d __attribute__((vector_size(32)));

static inline double lane_sum(v4d v) { return ((v[0] + v[1]) + v[2]) + v[3]; }

static void cell_task_simd(const Prepared& w, const PairModel& m, uint32_t req, int64_t task,
                           std::vector<double>& force, double& e_out, double vir[9], int64_t& npairs) {
  constexpr int W = 4;
  double e = 0;
  double v[9] = {0};
  const bool wantE = req & PFW_REQ_ENERGY, wantF = req & PFW_REQ_FORCES, wantV = req & PFW_REQ_VIRIAL;
  const double c2 = w.c * w.c;
  const double invc2 = 1.0 / (m.cutoff * m.cutoff);
  double qc = 0;
  if (m.kind == 1) {
    const double rc = m.sigma / m.cutoff, qc2 = rc * rc;
    qc = qc2 * qc2 * qc2;
  }
  auto [first_i, last_i] = w.ranges[task];
  for (int64_t i = first_i; i <= last_i; ++i) {
    double central[3] = {0, 0, 0};
    const double xi = w.x[i], yi = w.y[i], zi = w.z[i];
    for (const auto& img : w.images[task]) {
      auto [rf, rl] = w.ranges[img.cell];
      const int64_t lo = std::max(rf, i + (img.self ? 0 : 1));
      for (int64_t j = lo; j <= rl; j += W) {
        int64_t js[W];
        v4d dx, dy, dz, structural;
        for (int k = 0; k < W; ++k) {
          js[k] = std::min(j + k, rl);
          structural[k] = ((j + k <= rl) && (js[k] > i || (img.self && js[k] == i))) ? 1.0 : 0.0;
          dx[k] = w.x[js[k]] - xi;
          dy[k] = w.y[js[k]] - yi;
          dz[k] = w.z[js[k]] - zi;
        }
        if (w.minimum_image) {
          v4d* dd[3] = {&dx, &dy, &dz};
          for (int a = 0; a < 3; ++a)
            if (w.pbc[a]) {
              v4d q = *dd[a] / w.L[a];
              for (int k = 0; k < W; ++k) q[k] = __builtin_roundeven(q[k]);
              *dd[a] = *dd[a] - q * w.L[a];
            }
        } else {
          dx = dx + img.shift[0];
          dy = dy + img.shift[1];
          dz = dz + img.shift[2];
        }
        v4d r2 = dx * dx;
        r2 = r2 + dy * dy;
        r2 = r2 + dz * dz;
        const auto act = (r2 < c2) & (structural != 0.0);
        if (!(act[0] | act[1] | act[2] | act[3])) continue;
        // safe geometry before the pair function (geometry.jl:21-27)
        const v4d one = {1.0, 1.0, 1.0, 1.0}, zero = {0.0, 0.0, 0.0, 0.0};
        dx = act ? dx : one;
        dy = act ? dy : zero;
        dz = act ? dz : zero;
        v4d r = dx * dx;
        r = r + dy * dy;
        r = r + dz * dz;
        for (int k = 0; k < W; ++k) r[k] = std::sqrt(r[k]);
        v4d en, dedr;
        if (m.kind == 0) {
          v4d a;
          for (int k = 0; k < W; ++k) a[k] = m.A[w.species[i] * m.nz + w.species[js[k]]];
          const v4d q = 1.0 - r * r * invc2;
          en = a * q * q * q;
          dedr = -6.0 * a * q * q * invc2 * r;
        } else {
          const v4d ratio = m.sigma / r, ratio2 = ratio * ratio, q = ratio2 * ratio2 * ratio2;
          en = 4.0 * m.eps * (q * q - q - qc * qc + qc);
          dedr = 24.0 * m.eps * (q - 2.0 * q * q) / r;
        }
        en = act ? en : zero;
        const v4d coef = dedr / (r > 0.0 ? r : one);
        v4d gx = coef * dx, gy = coef * dy, gz = coef * dz;
        gx = act ? gx : zero;
        gy = act ? gy : zero;
        gz = act ? gz : zero;
        for (int k = 0; k < W; ++k) npairs += act[k] ? 1 : 0;
        if (wantE) e += lane_sum(en);
        if (wantF) {
          central[0] += lane_sum(gx);
          central[1] += lane_sum(gy);
          central[2] += lane_sum(gz);
          for (int k = 0; k < W; ++k) {
            if (!act[k]) continue;
            force[3 * js[k]] -= gx[k];
            force[3 * js[k] + 1] -= gy[k];
            force[3 * js[k] + 2] -= gz[k];
          }
        }
        if (wantV) {
          const v4d* d[3] = {&dx, &dy, &dz};
          const v4d* g[3] = {&gx, &gy, &gz};
          for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) v[a + 3 * b] -= lane_sum((*d[a]) * (*g[b]));
        }
      }
    }
    if (wantF)
      for (int a = 0; a < 3; ++a) force[3 * i + a] += central[a];
  }
  e_out = e;
  for (int k = 0; k < 9; ++k) vir[k] = v[k];
}

// ---------------------------------------------------------------------------
// Neighbour snapshot (NeighbourList/interface.jl:85-143)
// ---------------------------------------------------------------------------
struct Entry {
  int64_t b;
  double R[3];
  int64_t S[3];
};

static std::vector<std::vector<Entry>> materialize(const Prepared& w, const double* X, int W) {
  int64_t n = w.n;
  // image_windings! (interface.jl:100-114)
  std::vector<std::array<int64_t, 3>> wind(n);
  M3 rec = w.reciprocal;
  if (!w.minimum_image) rec = inv3(periodic_basis(w.H, w.pbc));
  for (int64_t i = 0; i < n; ++i) {
    double r[3] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]}, f[3];
    if (!w.minimum_image) matvec(rec, r, f);
    for (int a = 0; a < 3; ++a)
      wind[i][a] = !w.pbc[a] ? 0 : jl_floor_int(w.minimum_image ? r[a] / w.L[a] : f[a]);
  }
  std::vector<std::vector<Entry>> out(n);
  for (int64_t task = 0; task < (int64_t)w.ranges.size(); ++task) {
    auto [fi, li] = w.ranges[task];
    for (int64_t i = fi; i <= li; ++i)
      for (const auto& img : w.images[task]) {
        auto [rf, rl] = w.ranges[img.cell];
        int64_t lo = std::max(rf, i + (img.self ? 0 : 1));
        for (int64_t j = lo; j <= rl; j += W)
          for (int k = 0; k < W; ++k) {
            int64_t jj = std::min(j + k, rl);
            bool structural = (j + k <= rl) && (jj > i || (img.self && jj == i));
            double d[3];
            bool active;
            lane_geometry(w, i, jj, img, d, active);
            if (!(active && structural)) continue;
            int64_t a = w.p[i], bb = w.p[jj];
            int64_t lattice[3];
            if (w.minimum_image) {
              double dd[3] = {w.x[jj] - w.x[i], w.y[jj] - w.y[i], w.z[jj] - w.z[i]};
              for (int ax = 0; ax < 3; ++ax)
                lattice[ax] = w.pbc[ax] ? -(int64_t)jl_round(dd[ax] / w.L[ax]) : 0;
            } else {
              for (int ax = 0; ax < 3; ++ax) lattice[ax] = img.lattice[ax];
            }
            Entry e1, e2;
            e1.b = bb;
            e2.b = a;
            for (int ax = 0; ax < 3; ++ax) {
              int64_t S = lattice[ax] + wind[a][ax] - wind[bb][ax];
              if (S > INT32_MAX || S < -INT32_MAX) throw Error(PFW_EINVAL, "shift overflows Int32");
              e1.S[ax] = S;
              e2.S[ax] = -S;
              e1.R[ax] = d[ax];
              e2.R[ax] = -d[ax];
            }
            out[a].push_back(e1);
            out[bb].push_back(e2);
          }
      }
  }
  return out;
}

// ---------------------------------------------------------------------------
// ACE (ACE/resolved.jl, serial.jl, angular_blocks.jl, projection.jl, cpu.jl)
// ---------------------------------------------------------------------------
struct Family {
  int nch = 0, nknots = 0, nz = 0;
  std::vector<int32_t> lengths;
  std::vector<double> nodes, coeff, transform, envelope;
  std::vector<int32_t> powers, env_kind;
};

struct AceModel {
  int nz, lmax, nY;
  Family R, Q;
  std::vector<std::array<int32_t, 2>> density;
  std::vector<std::vector<int32_t>> products;
  int nbasis;
  std::vector<int32_t> crow, ccol;
  std::vector<double> cval;
  std::vector<double> WB, Wpair, reference;
  std::vector<uint8_t> pair_allowed;
  double cutoff;
  std::vector<double> weights;  // [nz][P] = Cᵀ·WB
  std::vector<double> F;        // BlockAngular normalisation [(lmax+1)^2]
  // trainable radial scales ps.radial.scale / ps.pair.scale, Julia layout
  // (n, iz, jz) column-major; empty = the unit scales (serial.jl:12-17)
  std::vector<double> rscale, qscale;
  bool solid = false;  // real solid harmonics r^l·Y_lm (angular_blocks.jl:47-48)
};

static Family copy_family(const pfw_radial_family& f, int nz) {
  Family o;
  o.nch = f.nchannels;
  o.nknots = f.nknots;
  o.nz = nz;
  int np = nz * nz;
  o.lengths.assign(f.lengths, f.lengths + np);
  o.nodes.assign(f.nodes, f.nodes + (size_t)np * f.nknots);
  o.coeff.assign(f.coeff, f.coeff + (size_t)np * (f.nknots - 1) * f.nchannels * 4);
  o.transform.assign(f.transform, f.transform + np * 6);
  o.powers.assign(f.powers, f.powers + np * 2);
  o.env_kind.assign(f.envelope_kind, f.envelope_kind + np);
  o.envelope.assign(f.envelope, f.envelope + np * 5);
  return o;
}

// transformed (resolved.jl:156-160)
static inline double agnesi(const double* t, int p, int q, double r) {
  double a = t[0], rin = t[1], r0 = t[2], yin = t[3], ycut = t[4];
  double s = (r - rin) / (r0 - rin);
  double y = r <= rin ? 1.0 : 1.0 / (1.0 + a * ipow(s, q) / (1.0 + ipow(s, q - p)));
  double x = -1.0 + 2.0 * (y - yin) / (ycut - yin);
  return std::clamp(x, -1.0, 1.0);
}

// envelope / envelope_derivative (resolved.jl:161-179, serial.jl:193-208)
static inline void envelope_ed(int kind, const double* e, double r, double x, double dx, double& ev,
                               double& de) {
  if (kind == 1) {  // PolyEnvelope2sX
    int p = (int)e[2], q = (int)e[3];
    if (e[0] < x && x < e[1]) {
      ev = e[4] * ipow(x - e[0], p) * ipow(e[1] - x, q);
      de = e[4] * (p * ipow(x - e[0], p - 1) * ipow(e[1] - x, q) -
                   q * ipow(x - e[0], p) * ipow(e[1] - x, q - 1)) * dx;
    } else {
      ev = 0;
      de = 0;
    }
  } else if (kind == 2) {  // ACE1_PolyEnvelope1sR: rcut, r0, p
    double rc = e[0], r0 = e[1];
    int p = (int)e[2];
    if (r > rc) { ev = 0; de = 0; return; }
    if (!(r > 0)) throw Error(PFW_EDOMAIN, "singular imported pair envelope at coincident atoms");
    double s = r / r0, sc = rc / r0;
    ev = ipow(s, -p) - ipow(sc, -p) + p * ipow(sc, -p - 1) * (s - sc);
    de = p / r0 * (ipow(rc / r0, -p - 1) - ipow(r / r0, -p - 1));
  } else if (kind == 3) {  // PolyEnvelope1sR: rcut, p
    double rc = e[0];
    int p = (int)e[1];
    if (r >= rc) { ev = 0; de = 0; return; }
    if (!(r > 0)) throw Error(PFW_EDOMAIN, "singular imported pair envelope at coincident atoms");
    double s = r / rc;
    ev = (ipow(s, -p) - 1.0) * (1.0 - s);
    de = (-p * ipow(s, -p - 1) * (1.0 - s) - (ipow(s, -p) - 1.0)) / rc;
  } else {
    throw Error(PFW_EINVAL, "unsupported radial envelope");
  }
}

// radial_ed (serial.jl:228-250): values and d/dr of all channels of (iz,jz).
static void radial_ed(const Family& f, int pairidx, double r, double* val, double* der) {
  const double* t = &f.transform[pairidx * 6];
  int p = f.powers[pairidx * 2], q = f.powers[pairidx * 2 + 1];
  double a = t[0], rin = t[1], r0 = t[2], yin = t[3], ycut = t[4];
  double x = agnesi(t, p, q, r);
  double s = (r - rin) / (r0 - rin);
  int h = q - p;
  double dx;
  if (r <= rin || x <= -1 || x >= 1) {
    dx = 0;
  } else {
    double den = 1.0 + ipow(s, h);
    double u = ipow(s, q) / den;
    double du = (q * ipow(s, q - 1) / den - (h == 0 ? 0.0 : h * ipow(s, q + h - 1) / (den * den))) / (r0 - rin);
    double w = 1.0 + a * u;
    dx = -2.0 * a * du / ((w * w) * (ycut - yin));
  }
  double ev, de;
  envelope_ed(f.env_kind[pairidx], &f.envelope[pairidx * 5], r, x, dx, ev, de);
  const double* nodes = &f.nodes[(size_t)pairidx * f.nknots];
  int K = f.lengths[pairidx];
  // searchsortedlast: last index with nodes[k] <= x (1-based), clamped to [1, K-1]
  int k = (int)(std::upper_bound(nodes, nodes + K, x) - nodes);  // count of nodes <= x
  k = std::clamp(k, 1, K - 1);
  int k0 = k - 1;  // 0-based interval
  double step = nodes[k0 + 1] - nodes[k0];
  double u = (x - nodes[k0]) / step;
  const double* c = &f.coeff[((size_t)pairidx * (f.nknots - 1) + k0) * f.nch * 4];
  for (int n = 0; n < f.nch; ++n) {
    const double* cn = c + 4 * n;
    double v = ((cn[3] * u + cn[2]) * u + cn[1]) * u + cn[0];
    double dv = (3.0 * cn[3] * (u * u) + 2.0 * cn[2] * u + cn[1]) / step;
    val[n] = ev * v;
    der[n] = de * v + ev * dv * dx;
  }
}

// BlockAngular (angular_blocks.jl:19-81) for one direction, with first-order
// Cartesian jets.  Y[nY], dY[nY][3].
struct Jet {
  double v, g[3];
};
static inline Jet jmul(const Jet& a, const Jet& b) {
  return Jet{a.v * b.v, {a.g[0] * b.v + a.v * b.g[0], a.g[1] * b.v + a.v * b.g[1], a.g[2] * b.v + a.v * b.g[2]}};
}
static inline Jet jadd(const Jet& a, const Jet& b) { return Jet{a.v + b.v, {a.g[0] + b.g[0], a.g[1] + b.g[1], a.g[2] + b.g[2]}}; }
static inline Jet jsub(const Jet& a, const Jet& b) { return Jet{a.v - b.v, {a.g[0] - b.g[0], a.g[1] - b.g[1], a.g[2] - b.g[2]}}; }
static inline Jet jscale(double s, const Jet& b) { return Jet{s * b.v, {s * b.g[0], s * b.g[1], s * b.g[2]}}; }
static inline Jet jdiv(const Jet& a, double s) { return Jet{a.v / s, {a.g[0] / s, a.g[1] / s, a.g[2] / s}}; }

static std::vector<double> angular_normalisation(int L) {
  // BlockAngular(lmax) (angular_blocks.jl:25-34): F[l,0] = sqrt((2l+1)/(2π)),
  // F[l,m] = -F[l,m-1]/sqrt((l+m)(l+1-m)).
  std::vector<double> F((L + 1) * (L + 1), 0.0);
  const double twopi = 6.283185307179586;
  for (int l = 0; l <= L; ++l) {
    F[l * (L + 1) + 0] = std::sqrt((double)(2 * l + 1) / twopi);
    for (int m = 1; m <= l; ++m)
      F[l * (L + 1) + m] = -F[l * (L + 1) + m - 1] / std::sqrt((double)((l + m) * (l + 1 - m)));
  }
  return F;
}

// solid: the recurrences on the raw displacement with unit gradients, i.e. the
// real solid harmonics r^l·Y_lm (BlockAngular solid=true, angular_blocks.jl:47-48).
static void angular_ed(int L, const std::vector<double>& F, const double d[3], double* Y, double* dY,
                       bool solid = false) {
  double radius = d[0] * d[0];
  radius = radius + d[1] * d[1];
  radius = radius + d[2] * d[2];
  radius = std::sqrt(radius);
  if (!(radius > 0)) throw Error(PFW_EDOMAIN, "physical zero directions are unsupported");
  double u[3] = {d[0] / radius, d[1] / radius, d[2] / radius};
  if (solid)
    for (int a = 0; a < 3; ++a) u[a] = d[a];
  Jet jx[3];
  for (int a = 0; a < 3; ++a) {
    jx[a].v = u[a];
    for (int c = 0; c < 3; ++c)
      jx[a].g[c] = solid ? (a == c ? 1.0 : 0.0) : ((a == c ? 1.0 : 0.0) - u[a] * u[c]) / radius;
  }
  Jet x = jx[0], y = jx[1], z = jx[2];
  Jet r2 = jadd(jadd(jmul(x, x), jmul(y, y)), jmul(z, z));
  const Jet one{1.0, {0, 0, 0}}, zero{0.0, {0, 0, 0}};
  std::vector<Jet> cs(L + 1, zero), sn(L + 1, zero), Q((L + 1) * (L + 1), zero);
  auto q = [&](int l, int m) -> Jet& { return Q[l * (L + 1) + m]; };
  cs[0] = one;
  sn[0] = zero;
  q(0, 0) = one;
  for (int m = 1; m <= L; ++m) {
    cs[m] = jsub(jmul(cs[m - 1], x), jmul(sn[m - 1], y));
    sn[m] = jadd(jmul(sn[m - 1], x), jmul(cs[m - 1], y));
  }
  cs[0] = jdiv(one, std::sqrt(2.0));
  for (int l = 0; l <= L; ++l) {
    if (l > 0) {
      q(l, l) = jscale((double)(-(2 * l - 1)), q(l - 1, l - 1));
      q(l, l - 1) = jscale((double)(2 * l - 1), jmul(z, q(l - 1, l - 1)));
      for (int m = 0; m <= l - 2; ++m)
        q(l, m) = jdiv(jsub(jscale((double)(2 * l - 1), jmul(z, q(l - 1, m))),
                            jscale((double)(l + m - 1), jmul(r2, q(l - 2, m)))),
                       (double)(l - m));
    }
    for (int m = 0; m <= l; ++m) {
      double Fl = F[l * (L + 1) + m];
      Jet pos = jscale(Fl, jmul(q(l, m), cs[m]));
      Jet neg = jscale(Fl, jmul(q(l, m), sn[m]));
      int ip = l * l + l + m, im = l * l + l - m;
      Y[ip] = pos.v;
      for (int c = 0; c < 3; ++c) dY[3 * ip + c] = pos.g[c];
      if (m > 0) {
        Y[im] = neg.v;
        for (int c = 0; c < 3; ++c) dY[3 * im + c] = neg.g[c];
      }
    }
  }
}

static AceModel make_model(const pfw_ace_tables* t) {
  AceModel m;
  m.nz = t->nz;
  m.lmax = t->lmax;
  m.solid = t->angular_kind == 1;
  m.nY = (t->lmax + 1) * (t->lmax + 1);
  m.R = copy_family(t->radial, t->nz);
  m.Q = copy_family(t->pair, t->nz);
  m.density.resize(t->ndensity);
  for (int a = 0; a < t->ndensity; ++a) m.density[a] = {t->density[2 * a], t->density[2 * a + 1]};
  m.products.resize(t->nproducts);
  for (int k = 0; k < t->nproducts; ++k)
    m.products[k].assign(t->product_factors + t->product_offsets[k], t->product_factors + t->product_offsets[k + 1]);
  m.nbasis = t->nbasis;
  m.crow.assign(t->coupling_rows, t->coupling_rows + t->ncoupling);
  m.ccol.assign(t->coupling_cols, t->coupling_cols + t->ncoupling);
  m.cval.assign(t->coupling_vals, t->coupling_vals + t->ncoupling);
  m.WB.assign(t->WB, t->WB + (size_t)t->nz * t->nbasis);
  m.Wpair.assign(t->Wpair, t->Wpair + (size_t)t->nz * t->pair.nchannels);
  m.reference.assign(t->reference, t->reference + t->nz);
  m.pair_allowed.assign(t->pair_allowed, t->pair_allowed + t->nz);
  m.cutoff = t->cutoff;
  // weights = Cᵀ·(mask∘WB)  (cpu.jl:265-268): per stored entry in CSC order
  int P = t->nproducts;
  m.weights.assign((size_t)t->nz * P, 0.0);
  for (int z = 0; z < t->nz; ++z)
    for (int e = 0; e < t->ncoupling; ++e)
      m.weights[(size_t)z * P + m.ccol[e]] += m.cval[e] * m.WB[(size_t)z * t->nbasis + m.crow[e]];
  m.F = angular_normalisation(t->lmax);
  return m;
}

struct SiteEdge {
  int64_t j;     // original index
  double d[3];   // X_j - X_i + H·S
};

struct SiteResult {
  double energy;
  std::vector<std::array<double, 3>> g;  // per edge
  std::vector<double> B;                 // masked basis values (nbasis)
  std::vector<double> Qsum;              // Σ_j Q[j,:] (nQ)
};

// NI.evaluate_site!(::PreparedACE) (ACE/cpu.jl:162-237), scalar radial path,
// unrestricted products (projection.jl:130-147).  Edges are already bucketed
// by neighbour species (environments.jl:42-76).
static SiteResult evaluate_site(const AceModel& m, int iz, const std::vector<SiteEdge>& edges,
                                const std::vector<int32_t>& zs, bool want_grad, bool want_features) {
  int E = (int)edges.size(), nR = m.R.nch, nQ = m.Q.nch, nY = m.nY, D = (int)m.density.size();
  int P = (int)m.products.size();
  std::vector<double> R((size_t)E * nR), dR((size_t)E * nR), Qv((size_t)E * nQ), dQ((size_t)E * nQ);
  std::vector<double> Y((size_t)E * nY), dY((size_t)E * nY * 3), rs(E);
  for (int j = 0; j < E; ++j) {
    const double* d = edges[j].d;
    double r = d[0] * d[0];
    r = r + d[1] * d[1];
    r = r + d[2] * d[2];
    r = std::sqrt(r);
    if (r == 0) throw Error(PFW_EDOMAIN, "coincident atoms");
    rs[j] = r;
    int pidx = iz * m.nz + zs[j];
    radial_ed(m.R, pidx, r, &R[(size_t)j * nR], &dR[(size_t)j * nR]);
    radial_ed(m.Q, pidx, r, &Qv[(size_t)j * nQ], &dQ[(size_t)j * nQ]);
    // radial_scale (serial.jl:17; gpu.jl:74-91,229-238): scale · R applied at run time
    if (!m.rscale.empty())
      for (int n = 0; n < nR; ++n) {
        const double sc = m.rscale[n + (size_t)nR * (iz + (size_t)m.nz * zs[j])];
        R[(size_t)j * nR + n] *= sc;
        dR[(size_t)j * nR + n] *= sc;
      }
    if (!m.qscale.empty())
      for (int n = 0; n < nQ; ++n) {
        const double sc = m.qscale[n + (size_t)nQ * (iz + (size_t)m.nz * zs[j])];
        Qv[(size_t)j * nQ + n] *= sc;
        dQ[(size_t)j * nQ + n] *= sc;
      }
    if (!m.pair_allowed[zs[j]])
      for (int n = 0; n < nQ; ++n) Qv[(size_t)j * nQ + n] = dQ[(size_t)j * nQ + n] = 0;
    angular_ed(m.lmax, m.F, d, &Y[(size_t)j * nY], &dY[(size_t)j * nY * 3], m.solid);
  }
  // project_rows! (cpu.jl:156-161): for (a,(r,m)), j
  std::vector<double> A(D, 0.0);
  for (int a = 0; a < D; ++a) {
    int rn = m.density[a][0], ym = m.density[a][1];
    double s = 0;
    for (int j = 0; j < E; ++j) s += R[(size_t)j * nR + rn] * Y[(size_t)j * nY + ym];
    A[a] = s;
  }
  // unrestricted_products! with U = A, V = 0
  const double* w = &m.weights[(size_t)iz * P];
  std::vector<double> Pv(P), dA(D, 0.0), prefix(16);
  for (int k = 0; k < P; ++k) {
    const auto& idx = m.products[k];
    int nu = (int)idx.size();
    if ((int)prefix.size() < nu + 1) prefix.resize(nu + 1);
    prefix[0] = 1.0;
    for (int t = 0; t < nu; ++t) prefix[t + 1] = prefix[t] * (A[idx[t]] + 0.0);
    Pv[k] = prefix[nu];
    double adj = w[k];
    for (int t = nu - 1; t >= 0; --t) {
      int a = idx[t];
      double g = adj * prefix[t];
      dA[a] += g;
      adj *= A[a] + 0.0;
    }
  }
  double energy = m.reference[iz];
  for (int k = 0; k < P; ++k) energy += w[k] * Pv[k];
  const double* wp = &m.Wpair[(size_t)iz * nQ];
  for (int j = 0; j < E; ++j)
    for (int n = 0; n < nQ; ++n) energy += Qv[(size_t)j * nQ + n] * wp[n];
  SiteResult out;
  out.energy = energy;
  if (want_features) {
    // fitting.jl:28-29: B = (C·P) .* mask; Σ_j Q[j,:]
    out.B.assign(m.nbasis, 0.0);
    for (size_t e = 0; e < m.cval.size(); ++e) out.B[m.crow[e]] += m.cval[e] * Pv[m.ccol[e]];
    out.Qsum.assign(nQ, 0.0);
    for (int j = 0; j < E; ++j)
      for (int n = 0; n < nQ; ++n) out.Qsum[n] += Qv[(size_t)j * nQ + n];
  }
  if (want_grad) {
    out.g.resize(E);
    for (int j = 0; j < E; ++j) {
      double r = rs[j];
      double dir[3] = {edges[j].d[0] / r, edges[j].d[1] / r, edges[j].d[2] / r};
      double g[3] = {0, 0, 0};
      for (int a = 0; a < D; ++a) {
        int rn = m.density[a][0], ym = m.density[a][1];
        double t1 = dR[(size_t)j * nR + rn] * Y[(size_t)j * nY + ym];
        double Rv = R[(size_t)j * nR + rn];
        for (int c = 0; c < 3; ++c) g[c] = g[c] + dA[a] * (t1 * dir[c] + Rv * dY[((size_t)j * nY + ym) * 3 + c]);
      }
      for (int n = 0; n < nQ; ++n) {
        double s = wp[n] * dQ[(size_t)j * nQ + n];
        for (int c = 0; c < 3; ++c) g[c] = g[c] + s * dir[c];
      }
      out.g[j] = {g[0], g[1], g[2]};
    }
  }
  return out;
}

}  // namespace pfo

using namespace pfo;

// ---------------------------------------------------------------------------
// extern "C" surface (ctypes)
// ---------------------------------------------------------------------------
extern "C" {

const char* pfo_last_error(void) { return g_error.c_str(); }

#define PFO_TRY try {
#define PFO_CATCH                               \
  }                                             \
  catch (const Error& e) {                      \
    g_error = e.what();                         \
    return e.code;                              \
  }                                             \
  catch (const std::exception& e) {             \
    g_error = e.what();                         \
    return PFW_EINVAL;                          \
  }

// evaluate!(Workspace(width, bruteforce_threshold), sys, p; request, parallel)
// (PairPotentials/evaluation.jl:31-52).  kind 0: SmoothPair with params = A
// (nz×nz, row-major = symmetric), kind 1: LJ with params = {eps, sigma}.
// nthreads > 1 runs the phase-coloured parallel executor (execution.jl:223-238).
int pfo_pair_evaluate(int64_t n, const double* X, const double* H, const uint8_t* pbc,
                      const int32_t* species, int32_t kind, int32_t nz, const double* params,
                      double cutoff, int32_t width, int32_t brute_threshold, uint32_t request,
                      int32_t nthreads, double* E, double* F, double* W, int64_t* npairs) {
  PFO_TRY
  PairModel m;
  m.kind = kind;
  m.nz = nz;
  m.cutoff = cutoff;
  if (kind == 0) m.A.assign(params, params + (size_t)nz * nz);
  else { m.eps = params[0]; m.sigma = params[1]; }
  Prepared w = prepare(n, X, H, pbc, species, cutoff, brute_threshold, true);
  int64_t ncell = (int64_t)w.keys.size();
  std::vector<double> force(3 * n, 0.0), energies(ncell, 0.0), virials(9 * ncell, 0.0);
  std::vector<int64_t> counts(ncell, 0);
  // width -4: the W = 4 lanes as SIMD vectors (cell_task_simd), else scalar lanes
  const bool simd = width == -4;
  int Wd = width > 0 ? width : 4;
  auto task = [&](int64_t t) {
    if (simd) cell_task_simd(w, m, request, t, force, energies[t], &virials[9 * t], counts[t]);
    else cell_task(w, m, request, t, Wd, force, energies[t], &virials[9 * t], counts[t]);
  };
  if (nthreads <= 1) {
    for (int64_t t = 0; t < ncell; ++t) task(t);
  } else {
    for (auto& phase : w.phases) parallel_for(nthreads, (int64_t)phase.size(), [&](int64_t k) { task(phase[k]); });
  }
  // outputs (evaluation.jl:8-25)
  if (E) {
    double s = 0;
    for (double e : energies) s += e;
    *E = s;
  }
  if (W) {
    for (int k = 0; k < 9; ++k) {
      double s = 0;
      for (int64_t t = 0; t < ncell; ++t) s += virials[9 * t + k];
      W[k] = s;
    }
  }
  if (F)
    for (int64_t k = 0; k < n; ++k)
      for (int a = 0; a < 3; ++a) F[3 * w.p[k] + a] = force[3 * k + a];
  if (npairs) {
    int64_t s = 0;
    for (auto c : counts) s += c;
    *npairs = s;
  }
  return 0;
  PFO_CATCH
}

// neighbour_list(X, cutoff, cell, pbc) + neighbours(list, i) (interface.jl:47-151).
// Call with capacity < total to query total; entries are grouped by original
// centre, in the reference's emission order.
int pfo_neighbour_list(int64_t n, const double* X, const double* H, const uint8_t* pbc,
                       double cutoff, int32_t brute_threshold, int64_t capacity, int64_t* offsets,
                       int32_t* jout, int32_t* Sout, double* Rout, int64_t* total) {
  PFO_TRY
  Prepared w = prepare(n, X, H, pbc, nullptr, cutoff, brute_threshold, false);
  auto lists = materialize(w, X, 4);
  int64_t tot = 0;
  for (auto& l : lists) tot += (int64_t)l.size();
  *total = tot;
  if (capacity < tot) return 0;
  int64_t o = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (offsets) offsets[i] = o;
    for (auto& e : lists[i]) {
      if (jout) jout[o] = (int32_t)e.b;
      for (int a = 0; a < 3; ++a) {
        if (Sout) Sout[3 * o + a] = (int32_t)e.S[a];
        if (Rout) Rout[3 * o + a] = e.R[a];
      }
      ++o;
    }
  }
  if (offsets) offsets[n] = o;
  return 0;
  PFO_CATCH
}

void* pfo_ace_model_create(const pfw_ace_tables* t) {
  try {
    return new AceModel(make_model(t));
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}
void pfo_ace_model_destroy(void* m) { delete (AceModel*)m; }

// AC.energy_forces_virial(sys, ACECalculator) (ACE/calculators.jl:48-96):
// full environments from the snapshot (NeighbourList/environments.jl:33-76),
// edge displacements X_j - X_i + H·S with open generators zeroed
// (ACE/environments.jl:20-25, NeighbourList/environments.jl:97-102), site
// evaluation and reduce_site! (execution.jl:256-273).  site_energy [n] and
// features [n][nz*(nB+nQ)] (per-site fitting energy row, fitting.jl:28-29)
// are optional.  nthreads > 1: sites in parallel with a deterministic reduction.
int pfo_ace_evaluate(void* model, int64_t n, const double* X, const double* H, const uint8_t* pbc,
                     const int32_t* species, int32_t brute_threshold, uint32_t request, int32_t nthreads,
                     double* E, double* F, double* W, double* site_energy, double* features) {
  PFO_TRY
  const AceModel& m = *(const AceModel*)model;
  Prepared w = prepare(n, X, H, pbc, nullptr, m.cutoff, brute_threshold, false);
  auto lists = materialize(w, X, 4);
  double Hz[9];
  for (int b = 0; b < 3; ++b)
    for (int a = 0; a < 3; ++a) Hz[a + 3 * b] = pbc[b] ? H[a + 3 * b] : 0.0;
  std::vector<double> es(n, 0.0);
  std::vector<std::vector<SiteEdge>> site_edges(n);
  std::vector<std::vector<int32_t>> site_z(n);
  for (int64_t i = 0; i < n; ++i) {
    // pack_environment!: bucket by neighbour species, traversal order kept
    for (int z = 0; z < m.nz; ++z)
      for (auto& e : lists[i]) {
        if (species[e.b] != z) continue;
        SiteEdge se;
        se.j = e.b;
        for (int a = 0; a < 3; ++a) {
          double s = Hz[a] * (double)e.S[0];
          s = s + Hz[a + 3] * (double)e.S[1];
          s = s + Hz[a + 6] * (double)e.S[2];
          se.d[a] = X[3 * e.b + a] - X[3 * i + a] + s;
        }
        site_edges[i].push_back(se);
        site_z[i].push_back(z);
      }
  }
  bool want_grad = request & (PFW_REQ_FORCES | PFW_REQ_VIRIAL);
  int nfeat = m.nz * (m.nbasis + m.Q.nch);
  std::vector<SiteResult> res(n);
  std::vector<int> codes(n, 0);
  std::vector<std::string> msgs(n);
  parallel_for(nthreads, n, [&](int64_t i) {
    try {
      res[i] = evaluate_site(m, species[i], site_edges[i], site_z[i], want_grad, features != nullptr);
    } catch (const Error& e) {
      codes[i] = e.code;
      msgs[i] = e.what();
    }
  });
  for (int64_t i = 0; i < n; ++i)
    if (codes[i]) throw Error(codes[i], msgs[i]);
  double etot = 0, vir[9] = {0};
  std::vector<double> force(3 * n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    es[i] = res[i].energy;
    etot += res[i].energy;
    if (want_grad)
      for (size_t k = 0; k < site_edges[i].size(); ++k) {
        const auto& g = res[i].g[k];
        int64_t j = site_edges[i][k].j;
        for (int a = 0; a < 3; ++a) {
          force[3 * i + a] += g[a];
          force[3 * j + a] -= g[a];
        }
        for (int b = 0; b < 3; ++b)
          for (int a = 0; a < 3; ++a) vir[a + 3 * b] -= site_edges[i][k].d[a] * g[b];
      }
    if (features) {
      double* f = features + (size_t)i * nfeat;
      std::fill(f, f + nfeat, 0.0);
      int iz = species[i];
      for (int b = 0; b < m.nbasis; ++b) f[(size_t)iz * m.nbasis + b] = res[i].B[b];
      for (int q = 0; q < m.Q.nch; ++q) f[(size_t)m.nz * m.nbasis + (size_t)iz * m.Q.nch + q] = res[i].Qsum[q];
    }
  }
  if (E) *E = etot;
  if (F) std::copy(force.begin(), force.end(), F);
  if (W) std::copy(vir, vir + 9, W);
  if (site_energy) std::copy(es.begin(), es.end(), site_energy);
  return 0;
  PFO_CATCH
}

// Trainable radial scales of trainable_parameters (serial.jl:12-16): radial
// [nR][nz][nz] and pair [nQ][nz][nz] in Julia column-major (n, iz, jz) order;
// a null pointer restores the unit scales.
int pfo_ace_set_scales(void* model, const double* radial_scale, const double* pair_scale) {
  PFO_TRY
  AceModel& m = *(AceModel*)model;
  const size_t zz = (size_t)m.nz * m.nz;
  if (radial_scale) m.rscale.assign(radial_scale, radial_scale + zz * m.R.nch);
  else m.rscale.clear();
  if (pair_scale) m.qscale.assign(pair_scale, pair_scale + zz * m.Q.nch);
  else m.qscale.clear();
  return 0;
  PFO_CATCH
}

// Independent pieces exposed for unit tests.
int pfo_radial_ed(void* model, int32_t family, int32_t iz, int32_t jz, double r, double* val, double* der) {
  PFO_TRY
  const AceModel& m = *(const AceModel*)model;
  radial_ed(family == 0 ? m.R : m.Q, iz * m.nz + jz, r, val, der);
  return 0;
  PFO_CATCH
}
int pfo_angular_ed(int32_t lmax, const double* d, double* Y, double* dY) {
  PFO_TRY
  auto F = angular_normalisation(lmax);
  angular_ed(lmax, F, d, Y, dY);
  return 0;
  PFO_CATCH
}
int pfo_solid_ed(int32_t lmax, const double* d, double* Y, double* dY) {
  PFO_TRY
  auto F = angular_normalisation(lmax);
  angular_ed(lmax, F, d, Y, dY, true);
  return 0;
  PFO_CATCH
}

}  // extern "C"
