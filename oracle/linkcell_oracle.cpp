// linkcell oracle: TEST INFRASTRUCTURE, not product code.
//
// CPU restatement of the reference periodic linked-cell k-nearest walk,
// HaoZeke/linkcell v0.3.3. Every function cites the reference lines it
// follows. Compile with -ffp-contract=off: the Rust source never fuses a
// multiply into an add, and every sum below is written left to right in
// the same association as the Rust expression it restates.
//
// Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg, as the checker.

#include "linkcell_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace {

// ---------------------------------------------------------------- errors
// src/error.rs:7-36. The strings are part of the C ABI contract.
enum class Err { None, ZeroK, BadBox, Empty, BufferSize, Overflow, MaskLen, TooManyCells };

const char *err_text(Err e) {
  switch (e) {
    case Err::ZeroK: return "k must be at least 1";
    case Err::BadBox: return "singular or non-positive cell";
    case Err::Empty: return "no points";
    case Err::BufferSize: return "out buffer length must be n * k";
    case Err::Overflow: return "n * k overflows";
    case Err::MaskLen: return "mask length must be n";
    case Err::TooManyCells: return "linked-cell mesh is too fine";
    case Err::None: break;
  }
  return "";
}

thread_local std::string g_last_error;
thread_local bool g_has_error = false;

int fail(Err e) {
  g_last_error = err_text(e);
  g_has_error = true;
  return 1;
}
int fail_msg(const char *m) {
  g_last_error = m;
  g_has_error = true;
  return 1;
}
void clear_error() {
  g_last_error.clear();
  g_has_error = false;
}

// ---------------------------------------------------------------- cell
// src/cell.rs:35-46. h[col][row]: h[0] is lattice vector a.
struct Cell {
  double h[3][3];
  double hinv[3][3];
  double origin[3];
  double widths[3];
  bool ortho;
};

using V3 = double[3];

// src/cell.rs:333-341: H is stored by columns, mul(h, v) = H v.
inline void mul(const double m[3][3], const double v[3], double out[3]) {
  out[0] = m[0][0] * v[0] + m[1][0] * v[1] + m[2][0] * v[2];
  out[1] = m[0][1] * v[0] + m[1][1] * v[1] + m[2][1] * v[2];
  out[2] = m[0][2] * v[0] + m[1][2] * v[1] + m[2][2] * v[2];
}

// src/cell.rs:343-349
inline void cross(const double u[3], const double v[3], double out[3]) {
  out[0] = u[1] * v[2] - u[2] * v[1];
  out[1] = u[2] * v[0] - u[0] * v[2];
  out[2] = u[0] * v[1] - u[1] * v[0];
}

// src/cell.rs:351-353
inline double norm(const double v[3]) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// Rust f64::min / f64::max ignore a NaN operand; std::fmin / std::fmax do too.
inline double rmin(double a, double b) { return std::fmin(a, b); }
inline double rmax(double a, double b) { return std::fmax(a, b); }

// src/cell.rs:355-388. Returns false where the reference returns None.
bool invert_columns(const double h[3][3], double inv[3][3], double *det_out) {
  const double *a = h[0];
  const double *b = h[1];
  const double *c = h[2];
  const double det = a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
                     a[2] * (b[0] * c[1] - b[1] * c[0]);
  if (!std::isfinite(det) || std::fabs(det) < 1e-18) return false;
  const double invdet = 1.0 / det;
  inv[0][0] = (b[1] * c[2] - b[2] * c[1]) * invdet;
  inv[0][1] = (a[2] * c[1] - a[1] * c[2]) * invdet;
  inv[0][2] = (a[1] * b[2] - a[2] * b[1]) * invdet;
  inv[1][0] = (b[2] * c[0] - b[0] * c[2]) * invdet;
  inv[1][1] = (a[0] * c[2] - a[2] * c[0]) * invdet;
  inv[1][2] = (a[2] * b[0] - a[0] * b[2]) * invdet;
  inv[2][0] = (b[0] * c[1] - b[1] * c[0]) * invdet;
  inv[2][1] = (a[1] * c[0] - a[0] * c[1]) * invdet;
  inv[2][2] = (a[0] * b[1] - a[1] * b[0]) * invdet;
  *det_out = det;
  return true;
}

// src/cell.rs:322-331
bool is_axis_aligned(const double h[3][3]) {
  const double scale = rmax(norm(h[0]) + norm(h[1]) + norm(h[2]), 1.0);
  const double tol = 1e-12 * scale;
  return std::fabs(h[0][1]) <= tol && std::fabs(h[0][2]) <= tol && std::fabs(h[1][0]) <= tol &&
         std::fabs(h[1][2]) <= tol && std::fabs(h[2][0]) <= tol && std::fabs(h[2][1]) <= tol;
}

// src/cell.rs:97-124 (Cell::from_vectors).
bool make_cell(const orc_cell &c, Cell &out) {
  std::memset(&out, 0, sizeof(out));
  const double a[3] = {c.ax, c.ay, c.az};
  const double b[3] = {c.bx, c.by, c.bz};
  const double cc[3] = {c.cx, c.cy, c.cz};
  for (int r = 0; r < 3; ++r) {
    out.h[0][r] = a[r];
    out.h[1][r] = b[r];
    out.h[2][r] = cc[r];
  }
  double det = 0.0;
  if (!invert_columns(out.h, out.hinv, &det)) return false;
  if (!std::isfinite(det) || std::fabs(det) < 1e-18) return false;
  double bc[3], ca[3], ab[3];
  cross(b, cc, bc);
  cross(cc, a, ca);
  cross(a, b, ab);
  const double wa = std::fabs(det) / norm(bc);
  const double wb = std::fabs(det) / norm(ca);
  const double wc = std::fabs(det) / norm(ab);
  if (!(wa > 0.0 && wb > 0.0 && wc > 0.0)) return false;
  out.origin[0] = c.ox;
  out.origin[1] = c.oy;
  out.origin[2] = c.oz;
  out.widths[0] = wa;
  out.widths[1] = wb;
  out.widths[2] = wc;
  out.ortho = is_axis_aligned(out.h);
  return true;
}

// src/cell.rs:290-298
inline double wrap01(double s) {
  s -= std::floor(s);
  return s >= 1.0 ? 0.0 : s;
}

// src/cell.rs:175-194
inline void fractional(const Cell &c, const double r[3], double s[3]) {
  if (c.ortho) {
    s[0] = wrap01((r[0] - c.origin[0]) / c.widths[0]);
    s[1] = wrap01((r[1] - c.origin[1]) / c.widths[1]);
    s[2] = wrap01((r[2] - c.origin[2]) / c.widths[2]);
    return;
  }
  const double d[3] = {r[0] - c.origin[0], r[1] - c.origin[1], r[2] - c.origin[2]};
  mul(c.hinv, d, s);
  for (int e = 0; e < 3; ++e) s[e] = wrap01(s[e]);
}

// src/cell.rs:199-207
inline void cartesian(const Cell &c, const double s[3], double out[3]) {
  double r[3];
  mul(c.h, s, r);
  out[0] = r[0] + c.origin[0];
  out[1] = r[1] + c.origin[1];
  out[2] = r[2] + c.origin[2];
}

// src/cell.rs:226-247
inline void lattice_shift(const Cell &c, int na, int nb, int nc, double out[3]) {
  if (c.ortho) {
    out[0] = double(na) * c.widths[0];
    out[1] = double(nb) * c.widths[1];
    out[2] = double(nc) * c.widths[2];
    return;
  }
  const double *a = c.h[0];
  const double *b = c.h[1];
  const double *cc = c.h[2];
  const double fa = double(na), fb = double(nb), fc = double(nc);
  out[0] = fa * a[0] + fb * b[0] + fc * cc[0];
  out[1] = fa * a[1] + fb * b[1] + fc * cc[1];
  out[2] = fa * a[2] + fb * b[2] + fc * cc[2];
}

// src/cell.rs:268-274: dx = q + shift - p, in that association.
inline double dist2_shifted(const double p[3], const double q[3], const double s[3]) {
  const double dx = q[0] + s[0] - p[0];
  const double dy = q[1] + s[1] - p[1];
  const double dz = q[2] + s[2] - p[2];
  return dx * dx + dy * dy + dz * dz;
}

// src/cell.rs:300-309
inline double dist2_ortho(const double l[3], const double p[3], const double q[3]) {
  double r2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    double d = std::fabs(q[k] - p[k]);
    d -= l[k] * std::round(d / l[k]);
    r2 += d * d;
  }
  return r2;
}

// src/cell.rs:311-320
inline double dist2_general(const Cell &c, const double p[3], const double q[3]) {
  const double dp[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
  double ds[3];
  mul(c.hinv, dp, ds);
  for (int e = 0; e < 3; ++e) ds[e] -= std::round(ds[e]);
  double dr[3];
  mul(c.h, ds, dr);
  return dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
}

// src/cell.rs:281-287
inline double cell_dist2(const Cell &c, const double p[3], const double q[3]) {
  if (c.ortho) return dist2_ortho(c.widths, p, q);
  return dist2_general(c, p, q);
}

// src/knearest.rs:24-40
inline double pair_dist2(const Cell &c, const double p[3], const double q[3]) {
  if (c.ortho) return cell_dist2(c, p, q);
  double best = std::numeric_limits<double>::infinity();
  for (int na = -1; na <= 1; ++na)
    for (int nb = -1; nb <= 1; ++nb)
      for (int nc = -1; nc <= 1; ++nc) {
        double s[3];
        lattice_shift(c, na, nb, nc, s);
        const double d2 = dist2_shifted(p, q, s);
        if (d2 < best) best = d2;
      }
  return best;
}

// f64::total_cmp (IEEE 754 totalOrder) as a signed integer key.
inline int64_t total_key(double v) {
  int64_t b;
  std::memcpy(&b, &v, 8);
  b ^= int64_t(uint64_t(b >> 63) >> 1);
  return b;
}
inline bool pair_less(const std::pair<double, size_t> &x, const std::pair<double, size_t> &y) {
  const int64_t kx = total_key(x.first), ky = total_key(y.first);
  if (kx != ky) return kx < ky;
  return x.second < y.second;
}

// ---------------------------------------------------------------- KHeap
// src/knearest.rs:50-159. The k <= 16 inline array versus the Vec spill
// is only storage; one vector restates both.
struct KHeap {
  std::vector<double> d2;
  std::vector<size_t> idx;
  size_t n = 0, k = 0;
  explicit KHeap(size_t kk) : d2(kk, 0.0), idx(kk, 0), k(kk) {}
  void reset() { n = 0; }
  // src/knearest.rs:106-129
  void push(double d, size_t j) {
    for (size_t t = 0; t < n; ++t) {
      if (idx[t] == j) {
        if (d < d2[t]) {
          d2[t] = d;
          idx[t] = j;
        }
        return;
      }
    }
    if (n < k) {
      d2[n] = d;
      idx[n] = j;
      ++n;
      return;
    }
    size_t worst = 0;
    for (size_t t = 1; t < n; ++t)
      if (d2[t] > d2[worst]) worst = t;
    if (d < d2[worst]) {
      d2[worst] = d;
      idx[worst] = j;
    }
  }
  bool full() const { return n >= k; }
  // src/knearest.rs:135-144
  double worst() const {
    double w = d2[0];
    for (size_t t = 1; t < n; ++t)
      if (d2[t] > w) w = d2[t];
    return w;
  }
  // src/knearest.rs:146-158
  void finish(std::vector<std::pair<double, size_t>> &pairs) const {
    pairs.clear();
    for (size_t t = 0; t < n; ++t) pairs.emplace_back(d2[t], idx[t]);
    std::sort(pairs.begin(), pairs.end(), pair_less);
  }
};

// ---------------------------------------------------------------- search
constexpr int64_t kMaxCells = 16777216;  // src/knearest.rs:20

// src/knearest.rs:42-48
bool bins_1d(double width, double edge, int *out) {
  const double n = rmax(std::floor(width / edge), 1.0);
  if (!std::isfinite(n) || n > 1000000.0) return false;
  *out = int(n);
  return true;
}

inline int rem_euclid(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}
inline int div_euclid(int a, int n) {
  const int q = a / n;
  return (a % n < 0) ? q - 1 : q;
}

struct Grid {
  int nx, ny, nz;
  double cell_min;
  int max_reach;
  size_t ncell;
};

// src/knearest.rs:377-397,430
Err plan_grid(const Cell &c, bool has_hint, double hint, Grid &g) {
  double edge = has_hint ? hint : 3.0;
  if (!std::isfinite(edge) || edge <= 0.0) edge = 3.0;
  edge = rmin(rmin(rmin(edge, c.widths[0]), c.widths[1]), c.widths[2]);
  if (!bins_1d(c.widths[0], edge, &g.nx)) return Err::TooManyCells;
  if (!bins_1d(c.widths[1], edge, &g.ny)) return Err::TooManyCells;
  if (!bins_1d(c.widths[2], edge, &g.nz)) return Err::TooManyCells;
  const int64_t v = int64_t(g.nx) * int64_t(g.ny) * int64_t(g.nz);
  if (!(v > 0 && v <= kMaxCells)) return Err::TooManyCells;
  g.ncell = size_t(v);
  g.cell_min = rmin(rmin(c.widths[0] / double(g.nx), c.widths[1] / double(g.ny)),
                    c.widths[2] / double(g.nz));
  g.max_reach = std::max(g.nx, std::max(g.ny, g.nz)) / 2 + 1;
  return Err::None;
}

// The binned state search() builds before its walk (src/knearest.rs:399-428).
struct Binned {
  const Cell *cell;
  Grid g;
  size_t n;
  std::vector<size_t> active;
  std::vector<double> folded;  // n*3
  std::vector<int> bx, by, bz;
  std::vector<int64_t> head, next;
  size_t k;

  size_t cell_index(int ix, int iy, int iz) const {
    const int cx = rem_euclid(ix, g.nx), cy = rem_euclid(iy, g.ny), cz = rem_euclid(iz, g.nz);
    return size_t((int64_t(cz) * g.ny + cy) * g.nx + cx);
  }
};

// src/knearest.rs:403-428
void build_bins(const double *xyz, size_t n, const std::vector<size_t> &active, Binned &b) {
  const Cell &c = *b.cell;
  b.n = n;
  b.folded.assign(n * 3, 0.0);
  b.bx.assign(n, 0);
  b.by.assign(n, 0);
  b.bz.assign(n, 0);
  const double invx = double(b.g.nx), invy = double(b.g.ny), invz = double(b.g.nz);
  for (size_t i : active) {
    double s[3];
    fractional(c, xyz + 3 * i, s);
    cartesian(c, s, &b.folded[3 * i]);
    // Rust `as i32` saturates and maps NaN to 0; clamp follows.
    auto to_i32 = [](double v) -> int {
      if (std::isnan(v)) return 0;
      if (v >= 2147483647.0) return 2147483647;
      if (v <= -2147483648.0) return -2147483647 - 1;
      return int(v);
    };
    b.bx[i] = std::clamp(to_i32(s[0] * invx), 0, b.g.nx - 1);
    b.by[i] = std::clamp(to_i32(s[1] * invy), 0, b.g.ny - 1);
    b.bz[i] = std::clamp(to_i32(s[2] * invz), 0, b.g.nz - 1);
  }
  b.head.assign(b.g.ncell, -1);
  b.next.assign(n, -1);
  for (size_t i : active) {
    const size_t ci = b.cell_index(b.bx[i], b.by[i], b.bz[i]);
    b.next[i] = b.head[ci];
    b.head[ci] = int64_t(i);
  }
}

// The per-source closure of search() (src/knearest.rs:431-475).
// Returns the reach at which the walk stopped; visits counts heap pushes.
int walk_one(const Binned &b, size_t i, KHeap &heap, long long *visits) {
  const Cell &c = *b.cell;
  heap.reset();
  const int ix = b.bx[i], iy = b.by[i], iz = b.bz[i];
  const double *p = &b.folded[3 * i];
  long long pushes = 0;
  int reach = 1;
  int stopped = 0;
  while (reach <= b.g.max_reach) {
    for (int dx = -reach; dx <= reach; ++dx)
      for (int dy = -reach; dy <= reach; ++dy)
        for (int dz = -reach; dz <= reach; ++dz) {
          const bool shell = reach == 1 || std::abs(dx) == reach || std::abs(dy) == reach ||
                             std::abs(dz) == reach;
          if (!shell && reach > 1) continue;
          const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
          const size_t ci = b.cell_index(jx, jy, jz);
          double sh[3];
          lattice_shift(c, div_euclid(jx, b.g.nx), div_euclid(jy, b.g.ny), div_euclid(jz, b.g.nz),
                        sh);
          int64_t j = b.head[ci];
          while (j >= 0) {
            const size_t ju = size_t(j);
            if (ju != i) {
              heap.push(dist2_shifted(p, &b.folded[3 * ju], sh), ju);
              ++pushes;
            }
            j = b.next[ju];
          }
        }
    stopped = reach;
    if (heap.full()) {
      const double bound = double(reach) * b.g.cell_min;
      if (heap.worst() <= bound * bound) break;
    }
    reach += 1;
  }
  if (visits) *visits = pushes;
  return stopped;
}

// Runs fn(i) over the given sources on `threads` threads (dynamic chunks).
template <class F>
void parallel_for(const std::vector<size_t> &items, int threads, F &&fn) {
  if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
  if (threads == 1 || items.size() < 64) {
    for (size_t t = 0; t < items.size(); ++t) fn(t, 0);
    return;
  }
  std::atomic<size_t> cursor{0};
  const size_t chunk = 64;
  std::vector<std::thread> pool;
  for (int w = 0; w < threads; ++w) {
    pool.emplace_back([&, w]() {
      for (;;) {
        const size_t lo = cursor.fetch_add(chunk);
        if (lo >= items.size()) break;
        const size_t hi = std::min(items.size(), lo + chunk);
        for (size_t t = lo; t < hi; ++t) fn(t, w);
      }
    });
  }
  for (auto &th : pool) th.join();
}

int resolve_threads(int threads) {
  if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
  return threads;
}

// write_one + search (src/knearest.rs:275-307,351-486) for one frame.
// `mask` is the already-converted boolean mask or null.
Err search_write(const double *xyz, size_t n, const Cell &c, size_t k, const uint8_t *mask,
                 bool has_hint, double hint, int *out_nn, double *out_d2, int threads,
                 int *stop_reach, long long *visits) {
  for (size_t t = 0; t < n * k; ++t) out_nn[t] = -1;
  if (out_d2)
    for (size_t t = 0; t < n * k; ++t) out_d2[t] = std::numeric_limits<double>::quiet_NaN();
  if (k == 0) return Err::ZeroK;
  if (n == 0) return Err::Empty;
  std::vector<size_t> active;
  active.reserve(n);
  for (size_t i = 0; i < n; ++i)
    if (!mask || mask[i]) active.push_back(i);
  if (active.empty()) return Err::None;
  Binned b;
  b.cell = &c;
  b.k = k;
  const Err ge = plan_grid(c, has_hint, hint, b.g);
  if (ge != Err::None) return ge;
  build_bins(xyz, n, active, b);
  const int nth = resolve_threads(threads);
  std::vector<KHeap> heaps(static_cast<size_t>(nth), KHeap(k));
  std::vector<std::vector<std::pair<double, size_t>>> rows(static_cast<size_t>(nth));
  parallel_for(active, nth, [&](size_t t, int w) {
    const size_t i = active[t];
    KHeap &heap = heaps[size_t(w)];
    long long v = 0;
    const int r = walk_one(b, i, heap, &v);
    if (stop_reach) stop_reach[i] = r;
    if (visits) visits[i] = v;
    auto &pairs = rows[size_t(w)];
    heap.finish(pairs);
    for (size_t s = 0; s < pairs.size(); ++s) {
      out_nn[i * k + s] = int(pairs[s].second);
      if (out_d2) out_d2[i * k + s] = pairs[s].first;
    }
  });
  return Err::None;
}

std::vector<uint8_t> to_bool_mask(const int *mask, size_t n) {
  std::vector<uint8_t> m;
  if (!mask) return m;
  m.resize(n);
  for (size_t i = 0; i < n; ++i) m[i] = mask[i] != 0;
  return m;
}

// The brute-force checkers: knearest_brute (src/knearest.rs:508-541) and
// oracle_knearest (tests/agree.rs:186-210). `mic27` selects the latter.
int brute_common(const double *xyz, size_t n, const orc_cell *cell, size_t k, const int *mask,
                 int *out_nn, double *out_d2, bool mic27) {
  if (k == 0) return fail(Err::ZeroK);
  if (n == 0) return fail(Err::Empty);
  if (!xyz || !cell || !out_nn) return fail_msg("null pointer");
  Cell c;
  if (!make_cell(*cell, c)) return fail(Err::BadBox);
  for (size_t t = 0; t < n * k; ++t) out_nn[t] = -1;
  if (out_d2)
    for (size_t t = 0; t < n * k; ++t) out_d2[t] = std::numeric_limits<double>::quiet_NaN();
  std::vector<size_t> active;
  for (size_t i = 0; i < n; ++i)
    if (!mask || mask[i] != 0) active.push_back(i);
  std::vector<std::pair<double, size_t>> pairs;
  for (size_t i : active) {
    pairs.clear();
    for (size_t j : active) {
      if (j == i) continue;
      double d;
      if (mic27) {
        // tests/agree.rs:161-184: q + fa a + fb b + fc c - p, left to right.
        double best = std::numeric_limits<double>::infinity();
        const double *p = xyz + 3 * i, *q = xyz + 3 * j;
        for (int na = -1; na <= 1; ++na)
          for (int nb = -1; nb <= 1; ++nb)
            for (int nc = -1; nc <= 1; ++nc) {
              const double fa = na, fb = nb, fc = nc;
              const double dx = q[0] + fa * c.h[0][0] + fb * c.h[1][0] + fc * c.h[2][0] - p[0];
              const double dy = q[1] + fa * c.h[0][1] + fb * c.h[1][1] + fc * c.h[2][1] - p[1];
              const double dz = q[2] + fa * c.h[0][2] + fb * c.h[1][2] + fc * c.h[2][2] - p[2];
              const double r2 = dx * dx + dy * dy + dz * dz;
              if (r2 < best) best = r2;
            }
        d = best;
      } else {
        d = pair_dist2(c, xyz + 3 * i, xyz + 3 * j);
      }
      pairs.emplace_back(d, j);
    }
    std::sort(pairs.begin(), pairs.end(), pair_less);
    if (pairs.size() > k) pairs.resize(k);
    for (size_t s = 0; s < pairs.size(); ++s) {
      out_nn[i * k + s] = int(pairs[s].second);
      if (out_d2) out_d2[i * k + s] = pairs[s].first;
    }
  }
  clear_error();
  return 0;
}

}  // namespace

extern "C" {

const char *orc_last_error(void) { return g_has_error ? g_last_error.c_str() : nullptr; }

const char *orc_version(void) { return "0.3.3"; }

// src/capi.rs:184-259
int orc_knearest_many(const double *xyz, size_t n, size_t n_frames, const orc_cell *cell, size_t k,
                      const int *mask, double cell_hint, int *out_nn, double *out_d2, int threads) {
  if (n == 0 || n_frames == 0) return fail(Err::Empty);
  if (k == 0) return fail(Err::ZeroK);
  if (!xyz || !cell || !out_nn) return fail_msg("null pointer");
  // checked_mul on usize, then the isize::MAX bounds (src/capi.rs:204-214).
  const size_t smax = std::numeric_limits<size_t>::max();
  if (n > smax / n_frames) return fail(Err::Overflow);
  const size_t n_pts = n * n_frames;
  if (n_pts > smax / k) return fail(Err::Overflow);
  const size_t need = n_pts * k;
  const size_t imax = size_t(std::numeric_limits<int64_t>::max());
  if (n_pts > imax / 3 || need > imax / sizeof(int)) return fail(Err::Overflow);
  Cell c;
  if (!make_cell(*cell, c)) return fail(Err::BadBox);
  const std::vector<uint8_t> m = to_bool_mask(mask, n);
  const bool has_hint = cell_hint > 0.0;  // src/capi.rs:235-239
  for (size_t f = 0; f < n_frames; ++f) {
    const Err e = search_write(xyz + 3 * n * f, n, c, k, mask ? m.data() : nullptr, has_hint,
                               cell_hint, out_nn + n * k * f, out_d2 ? out_d2 + n * k * f : nullptr,
                               threads, nullptr, nullptr);
    if (e != Err::None) return fail(e);
  }
  clear_error();
  return 0;
}

int orc_knearest_brute(const double *xyz, size_t n, const orc_cell *cell, size_t k, const int *mask,
                       int *out_nn, double *out_d2) {
  return brute_common(xyz, n, cell, k, mask, out_nn, out_d2, false);
}

int orc_knearest_mic27(const double *xyz, size_t n, const orc_cell *cell, size_t k, const int *mask,
                       int *out_nn, double *out_d2) {
  return brute_common(xyz, n, cell, k, mask, out_nn, out_d2, true);
}

int orc_cell_info(const orc_cell *cell, double cell_hint, double *info, double *h, double *hinv,
                  int *grid) {
  Cell c;
  if (!cell || !make_cell(*cell, c)) {
    fail(Err::BadBox);
    return 1;
  }
  info[0] = c.widths[0];
  info[1] = c.widths[1];
  info[2] = c.widths[2];
  info[4] = c.ortho ? 1.0 : 0.0;
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row) {
      h[col * 3 + row] = c.h[col][row];
      hinv[col * 3 + row] = c.hinv[col][row];
    }
  Grid g;
  const Err e = plan_grid(c, cell_hint > 0.0, cell_hint, g);
  if (e != Err::None) {
    fail(e);
    return 2;
  }
  info[3] = g.cell_min;
  grid[0] = g.nx;
  grid[1] = g.ny;
  grid[2] = g.nz;
  grid[3] = g.max_reach;
  clear_error();
  return 0;
}

int orc_fold_bin(const double *xyz, size_t n, const orc_cell *cell, const int *mask,
                 double cell_hint, double *folded, int *cell_id) {
  Cell c;
  if (!cell || !make_cell(*cell, c)) return fail(Err::BadBox);
  Binned b;
  b.cell = &c;
  const Err ge = plan_grid(c, cell_hint > 0.0, cell_hint, b.g);
  if (ge != Err::None) return fail(ge);
  std::vector<size_t> active;
  for (size_t i = 0; i < n; ++i)
    if (!mask || mask[i] != 0) active.push_back(i);
  build_bins(xyz, n, active, b);
  for (size_t i = 0; i < n; ++i) {
    const bool on = !mask || mask[i] != 0;
    folded[3 * i + 0] = b.folded[3 * i + 0];
    folded[3 * i + 1] = b.folded[3 * i + 1];
    folded[3 * i + 2] = b.folded[3 * i + 2];
    cell_id[i] = on ? int(b.cell_index(b.bx[i], b.by[i], b.bz[i])) : -1;
  }
  clear_error();
  return 0;
}

int orc_walk_stats(const double *xyz, size_t n, const orc_cell *cell, size_t k, const int *mask,
                   double cell_hint, int *stop_reach, long long *visits, int threads) {
  if (n == 0) return fail(Err::Empty);
  if (k == 0) return fail(Err::ZeroK);
  Cell c;
  if (!cell || !make_cell(*cell, c)) return fail(Err::BadBox);
  for (size_t i = 0; i < n; ++i) {
    stop_reach[i] = 0;
    visits[i] = 0;
  }
  std::vector<int> nn(n * k);
  const std::vector<uint8_t> m = to_bool_mask(mask, n);
  const Err e = search_write(xyz, n, c, k, mask ? m.data() : nullptr, cell_hint > 0.0, cell_hint,
                             nn.data(), nullptr, threads, stop_reach, visits);
  if (e != Err::None) return fail(e);
  clear_error();
  return 0;
}

int orc_knearest_subset(const double *xyz, size_t n, const orc_cell *cell, size_t k,
                        const int *mask, double cell_hint, const long long *sources,
                        size_t count, int *out_nn, double *out_d2, int threads,
                        long long *visits) {
  if (n == 0) return fail(Err::Empty);
  if (k == 0) return fail(Err::ZeroK);
  Cell c;
  if (!cell || !make_cell(*cell, c)) return fail(Err::BadBox);
  for (size_t t = 0; t < count * k; ++t) out_nn[t] = -1;
  if (out_d2)
    for (size_t t = 0; t < count * k; ++t) out_d2[t] = std::numeric_limits<double>::quiet_NaN();
  if (visits)
    for (size_t t = 0; t < count; ++t) visits[t] = 0;
  std::vector<size_t> active;
  for (size_t i = 0; i < n; ++i)
    if (!mask || mask[i] != 0) active.push_back(i);
  if (active.empty()) {
    clear_error();
    return 0;
  }
  Binned b;
  b.cell = &c;
  b.k = k;
  const Err ge = plan_grid(c, cell_hint > 0.0, cell_hint, b.g);
  if (ge != Err::None) return fail(ge);
  build_bins(xyz, n, active, b);
  std::vector<size_t> items(count);
  for (size_t t = 0; t < count; ++t) items[t] = t;
  const int nth = resolve_threads(threads);
  std::vector<KHeap> heaps(static_cast<size_t>(nth), KHeap(k));
  std::vector<std::vector<std::pair<double, size_t>>> rows(static_cast<size_t>(nth));
  parallel_for(items, nth, [&](size_t t, int w) {
    const long long src = sources[t];
    if (src < 0 || size_t(src) >= n) return;
    const size_t i = size_t(src);
    if (mask && mask[i] == 0) return;
    KHeap &heap = heaps[size_t(w)];
    walk_one(b, i, heap, visits ? &visits[t] : nullptr);
    heap.finish(rows[size_t(w)]);
    auto &pairs = rows[size_t(w)];
    for (size_t s = 0; s < pairs.size(); ++s) {
      out_nn[t * k + s] = int(pairs[s].second);
      if (out_d2) out_d2[t * k + s] = pairs[s].first;
    }
  });
  clear_error();
  return 0;
}

int orc_time_sample(const double *xyz, size_t n, const orc_cell *cell, size_t k, const int *mask,
                    double cell_hint, size_t first, size_t stride, size_t count, int threads,
                    double *prep_seconds, double *walk_seconds, long long *walked,
                    long long *checksum) {
  if (n == 0) return fail(Err::Empty);
  if (k == 0) return fail(Err::ZeroK);
  if (stride == 0) stride = 1;
  Cell c;
  if (!cell || !make_cell(*cell, c)) return fail(Err::BadBox);
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  std::vector<size_t> active;
  active.reserve(n);
  for (size_t i = 0; i < n; ++i)
    if (!mask || mask[i] != 0) active.push_back(i);
  Binned b;
  b.cell = &c;
  b.k = k;
  const Err ge = plan_grid(c, cell_hint > 0.0, cell_hint, b.g);
  if (ge != Err::None) return fail(ge);
  build_bins(xyz, n, active, b);
  const auto t1 = clk::now();
  std::vector<size_t> sources;
  for (size_t s = 0, i = first; s < count && i < n; ++s, i += stride)
    if (!mask || mask[i] != 0) sources.push_back(i);
  const int nth = resolve_threads(threads);
  std::vector<KHeap> heaps(static_cast<size_t>(nth), KHeap(k));
  std::vector<std::vector<std::pair<double, size_t>>> rows(static_cast<size_t>(nth));
  std::vector<long long> sums(static_cast<size_t>(nth), 0);
  parallel_for(sources, nth, [&](size_t t, int w) {
    KHeap &heap = heaps[size_t(w)];
    walk_one(b, sources[t], heap, nullptr);
    heap.finish(rows[size_t(w)]);
    long long acc = 0;
    for (auto &pr : rows[size_t(w)]) acc += (long long)pr.second;
    sums[size_t(w)] += acc;
  });
  const auto t2 = clk::now();
  long long tot = 0;
  for (long long v : sums) tot += v;
  *prep_seconds = std::chrono::duration<double>(t1 - t0).count();
  *walk_seconds = std::chrono::duration<double>(t2 - t1).count();
  *walked = (long long)sources.size();
  *checksum = tot;
  clear_error();
  return 0;
}

}  // extern "C"
