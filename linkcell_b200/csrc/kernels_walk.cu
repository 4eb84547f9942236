// Chebyshev-shell k-nearest walk kernels (sm_100a).
//
// Reference semantics (HaoZeke/linkcell v0.3.3, src/knearest.rs:431-475):
// for each source, shells reach = 1, 2, ... of cell offsets (dx, dy, dz);
// every offset is a visit of one primary cell under one lattice shift;
// every occupant j != i is pushed into a bounded k-heap (KHeap,
// src/knearest.rs:106-129) with dist2_shifted; after each full shell the
// walk stops once the heap is full and its worst value is at most
// (reach * cell_min)^2.
//
// Why an unordered walk is exact. KHeap keeps, for every index j it holds,
// the minimum distance over j's visits, and its value multiset after any
// prefix of visits is the k smallest of those per-index minima, whatever
// the visit order. The stop test only reads that multiset, so the stop
// reach R* is order-independent too. The reference's final row is
// therefore {j : m_j < v} plus the indices with m_j == v (v = k-th value),
// sorted by (d2, index) -- unless more indices tie at v than slots remain,
// in which case which of them survive depends on the exact push history.
// The walk detects that case (a rejected or evicted value equal to the
// final k-th value) and re-runs the reference push sequence literally for
// that source: shells ascending, offsets in lexicographic order, occupants
// in descending point index.
//
// Three walks share this skeleton:
//  - plain FP64: every candidate distance in exact FP64;
//  - FP32: candidate distances from FP32 cell-local offsets; a candidate is
//    dropped without FP64 work only when d32 > theta (1 + alpha) + beta,
//    which proves the exact distance exceeds the heap's worst value theta,
//    so the reference would reject it too; whole cells are skipped by an
//    FP32 lower bound under the same test; everything else is recomputed
//    in exact FP64 and pushed into the same exact heap;
//  - learned: the FP32 walk whose filter starts at the proposed shell's
//    stop bound (R_p cell_min)^2 instead of +inf. For every reach up to R_p
//    the stop decision is unchanged by that filter; a source whose walk
//    passes R_p without stopping restarts without it.
#include <cuda/atomic>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "lc_kernels.h"

namespace lc {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr float kU32 = 5.9604645e-08f;  // 2^-24, FP32 unit roundoff

__device__ __forceinline__ int frame_of_sorted(const BatchBuffers &b, long long p) {
  int lo = 0, hi = b.nframes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((long long)b.off[b.frames[mid].cell_base] <= p)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Visits the offsets of shell R in the reference order
// (src/knearest.rs:436-445): dx outer, dz inner, each ascending; reach 1
// covers the whole 3x3x3 cube, larger reaches only the cube's surface.
template <class F>
__device__ __forceinline__ void for_each_shell_offset(int R, F &&visit) {
  for (int dx = -R; dx <= R; ++dx) {
    const bool fx = dx == -R || dx == R;
    for (int dy = -R; dy <= R; ++dy) {
      const bool full = fx || dy == -R || dy == R || R == 1;
      const int step = full ? 1 : 2 * R;
      for (int dz = -R; dz <= R; dz += step) visit(dx, dy, dz);
    }
  }
}

// Primary cell coordinate and wrap count of j = i + d (rem/div_euclid).
__device__ __forceinline__ void wrap_axis(int j, int n, int &c, int &w) {
  if (j >= 0 && j < n) {
    c = j;
    w = 0;
  } else {
    c = rem_euclid(j, n);
    w = div_euclid(j, n);
  }
}

__device__ __forceinline__ void push_replay(const BatchBuffers &b, long long p) {
  const uint32_t q = atomicAdd(b.replay_count, 1u);
  if ((long long)q < b.replay_cap)
    b.replay_list[q] = int(p);
  else
    atomicOr(b.status, kStatusReplayOverflow);
}

// (d, idx) lexicographic order of the working heap.
__device__ __forceinline__ bool key_gt(double d1, int i1, double d2, int i2) {
  return d1 > d2 || (d1 == d2 && i1 > i2);
}

// Max-heap of (d, idx), one slot every S words.
__device__ __forceinline__ void heap_sift_down(double *hd, int *hi, int S, int pos, int n) {
  const double d = hd[pos * S];
  const int id = hi[pos * S];
  for (;;) {
    int c = 2 * pos + 1;
    if (c >= n) break;
    double dc = hd[c * S];
    int ic = hi[c * S];
    if (c + 1 < n) {
      const double d2 = hd[(c + 1) * S];
      const int i2 = hi[(c + 1) * S];
      if (key_gt(d2, i2, dc, ic)) {
        c = c + 1;
        dc = d2;
        ic = i2;
      }
    }
    if (!key_gt(dc, ic, d, id)) break;
    hd[pos * S] = dc;
    hi[pos * S] = ic;
    pos = c;
  }
  hd[pos * S] = d;
  hi[pos * S] = id;
}

__device__ __forceinline__ void heap_build(double *hd, int *hi, int S, int n) {
  for (int s = n / 2 - 1; s >= 0; --s) heap_sift_down(hd, hi, S, s, n);
}

// In-place heapsort: ascending (d, idx).
__device__ __forceinline__ void heap_sort(double *hd, int *hi, int S, int n) {
  for (int end = n - 1; end > 0; --end) {
    const double td = hd[0];
    const int ti = hi[0];
    hd[0] = hd[end * S];
    hi[0] = hi[end * S];
    hd[end * S] = td;
    hi[end * S] = ti;
    heap_sift_down(hd, hi, S, 0, end);
  }
}

__device__ __forceinline__ double qnan() { return __longlong_as_double(0x7ff8000000000000ll); }
__device__ __forceinline__ double pinf() { return __longlong_as_double(0x7ff0000000000000ll); }

__device__ __forceinline__ void write_row(const BatchBuffers &b, const FrameDesc &fr, int i,
                                          const double *hd, const int *hi, int S, int n) {
  const int k = fr.k;
  int *row = b.out_nn + fr.out_base + (long long)i * k;
  for (int s = 0; s < k; ++s) row[s] = s < n ? hi[s * S] : -1;
  if (b.out_d2) {
    double *drow = b.out_d2 + fr.out_base + (long long)i * k;
    for (int s = 0; s < k; ++s) drow[s] = s < n ? hd[s * S] : qnan();
  }
}

struct LocalCounters {
  long long v[kNumCounters] = {};
};

__device__ __forceinline__ void flush_counters(const BatchBuffers &b, LocalCounters &c) {
#pragma unroll
  for (int t = 0; t < 10; ++t) {
    long long x = c.v[t];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(kFull, x, d);
    if ((threadIdx.x & 31) == 0 && x)
      atomicAdd((unsigned long long *)&b.counters[t], (unsigned long long)x);
  }
}

// ------------------------------------------------------------------------
// Literal replay of the reference walk for one source (KHeap::push,
// src/knearest.rs:106-129, in the reference visit order). The pushes that
// the reference turns into no-ops are skipped: a push of an index not in a
// full heap with d >= the heap's first maximum, and the index scan outside
// the wrapping regime, where no index is visited twice. Leaves the row
// sorted by (total_cmp, index) in hd / hi (stride S) and returns its length.
__device__ int replay_walk(const BatchBuffers &b, const FrameDesc &fr, long long p, double *hd,
                           int *hi, int S) {
  const int k = fr.k;
  const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
  const uint32_t lc = b.scell[p];
  const int ix = int(lc % uint32_t(nx));
  const int iy = int((lc / uint32_t(nx)) % uint32_t(ny));
  const int iz = int(lc / (uint32_t(nx) * uint32_t(ny)));
  const double px = b.sx[p], py = b.sy[p], pz = b.sz[p];
  const long long cb = fr.cell_base;
  int n = 0;
  int widx = 0;       // first slot holding the maximum (valid when n == k)
  double wmax = 0.0;  // hd[widx]
  auto rescan = [&]() {
    int w = 0;
    for (int u = 1; u < n; ++u)
      if (hd[u * S] > hd[w * S]) w = u;
    widx = w;
    wmax = hd[w * S];
  };
  for (int R = 1; R <= fr.max_reach; ++R) {
    const bool dedupe = 2 * R + 1 > nx || 2 * R + 1 > ny || 2 * R + 1 > nz;
    for_each_shell_offset(R, [&](int dx, int dy, int dz) {
      int cx, cy, cz, wa, wb, wc;
      wrap_axis(ix + dx, nx, cx, wa);
      wrap_axis(iy + dy, ny, cy, wb);
      wrap_axis(iz + dz, nz, cz, wc);
      const long long c = cb + ((long long)cz * ny + cy) * (long long)nx + cx;
      const uint32_t a0 = b.off[c], a1 = b.off[c + 1];
      if (a0 == a1) return;
      double shx, shy, shz;
      lattice_shift(fr, wa, wb, wc, shx, shy, shz);
      // the reference list of a cell runs in descending point index
      for (uint32_t t = a1; t-- > a0;) {
        if ((long long)t == p) continue;
        const double d = dist2_shifted(px, py, pz, b.sx[t], b.sy[t], b.sz[t], shx, shy, shz);
        const int j = b.sidx[t];
        if (dedupe) {
          int s = 0;
          for (; s < n; ++s)
            if (hi[s * S] == j) break;
          if (s < n) {
            if (d < hd[s * S]) {
              hd[s * S] = d;
              if (n == k) rescan();
            }
            continue;
          }
        }
        if (n < k) {
          hd[n * S] = d;
          hi[n * S] = j;
          ++n;
          if (n == k) rescan();
          continue;
        }
        if (d < wmax) {
          hd[widx * S] = d;
          hi[widx * S] = j;
          rescan();
        }
      }
    });
    if (n >= k && wmax <= stop_bound(R, fr.cell_min)) break;
  }
  // KHeap::finish: sort by (total_cmp, idx), src/knearest.rs:146-158
  for (int a = 1; a < n; ++a) {
    const double kd = hd[a * S];
    const int ki = hi[a * S];
    const long long kk = total_key(kd);
    int q = a;
    while (q > 0) {
      const long long pk = total_key(hd[(q - 1) * S]);
      if (pk > kk || (pk == kk && hi[(q - 1) * S] > ki)) {
        hd[q * S] = hd[(q - 1) * S];
        hi[q * S] = hi[(q - 1) * S];
        --q;
      } else {
        break;
      }
    }
    hd[q * S] = kd;
    hi[q * S] = ki;
  }
  return n;
}

// FP32 filter threshold: a candidate with d32 > thr(theta) has exact
// distance > theta. With e = per-component error bound of the FP32 offset
// (rounding of the cell-local offsets, of the edge-vector sum and of the
// two additions, plus the reference's own FP64 rounding eps64), the
// distance error is at most 6u d + 3 e^2 (1/u + 1) (the cross terms
// 2|D|e bounded by u D^2 + e^2 / u). alpha and beta carry margin.
__device__ __forceinline__ float fp32_threshold(double theta, double beta) {
  if (!(theta < pinf())) return __int_as_float(0x7f800000);
  return __double2float_ru(theta * (1.0 + 8.0 * double(kU32)) + beta);
}

__device__ __forceinline__ double fp32_beta(const FrameDesc &fr, int R) {
  const double e = double(kU32) * (6.0 * R + 8.0) * double(fr.ell) + fr.eps64 * (R + 2.0);
  return 4.0 * e * e / double(kU32) + 4.0 * e * e;
}

// ------------------------------------------------------------------------
// The walk of one source. MODE: kModePlainF64, kModeFastF32, kModeLearned.
template <int MODE>
__device__ void walk_source(const BatchBuffers &b, long long p, double *hd, int *hi, int S,
                            LocalCounters &cnt) {
  const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
  const FrameDesc &fr = b.frames[f];
  if (b.frame_flags[f] & kFrameNaN) {
    push_replay(b, p);
    ++cnt.v[kCntReplays];
    return;
  }
  const int k = fr.k;
  const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
  const uint32_t lc = b.scell[p];
  const int ix = int(lc % uint32_t(nx));
  const int iy = int((lc / uint32_t(nx)) % uint32_t(ny));
  const int iz = int(lc / (uint32_t(nx) * uint32_t(ny)));
  const double px = b.sx[p], py = b.sy[p], pz = b.sz[p];
  const long long cb = fr.cell_base;
  const uint32_t *__restrict__ off = b.off;
  const int max_reach = fr.max_reach;
  const double cell_min = fr.cell_min;

  // FP32 view: the source's offset from its cell corner and its position
  // inside the cell in bin units (for the cell lower bound).
  float plx = 0.f, ply = 0.f, plz = 0.f, fa = 0.f, fb = 0.f, fc = 0.f;
  float ev[9];
  float lam = 0.f;
  if (MODE != kModePlainF64) {
    const float4 r = b.rec[p];
    plx = r.x;
    ply = r.y;
    plz = r.z;
#pragma unroll
    for (int t = 0; t < 9; ++t) ev[t] = fr.ev[t];
    fa = fr.nhinv[0] * plx + fr.nhinv[1] * ply + fr.nhinv[2] * plz;
    fb = fr.nhinv[3] * plx + fr.nhinv[4] * ply + fr.nhinv[5] * plz;
    fc = fr.nhinv[6] * plx + fr.nhinv[7] * ply + fr.nhinv[8] * plz;
    lam = float(fr.lam_min) * 0.99f;
  }
  int Rp = 0;
  if (MODE == kModeLearned && b.proposal) {
    Rp = b.proposal[p];
    if (Rp > max_reach) Rp = max_reach;
  }

  int n = 0;
  double rej = pinf();
  int stopped = 0;
  for (;;) {  // one pass, plus a restart when a learned proposal was short
    n = 0;
    rej = pinf();
    stopped = 0;
    const double filt = Rp > 0 ? stop_bound(Rp, cell_min) : pinf();
    double theta = filt;  // everything above theta is certainly rejected
    for (int R = 1; R <= max_reach; ++R) {
      const bool dedupe = 2 * R + 1 > nx || 2 * R + 1 > ny || 2 * R + 1 > nz;
      ++cnt.v[kCntShells];
      const double beta = MODE != kModePlainF64 ? fp32_beta(fr, R) : 0.0;
      float thr = MODE != kModePlainF64 ? fp32_threshold(theta, beta) : 0.f;
      for_each_shell_offset(R, [&](int dx, int dy, int dz) {
        int cx, cy, cz, wa, wb, wc;
        wrap_axis(ix + dx, nx, cx, wa);
        wrap_axis(iy + dy, ny, cy, wb);
        wrap_axis(iz + dz, nz, cz, wc);
        const long long c = cb + ((long long)cz * ny + cy) * (long long)nx + cx;
        const uint32_t a0 = off[c], a1 = off[c + 1];
        if (a0 == a1) return;
        float Dx = 0.f, Dy = 0.f, Dz = 0.f;
        if (MODE != kModePlainF64) {
          // lower bound of the distance to any point of the cell
          const float ga = dx > 0 ? dx - fa : (dx < 0 ? fa + float(-dx - 1) : 0.f);
          const float gb = dy > 0 ? dy - fb : (dy < 0 ? fb + float(-dy - 1) : 0.f);
          const float gc = dz > 0 ? dz - fc : (dz < 0 ? fc + float(-dz - 1) : 0.f);
          const float ga0 = fmaxf(ga, 0.f), gb0 = fmaxf(gb, 0.f), gc0 = fmaxf(gc, 0.f);
          const float lb = lam * (ga0 * ga0 + gb0 * gb0 + gc0 * gc0);
          if (lb > thr) {
            ++cnt.v[kCntPruned];
            return;
          }
          const float fdx = float(dx), fdy = float(dy), fdz = float(dz);
          Dx = fdx * ev[0] + fdy * ev[3] + fdz * ev[6];
          Dy = fdx * ev[1] + fdy * ev[4] + fdz * ev[7];
          Dz = fdx * ev[2] + fdy * ev[5] + fdz * ev[8];
        }
        bool have_shift = false;
        double shx = 0.0, shy = 0.0, shz = 0.0;
        for (uint32_t t = a0; t < a1; ++t) {
          if ((long long)t == p) continue;
          int j;
          if (MODE != kModePlainF64) {
            const float4 q = b.rec[t];
            const float ex = (q.x - plx) + Dx;
            const float ey = (q.y - ply) + Dy;
            const float ez = (q.z - plz) + Dz;
            const float d32 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
            ++cnt.v[kCntPairs];
            if (d32 > thr) continue;  // exact distance > theta: rejected
            ++cnt.v[kCntRerank];
          } else {
            ++cnt.v[kCntPairs];
          }
          j = -1;
          if (!have_shift) {
            lattice_shift(fr, wa, wb, wc, shx, shy, shz);
            have_shift = true;
          }
          const double d = dist2_shifted(px, py, pz, b.sx[t], b.sy[t], b.sz[t], shx, shy, shz);
          if (MODE == kModeLearned && d > filt) continue;  // beyond the proposed bound
          if (j < 0) j = b.sidx[t];
          if (dedupe) {
            int s = 0;
            for (; s < n; ++s)
              if (hi[s * S] == j) break;
            if (s < n) {
              if (d < hd[s * S]) {
                hd[s * S] = d;
                if (n >= k) {
                  heap_sift_down(hd, hi, S, s, n);
                  theta = fmin(hd[0], filt);
                  if (MODE != kModePlainF64) thr = fp32_threshold(theta, beta);
                }
              }
              continue;
            }
          }
          if (n < k) {
            hd[n * S] = d;
            hi[n * S] = j;
            ++n;
            ++cnt.v[kCntInserts];
            if (n == k) {
              heap_build(hd, hi, S, n);
              theta = fmin(hd[0], filt);
              if (MODE != kModePlainF64) thr = fp32_threshold(theta, beta);
            }
          } else if (d < hd[0]) {
            rej = fmin(rej, hd[0]);
            hd[0] = d;
            hi[0] = j;
            heap_sift_down(hd, hi, S, 0, n);
            ++cnt.v[kCntInserts];
            theta = fmin(hd[0], filt);
            if (MODE != kModePlainF64) thr = fp32_threshold(theta, beta);
          } else {
            rej = fmin(rej, d);
          }
        }
      });
      if (n >= k && hd[0] <= stop_bound(R, cell_min)) {
        stopped = R;
        break;
      }
      if (MODE == kModeLearned && Rp > 0 && R == Rp) break;  // proposal too short
    }
    if (MODE == kModeLearned && Rp > 0) {
      if (stopped == 0) {
        ++cnt.v[kCntPropUnder];
        cnt.v[kCntRevisit] += Rp;
        Rp = 0;
        continue;  // walk again without the filter
      }
      if (stopped < Rp)
        ++cnt.v[kCntPropOver];
      else
        ++cnt.v[kCntPropExact];
    }
    break;
  }
  if (b.stop_log) b.stop_log[p] = int8_t(stopped > 0 ? (stopped < 127 ? stopped : 127) : 0);
  const int i = b.sidx[p];
  if (n >= k && !(rej > hd[0])) {
    // a value equal to the k-th was left out: which of the tied indices the
    // reference keeps depends on its exact push order
    ++cnt.v[kCntReplays];
    const int m = replay_walk(b, fr, p, hd, hi, S);
    write_row(b, fr, i, hd, hi, S, m);
    return;
  }
  if (n < k) heap_build(hd, hi, S, n);
  heap_sort(hd, hi, S, n);
  write_row(b, fr, i, hd, hi, S, n);
}

// 128 registers per thread at every block size (the heap is in shared memory).
template <int MODE, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 65536 / (128 * BLOCK)) k_walk(BatchBuffers b) {
  extern __shared__ double smem[];
  double *hd = smem + threadIdx.x;
  int *hi = reinterpret_cast<int *>(smem + (size_t)b.kmax * BLOCK) + threadIdx.x;
  const long long total = walk_sources(b);
  const int lane = threadIdx.x & 31;
  LocalCounters cnt;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(b.work, 32u);
    base = __shfl_sync(kFull, base, 0);
    if ((long long)base >= total) break;
    const long long q = (long long)base + lane;
    const long long p = q < total ? walk_source_at(b, q) : -1;
    if (p >= 0) walk_source<MODE>(b, p, hd, hi, BLOCK, cnt);
    __syncwarp();
  }
  flush_counters(b, cnt);
}

// Every queued source through the literal replay (NaN frames, very large k).
__global__ void __launch_bounds__(128) k_replay(BatchBuffers b) {
  long long cnt = *b.replay_count;
  if (cnt > b.replay_cap) cnt = b.replay_cap;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= b.replay_threads) return;
  double *hd = b.replay_d + tid * b.kmax;
  int *hi = b.replay_i + tid * b.kmax;
  for (long long q = tid; q < cnt; q += b.replay_threads) {
    const long long p = b.replay_list[q];
    const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
    const FrameDesc &fr = b.frames[f];
    const int m = replay_walk(b, fr, p, hd, hi, 1);
    write_row(b, fr, b.sidx[p], hd, hi, 1, m);
  }
}

__global__ void k_queue_all(BatchBuffers b) {
  const long long total = walk_sources(b);
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const long long p = walk_source_at(b, q);
    if (p >= 0) push_replay(b, p);
  }
}

// ------------------------------------------------------------------------
// Team walk: one warp per source.
//
// Lanes take the offsets of a shell (32 at a time, near-first order), load
// their cells' occupant ranges, and a warp scan lays the candidates out so
// that every lane evaluates one candidate per round. The k best (d2, index)
// pairs live in a warp-distributed list sorted ascending: position
// lane * KPL + s. Control flow is uniform across the warp; only the FP32
// test, the exact recompute and the insertions are predicated.

// Offset e of shell R: the near-first table for R <= rmax (shell 1, the
// whole 3x3x3 cube, at [0, 27); shell R > 1 at [(2R-1)^3, (2R+1)^3)), else
// decoded from the index.
__device__ __forceinline__ void shell_offset(const BatchBuffers &b, int R, int e, int &dx, int &dy,
                                             int &dz) {
  if (R <= b.shell_rmax) {
    const int base = R == 1 ? 0 : (2 * R - 1) * (2 * R - 1) * (2 * R - 1);
    const uint32_t w = b.shell_table[base + e];
    dx = int(w & 1023u) - 512;
    dy = int((w >> 10) & 1023u) - 512;
    dz = int((w >> 20) & 1023u) - 512;
    return;
  }
  const int w = 2 * R + 1, v = 2 * R - 1;
  const int f1 = 2 * w * w, f2 = 2 * v * w;
  if (e < f1) {
    const int side = e / (w * w), r = e - side * w * w;
    dx = side ? R : -R;
    dy = r / w - R;
    dz = r % w - R;
  } else if (e < f1 + f2) {
    const int e2 = e - f1, side = e2 / (v * w), r = e2 - side * v * w;
    dy = side ? R : -R;
    dx = r / w - (R - 1);
    dz = r % w - R;
  } else {
    const int e3 = e - f1 - f2, side = e3 / (v * v), r = e3 - side * v * v;
    dz = side ? R : -R;
    dx = r / v - (R - 1);
    dy = r % v - (R - 1);
  }
}

__device__ __forceinline__ double shfl_d(double v, int src) {
  return __shfl_sync(kFull, v, src);
}

__device__ __forceinline__ bool lex_less(double d1, int i1, double d2, int i2) {
  return d1 < d2 || (d1 == d2 && i1 < i2);
}

// The warp's sorted k-list.
template <int KPL>
struct TeamList {
  double d[KPL];
  int j[KPL];
};

// Inserts (x, jx) (same on every lane) into the sorted list; returns the
// value pushed to position k (the evicted k-th entry) or +inf.
template <int KPL>
__device__ __forceinline__ double team_insert(TeamList<KPL> &L, int lane, int k, double x, int jx) {
  int c = 0;
#pragma unroll
  for (int s = 0; s < KPL; ++s) c += lex_less(L.d[s], L.j[s], x, jx) ? 1 : 0;
  int P;
  if (KPL == 1) {
    P = __popc(__ballot_sync(kFull, c != 0));
  } else {
    P = c;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) P += __shfl_xor_sync(kFull, P, o);
  }
  // value at position k-1 before the shift: evicted when P < k
  const double at_km1 = shfl_d(L.d[(k - 1) % KPL], (k - 1) / KPL);
  const double up_d = shfl_d(L.d[KPL - 1], (lane + 31) & 31);
  const int up_j = __shfl_sync(kFull, L.j[KPL - 1], (lane + 31) & 31);
#pragma unroll
  for (int s = KPL - 1; s >= 0; --s) {
    const int pos = lane * KPL + s;
    const double bd = s == 0 ? up_d : L.d[s - 1];
    const int bj = s == 0 ? up_j : L.j[s - 1];
    if (pos > P) {
      L.d[s] = bd;
      L.j[s] = bj;
    } else if (pos == P) {
      L.d[s] = x;
      L.j[s] = jx;
    }
  }
  return P < k ? at_km1 : x;
}

// Removes position q from the sorted list (entries above move down; the
// last slot becomes +inf).
template <int KPL>
__device__ __forceinline__ void team_remove(TeamList<KPL> &L, int lane, int q) {
  const double dn_d = shfl_d(L.d[0], (lane + 1) & 31);
  const int dn_j = __shfl_sync(kFull, L.j[0], (lane + 1) & 31);
#pragma unroll
  for (int s = 0; s < KPL; ++s) {
    const int pos = lane * KPL + s;
    if (pos >= q) {
      if (s + 1 < KPL) {
        L.d[s] = L.d[s + 1];
        L.j[s] = L.j[s + 1];
      } else if (lane < 31) {
        L.d[s] = dn_d;
        L.j[s] = dn_j;
      } else {
        L.d[s] = pinf();
        L.j[s] = 0x7fffffff;
      }
    }
  }
}

// Bitonic sort of one (d, j) pair per lane, ascending by (d, j).
__device__ __forceinline__ void warp_sort_pairs(double &d, int &j, int lane) {
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const double od = __shfl_xor_sync(kFull, d, stride);
      const int oj = __shfl_xor_sync(kFull, j, stride);
      const bool up = ((lane & size) == 0);
      const bool lower = (lane & stride) == 0;
      const bool other_less = lex_less(od, oj, d, j);
      const bool take = (lower == up) ? other_less : !other_less && !(od == d && oj == j);
      if (take) {
        d = od;
        j = oj;
      }
    }
  }
}

// Merges the (already filtered) candidates of a round, one per lane
// (+inf where none), into a KPL == 1 list. Returns, per lane, the smallest
// value that left the first k positions (or +inf).
__device__ __forceinline__ double team_merge32(TeamList<1> &L, int lane, int k, double cd, int cj) {
  warp_sort_pairs(cd, cj, lane);
  // reversed candidates against the ascending list: the lane-wise minima
  // are the 32 smallest of the union, as a bitonic sequence
  const double rd = __shfl_sync(kFull, cd, 31 - lane);
  const int rj = __shfl_sync(kFull, cj, 31 - lane);
  double out_d;
  if (lex_less(rd, rj, L.d[0], L.j[0])) {
    out_d = L.d[0];
    L.d[0] = rd;
    L.j[0] = rj;
  } else {
    out_d = rd;
  }
  // bitonic merge (ascending)
#pragma unroll
  for (int stride = 16; stride > 0; stride >>= 1) {
    const double od = __shfl_xor_sync(kFull, L.d[0], stride);
    const int oj = __shfl_xor_sync(kFull, L.j[0], stride);
    const bool lower = (lane & stride) == 0;
    const bool other_less = lex_less(od, oj, L.d[0], L.j[0]);
    if (lower ? other_less : (!other_less && !(od == L.d[0] && oj == L.j[0]))) {
      L.d[0] = od;
      L.j[0] = oj;
    }
  }
  // the lane-wise maxima left the list; so did positions >= k
  double gone = out_d;
  if (lane >= k) gone = fmin(gone, L.d[0]);
  return gone;
}

template <int MODE, int KPL>
__device__ void team_source(const BatchBuffers &b, long long p, int lane, LocalCounters &cnt) {
  const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
  const FrameDesc &fr = b.frames[f];
  if (b.frame_flags[f] & kFrameNaN) {
    if (lane == 0) {
      push_replay(b, p);
      ++cnt.v[kCntReplays];
    }
    return;
  }
  const int k = fr.k;
  const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
  const uint32_t lc = b.scell[p];
  const int ix = int(lc % uint32_t(nx));
  const int iy = int((lc / uint32_t(nx)) % uint32_t(ny));
  const int iz = int(lc / (uint32_t(nx) * uint32_t(ny)));
  const double px = b.sx[p], py = b.sy[p], pz = b.sz[p];
  const long long cb = fr.cell_base;
  const int max_reach = fr.max_reach;
  const double cell_min = fr.cell_min;

  float plx = 0.f, ply = 0.f, plz = 0.f, fa = 0.f, fb = 0.f, fc = 0.f, lam = 0.f;
  if (MODE != kModePlainF64) {
    const float4 r = b.rec[p];
    plx = r.x;
    ply = r.y;
    plz = r.z;
    fa = fr.nhinv[0] * plx + fr.nhinv[1] * ply + fr.nhinv[2] * plz;
    fb = fr.nhinv[3] * plx + fr.nhinv[4] * ply + fr.nhinv[5] * plz;
    fc = fr.nhinv[6] * plx + fr.nhinv[7] * ply + fr.nhinv[8] * plz;
    lam = float(fr.lam_min) * 0.99f;
  }
  int Rp = 0;
  if (MODE == kModeLearned && b.proposal) {
    Rp = b.proposal[p];
    if (Rp > max_reach) Rp = max_reach;
  }

  TeamList<KPL> L;
  int filled = 0;
  double rej = pinf();
  int stopped = 0;
  for (;;) {  // one pass, plus a restart when a learned proposal was short
#pragma unroll
    for (int s = 0; s < KPL; ++s) {
      L.d[s] = pinf();
      L.j[s] = 0x7fffffff;
    }
    filled = 0;
    rej = pinf();
    stopped = 0;
    const double filt = Rp > 0 ? stop_bound(Rp, cell_min) : pinf();
    double theta = filt;
    for (int R = 1; R <= max_reach; ++R) {
      const bool dedupe = 2 * R + 1 > nx || 2 * R + 1 > ny || 2 * R + 1 > nz;
      if (lane == 0) ++cnt.v[kCntShells];
      const double beta = MODE != kModePlainF64 ? fp32_beta(fr, R) : 0.0;
      float thr = MODE != kModePlainF64 ? fp32_threshold(theta, beta) : 0.f;
      const int E = R == 1 ? 27 : 24 * R * R + 2;
      for (int e0 = 0; e0 < E; e0 += 32) {
        const int e = e0 + lane;
        int a0 = 0, nc = 0, wa = 0, wb = 0, wc = 0;
        float Dx = 0.f, Dy = 0.f, Dz = 0.f;
        if (e < E) {
          int dx, dy, dz;
          shell_offset(b, R, e, dx, dy, dz);
          int cx, cy, cz;
          wrap_axis(ix + dx, nx, cx, wa);
          wrap_axis(iy + dy, ny, cy, wb);
          wrap_axis(iz + dz, nz, cz, wc);
          const long long c = cb + ((long long)cz * ny + cy) * (long long)nx + cx;
          a0 = int(b.off[c]);
          nc = int(b.off[c + 1]) - a0;
          if (MODE != kModePlainF64 && nc > 0) {
            const float ga = dx > 0 ? dx - fa : (dx < 0 ? fa + float(-dx - 1) : 0.f);
            const float gb = dy > 0 ? dy - fb : (dy < 0 ? fb + float(-dy - 1) : 0.f);
            const float gc = dz > 0 ? dz - fc : (dz < 0 ? fc + float(-dz - 1) : 0.f);
            const float ga0 = fmaxf(ga, 0.f), gb0 = fmaxf(gb, 0.f), gc0 = fmaxf(gc, 0.f);
            if (lam * (ga0 * ga0 + gb0 * gb0 + gc0 * gc0) > thr) {
              ++cnt.v[kCntPruned];
              nc = 0;
            } else {
              const float fdx = float(dx), fdy = float(dy), fdz = float(dz);
              Dx = fdx * fr.ev[0] + fdy * fr.ev[3] + fdz * fr.ev[6];
              Dy = fdx * fr.ev[1] + fdy * fr.ev[4] + fdz * fr.ev[7];
              Dz = fdx * fr.ev[2] + fdy * fr.ev[5] + fdz * fr.ev[8];
            }
          }
        }
        // candidates of this chunk: inclusive scan of the cell counts
        int incl = nc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += y;
        }
        const int tot = __shfl_sync(kFull, incl, 31);
        const int excl = incl - nc;
        for (int g0 = 0; g0 < tot; g0 += 32) {
          const int g = g0 + lane;
          // owner lane: number of lanes whose inclusive count is <= g
          int owner = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1) {
            const int v = __shfl_sync(kFull, incl, owner + step - 1);
            if (v <= g) owner += step;
          }
          owner &= 31;
          const int oa0 = __shfl_sync(kFull, a0, owner);
          const int oex = __shfl_sync(kFull, excl, owner);
          const int owa = __shfl_sync(kFull, wa, owner);
          const int owb = __shfl_sync(kFull, wb, owner);
          const int owc = __shfl_sync(kFull, wc, owner);
          const float oDx = __shfl_sync(kFull, Dx, owner);
          const float oDy = __shfl_sync(kFull, Dy, owner);
          const float oDz = __shfl_sync(kFull, Dz, owner);
          const long long t = (long long)oa0 + (g - oex);
          bool pass = g < tot && t != p;
          int j = 0;
          if (pass) {
            ++cnt.v[kCntPairs];
            if (MODE != kModePlainF64) {
              const float4 q = b.rec[t];
              const float ex = (q.x - plx) + oDx;
              const float ey = (q.y - ply) + oDy;
              const float ez = (q.z - plz) + oDz;
              const float d32 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
              pass = !(d32 > thr);
            }
            if (pass) j = b.sidx[t];
          }
          const unsigned pm = __ballot_sync(kFull, pass);
          if (pm == 0) continue;
          double d = pinf();
          if (pass) {
            if (MODE != kModePlainF64) ++cnt.v[kCntRerank];
            double shx, shy, shz;
            lattice_shift(fr, owa, owb, owc, shx, shy, shz);
            d = dist2_shifted(px, py, pz, b.sx[t], b.sy[t], b.sz[t], shx, shy, shz);
            if (MODE == kModeLearned && d > filt) pass = false;  // beyond the proposed bound
          }
          // insertion candidates: below theta, or anything while the list fills
          bool ins = pass && (filled < k || d < theta);
          if (pass && !ins) rej = fmin(rej, d);
          unsigned im = __ballot_sync(kFull, ins);
          if (im == 0) continue;
          if (KPL == 1 && !dedupe && __popc(im) >= 6) {
            const int added = __popc(im);
            const double gone = team_merge32(reinterpret_cast<TeamList<1> &>(L), lane, k,
                                             ins ? d : pinf(), ins ? j : 0x7fffffff);
            if (filled + added > k) rej = fmin(rej, gone);
            filled = min(filled + added, k);
            cnt.v[kCntInserts] += lane == 0 ? added : 0;
          } else {
            while (im) {
              const int src = __ffs(im) - 1;
              im &= im - 1;
              const double x = shfl_d(d, src);
              const int jx = __shfl_sync(kFull, j, src);
              if (filled >= k && !(x < theta)) {  // theta fell below it in this round
                rej = fmin(rej, x);
                continue;
              }
              if (dedupe) {
                // an index already listed keeps its smaller distance
                bool has = false;
                int qpos = 0;
#pragma unroll
                for (int s = 0; s < KPL; ++s) {
                  const int pos = lane * KPL + s;
                  const bool hit = pos < filled && L.j[s] == jx;
                  const unsigned hm = __ballot_sync(kFull, hit);
                  if (hm) {
                    has = true;
                    qpos = (__ffs(hm) - 1) * KPL + s;
                  }
                }
                if (has) {
                  const double old = shfl_d(L.d[qpos % KPL], qpos / KPL);
                  if (!(x < old)) continue;
                  team_remove(L, lane, qpos);
                  --filled;
                }
              }
              const double gone = team_insert(L, lane, k, x, jx);
              if (filled >= k) rej = fmin(rej, gone);
              filled = min(filled + 1, k);
              if (lane == 0) ++cnt.v[kCntInserts];
              if (filled >= k) {
                theta = fmin(shfl_d(L.d[(k - 1) % KPL], (k - 1) / KPL), filt);
                if (MODE != kModePlainF64) thr = fp32_threshold(theta, beta);
              }
            }
            continue;
          }
          if (filled >= k) {
            theta = fmin(shfl_d(L.d[(k - 1) % KPL], (k - 1) / KPL), filt);
            if (MODE != kModePlainF64) thr = fp32_threshold(theta, beta);
          }
        }
      }
      if (filled >= k && shfl_d(L.d[(k - 1) % KPL], (k - 1) / KPL) <= stop_bound(R, cell_min)) {
        stopped = R;
        break;
      }
      if (MODE == kModeLearned && Rp > 0 && R == Rp) break;  // proposal too short
    }
    if (MODE == kModeLearned && Rp > 0) {
      if (stopped == 0) {
        if (lane == 0) {
          ++cnt.v[kCntPropUnder];
          cnt.v[kCntRevisit] += Rp;
        }
        Rp = 0;
        continue;
      }
      if (lane == 0) ++cnt.v[stopped < Rp ? kCntPropOver : kCntPropExact];
    }
    break;
  }
  if (b.stop_log && lane == 0)
    b.stop_log[p] = int8_t(stopped > 0 ? (stopped < 127 ? stopped : 127) : 0);
  // tie across the k-th slot: the reference's push order decides
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) rej = fmin(rej, __shfl_xor_sync(kFull, rej, o));
  if (filled >= k) {
    const double vk = shfl_d(L.d[(k - 1) % KPL], (k - 1) / KPL);
    if (!(rej > vk)) {
      if (lane == 0) {
        push_replay(b, p);
        ++cnt.v[kCntReplays];
      }
      return;
    }
  }
  const int i = b.sidx[p];
  int *row = b.out_nn + fr.out_base + (long long)i * k;
  double *drow = b.out_d2 ? b.out_d2 + fr.out_base + (long long)i * k : nullptr;
#pragma unroll
  for (int s = 0; s < KPL; ++s) {
    const int pos = lane * KPL + s;
    if (pos < k) {
      const bool ok = pos < filled;
      row[pos] = ok ? L.j[s] : -1;
      if (drow) drow[pos] = ok ? L.d[s] : qnan();
    }
  }
}

template <int MODE, int KPL>
__global__ void __launch_bounds__(256, 2) k_team_walk(BatchBuffers b) {
  const long long total = walk_sources(b);
  const int lane = threadIdx.x & 31;
  LocalCounters cnt;
  constexpr int kGrab = 4;  // sources per work-queue grab (consecutive, share candidates)
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(b.work, uint32_t(kGrab));
    base = __shfl_sync(kFull, base, 0);
    if ((long long)base >= total) break;
    for (int q = 0; q < kGrab; ++q) {
      if ((long long)base + q >= total) break;
      const long long p = walk_source_at(b, (long long)base + q);
      if (p >= 0) team_source<MODE, KPL>(b, p, lane, cnt);
    }
  }
  flush_counters(b, cnt);
}

// ------------------------------------------------------------------------
// Cube select walk of the learned mode: one warp per source opens the
// proposed cube (shells 1..R_p) in one pass and selects instead of inserting.
//
//  1. Gather. The cube is (2 R_p + 1)^2 rows of cells along x; cells sort by
//     (z, y, x), so the cells of a row that survive the distance bound form
//     at most two contiguous ranges of the sorted points (two when the row
//     wraps the box in x). Each lane trims one row to the x range that can
//     hold a point within the filter (the Schur form of the bin-unit metric
//     bounds the other two axes' share), the warp walks the concatenated
//     ranges in two 32-candidate windows per trip (the row of candidate g is
//     found from one OR-reduction of row starts), and candidates below the
//     FP32 filter go to a per-warp buffer (FP32 distance, sorted position,
//     shell, wrap counts). The first gather covers only
//     rho2 = max(B(R_p - 1), q B(R_p)); when fewer than k candidates lie
//     within rho2, the whole ball B(R_p) = (R_p cell_min)^2 is gathered.
//  2. Stop reach. The reference stops at the first R with at least k
//     candidates of shells <= R within B(R). Each candidate counts from
//     reach max(shell, b(d)), b(d) = the first R >= 1 with d <= B(R), read
//     from sqrt(d32) / cell_min and decided in exact FP64 whenever that value
//     lies within its error band of an integer. No R <= R_p qualifies: the
//     proposal was short and the source goes to the literal replay.
//  3. Select. Two 32-bucket histograms (linear in d32 over [0, B(R*)], then
//     within the bucket holding the k-th value) give T = the largest d32 of
//     the buckets up to the k-th; S = the candidates of shells <= R* with
//     d32 <= T + 3 band(T) holds the k smallest exact distances and every
//     value tied with the k-th, and nothing else can tie (with the FP32 error
//     band(x) = 8u x + beta, any candidate above T + 3 band(T) has an exact
//     distance above T + band(T), which bounds the k-th value).
//  4. S is recomputed in exact FP64, every element is ranked in (d2, index)
//     order against the others, and ranks 0..k-1 are the row; a tie across
//     the k-th slot goes to the literal replay.
// Any proposal gives the reference result: a short proposal, a buffer
// overflow, a cube that wraps the box, k > 64 or an S larger than its buffer
// (64 entries for k <= 32, 128 for k <= 64) sends
// the source to the literal replay.
constexpr int kSelCap = 256;   // FP32-filtered candidates per warp (smem left to L1)
constexpr int kSelWin = 2;     // 32-candidate windows a gather trip loads at once
// Warps per block (the autotuner picks among two per S size): 8 or 4 for
// k <= 32, 4 or 2 for k <= 64. Resident warps per SM: 32 for k <= 32 (64
// registers, a few bytes spilled) and 28 for k <= 64; more warps hide the
// walk's dependency chains better than the registers they cost (4M k = 32:
// 8.28 ms at 24 warps, 7.99 ms at 32; k = 64: 16.0 ms at 20, 14.5 ms at 28).
template <int SN>
constexpr int sel_warps_per_sm() { return SN == 2 ? 32 : 28; }
template <int SN>
constexpr int sel_default_warps() { return SN == 2 ? 8 : 4; }

// One contiguous run of sorted points of a cube row: the cells of the row
// inside the box, or the ones across the x boundary (a row yields one or two).
struct __align__(16) SelSeg {
  int excl;        // first candidate position of the run
  int start;       // its first sorted position
  int xoff;        // dx = candidate cell x + xoff
  uint32_t meta;   // wrap index of its candidates in SelShared::tm layout
  float Dx, Dy, Dz;  // dy e_b + dz e_c (FP32)
  int syz;           // max(1, |dy|, |dz|)
};

// SN: elements of S per lane (S holds at most 32 SN; k <= 16 SN).
template <int SN>
struct SelShared {
  float d[kSelCap];
  // x: sorted position; y: shell | ((wa + 1) 9 + (wb + 1) 3 + (wc + 1)) << 8,
  // the wrap triple as its index into FrameDesc::shift27
  uint2 tm[kSelCap];
  SelSeg segs[64];
  double sd[32 * SN];
  int sj[32 * SN];
  int si[32 * SN];
  int hist[32];
  unsigned hmax[32];
  unsigned long long wc[16];  // warp-uniform counters (SelWarpCounter), lane 0 updates
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Ascending bitonic sort of 32 H unsigned keys held H per lane: position q
// is lane q % 32's key[q / 32]. Every comparator is ascending (the lower
// position keeps the smaller key): the merge of blocks of kk first pairs q
// with q ^ (kk - 1), the block reversed, then q with q ^ j for j = kk / 4
// .. 1. Within a lane's keys the lower position is the lower h; across lanes
// it is the lane whose bit j is clear, so each step is one shuffle and one
// min-or-max per key.
// LOWER: the last merge sorts only the lower half (positions 0 .. 31, key[0]):
// after its mirror step they hold the 32 smallest keys; the upper ones are
// left for bitonic_upper.
template <int H, bool LOWER = false>
__device__ __forceinline__ void bitonic_sort(uint32_t (&key)[H], int lane) {
#pragma unroll
  for (int kk = 2; kk <= 32 * H; kk <<= 1) {
#pragma unroll
    for (int j = kk >> 1; j > 0; j >>= 1) {
      const bool flip = j == (kk >> 1);
      if (j >= 32) {
        // partners in key h ^ dh: of the reversed lane (flip) or this lane
        const int dh = flip ? (kk - 1) >> 5 : j >> 5;
        uint32_t part[H];
#pragma unroll
        for (int h = 0; h < H; ++h)
          part[h] = flip ? __shfl_xor_sync(kFull, key[h ^ dh], 31) : key[h ^ dh];
#pragma unroll
        for (int h = 0; h < H; ++h)
          key[h] = h < (h ^ dh) ? min(key[h], part[h]) : max(key[h], part[h]);
      } else {
        const bool lower = (lane & j) == 0;
#pragma unroll
        for (int h = 0; h < H; ++h) {
          if (LOWER && kk == 32 * H && h > 0) continue;
          const uint32_t pk = __shfl_xor_sync(kFull, key[h], flip ? kk - 1 : j);
          key[h] = lower ? min(key[h], pk) : max(key[h], pk);
        }
      }
    }
  }
}

// The rest of bitonic_sort<2, true>: sorts the upper half (positions 32 ..
// 63, key[1]), a bitonic sequence after the last merge's mirror step.
__device__ __forceinline__ void bitonic_upper(uint32_t &k1, int lane) {
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) {
    const uint32_t pk = __shfl_xor_sync(kFull, k1, j);
    k1 = (lane & j) == 0 ? min(k1, pk) : max(k1, pk);
  }
}

// Walk statistics of a warp, kept in shared memory (lane 0 or shared
// atomics update them) so that they hold no registers.
enum SelWarpCounter {
  kWcInserts, kWcShells, kWcReplays, kWcUnder, kWcOver, kWcExact, kWcFallback, kWcRegather,
  kWcPairs, kWcPruned, kWcRerank, kWcSlots
};

// Packed FP32 pairs (Blackwell's f32x2 instructions round each component as
// the scalar instruction does).
__device__ __forceinline__ unsigned long long f2_pack(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}

// (q - p) + fma(f, e, D) for the x and y components at once.
__device__ __forceinline__ void offset_xy(float qx, float qy, unsigned long long pxy, float f,
                                          unsigned long long exy, float Dx, float Dy, float &ox,
                                          float &oy) {
  unsigned long long a, c, r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(a) : "l"(f2_pack(qx, qy)), "l"(pxy));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(c) : "l"(f2_pack(f, f)), "l"(exy), "l"(f2_pack(Dx, Dy)));
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(c));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(ox), "=f"(oy) : "l"(r));
}

// Square root from the hardware approximation (relative error below 2^-22),
// for bounds that carry a wider margin than that.
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Exact quotient of x by n from a double reciprocal estimate (x < 2^32).
__device__ __forceinline__ uint32_t quot(uint32_t x, uint32_t n, double inv) {
  uint32_t q = uint32_t(__double2uint_rz(double(x) * inv));
  if (q * n > x) --q;
  else if ((q + 1) * n <= x) ++q;
  return q;
}

// Steps 3-4 of the select walk when the gathered buffer holds at most 32 H
// candidates (H = 2 for k <= 32, 4 for k <= 64): a sort instead of
// histograms and ranking. With s = 6 slot bits for H = 2 and 7 for H = 4,
// and e = 2^(s - 23) the relative slot error:
//  - Every eligible candidate (shell <= R*, d32 within the histogram path's
//    bound) gets the key bits(d32) with its low s bits replaced by its buffer
//    slot: unique, and |key - d32| <= e d32. The 32 H keys are sorted.
//  - K = the k-th smallest key: k candidates have d32 <= Tup = K (1 + 2e),
//    so the k-th smallest exact distance v is at most Tup + band(Tup). S =
//    the sorted prefix with key <= (Tup + 3 band(Tup)) (1 + 2e): it holds
//    every candidate whose exact distance is at most Tup + band(Tup) (the k
//    smallest and everything tied with v), and nothing outside S can tie v
//    -- the histogram path's argument with the key's error added.
//  - S is recomputed in exact FP64. Sorted by key, two neighbours can be out
//    of exact (d2, index) order only if their keys lie within twice the
//    error bound band''(x) = band(x) + 2e x of each other; the runs of such
//    linked neighbours (clusters, almost always single elements) are ranked
//    exactly inside, and every other position is already its rank.
//  - A tie across the k-th slot (equal k-th and (k+1)-th exact values) sends
//    the source to the literal replay, as in the histogram path.
// The sorted selection takes the buffers of k <= 32 with at most 64
// candidates (two keys per lane), the histogram path the rest. (Four keys
// per lane for k <= 64 gave the same rows but a slower 4M walk: 14.88 ms
// against 14.49 ms with the histograms.)
template <int SN>
__device__ __forceinline__ bool sorted_fits(int total) {
  return SN == 2 && total <= 64;
}

template <int H, int SN, bool STATS>
__device__ bool select_sorted(const BatchBuffers &b, long long p, int lane, SelShared<SN> &sh,
                              const FrameDesc &fr, int o, int total, int Rs, int Rp, bool partial) {
  // kRel = 2e: 2^-16 (H = 2) or 2^-15 (H = 4)
  constexpr uint32_t kSlotMask = H == 2 ? 63u : 127u;
  constexpr float kRel = H == 2 ? 1.f / 65536.f : 1.f / 32768.f;
  const int k = fr.k;
  const float Bs_hi = (partial && Rs == Rp) ? fr.sel_rho_bhi[Rp] : fr.sel_bhi[Rs];
  const float beta_s = fr.sel_beta[Rs];
  uint32_t key[H];
#pragma unroll
  for (int h = 0; h < H; ++h) {
    const int idx = lane + 32 * h;
    key[h] = 0xffffffffu;
    if (idx < total) {
      const float d = sh.d[o + idx];
      if (int(sh.tm[o + idx].y & 255u) <= Rs && d <= Bs_hi)
        key[h] = (__float_as_uint(d) & ~kSlotMask) | uint32_t(idx);
    }
  }
  // k <= 32 (SN = 2): the k-th key is among the 32 smallest, so the upper
  // half is sorted only when S reaches into it
  constexpr bool kLower = H == 2 && SN == 2;
  bitonic_sort<H, kLower>(key, lane);
  uint32_t kv = key[0];
#pragma unroll
  for (int h = 1; h < H; ++h)
    if (h == (k - 1) >> 5) kv = key[h];
  const uint32_t kth = __shfl_sync(kFull, kv, (k - 1) & 31);
  if (kth == 0xffffffffu) return false;  // cannot happen: R* guarantees k eligible candidates
  const float Tup = __fmul_ru(__uint_as_float(kth), 1.f + kRel);
  const float TSk =
      __fmul_ru(__fadd_ru(Tup, __fmul_ru(3.f, __fmaf_ru(Tup, 8.f * kU32, beta_s))), 1.f + kRel);
  const uint32_t tsb = __float_as_uint(TSk);
  if (kLower && __any_sync(kFull, key[H - 1] <= tsb)) bitonic_upper(key[H - 1], lane);
  bool in[H];
  int nS = 0;
#pragma unroll
  for (int h = 0; h < H; ++h) {
    in[h] = key[h] <= tsb;
    nS += __popc(__ballot_sync(kFull, in[h]));
  }
  if (nS < k) return false;  // cannot happen
  if (STATS && lane == 0) sh.wc[kWcRerank] += unsigned(nS);
  // exact distances and indices of S (position lane + 32 h)
  double dd[H];
  int jj[H];
#pragma unroll
  for (int h = 0; h < H; ++h) {
    dd[h] = pinf();
    jj[h] = 0x7fffffff;
    if (32 * h < nS && in[h]) {
      const int i = o + int(key[h] & kSlotMask);
      const uint2 tm = sh.tm[i];
      const int t = int(tm.x);
      const double *sh3 = fr.shift27[tm.y >> 8];
      dd[h] = dist2_shifted(b.sx[p], b.sy[p], b.sz[p], b.sx[t], b.sy[t], b.sz[t], sh3[0], sh3[1],
                            sh3[2]);
      jj[h] = b.sidx[t];
    }
  }
  // clusters: position q is linked to q - 1 when their keys lie within
  // 2.01 band''(key_q); starts[h] bit l =
  // position l + 32 h does not link to its predecessor
  auto linked = [&](uint32_t kq, uint32_t kprev) -> bool {
    const float xq = __uint_as_float(kq), xp = __uint_as_float(kprev);
    const float bq = __fmaf_ru(xq, 8.f * kU32 + kRel, beta_s);
    return __fsub_ru(xq, xp) <= __fmul_ru(2.01f, bq);
  };
  unsigned starts[H];
  bool any_link = false;
#pragma unroll
  for (int h = 0; h < H; ++h) {
    const uint32_t up = __shfl_up_sync(kFull, key[h], 1);
    const uint32_t last = __shfl_sync(kFull, key[h > 0 ? h - 1 : 0], 31);
    const uint32_t prev = lane == 0 ? last : up;
    const int q = lane + 32 * h;
    const bool link = q > 0 && q < nS && linked(key[h], prev);
    starts[h] = __ballot_sync(kFull, !link);
    any_link |= starts[h] != 0xffffffffu && 32 * h < nS;
  }
  int rk[H];
#pragma unroll
  for (int h = 0; h < H; ++h) rk[h] = lane + 32 * h;
  if (any_link) {
    // cluster [a, e] of position q = lane + 32 h: a = the last start <= q,
    // e = the next start - 1 (or the last position of S)
    int a[H], e[H], sz = 1;
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const unsigned upto = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
      a[h] = 0;
      bool found = false;
#pragma unroll
      for (int g = H - 1; g >= 0; --g) {
        if (g > h || found) continue;
        const unsigned mk = g == h ? (starts[g] & upto) : starts[g];
        if (mk) {
          a[h] = 32 * g + 31 - __clz(mk);
          found = true;
        }
      }
      e[h] = nS - 1;
      found = false;
#pragma unroll
      for (int g = 0; g < H; ++g) {
        if (g < h || found) continue;
        const unsigned mk = g == h ? (starts[g] & ~upto) : starts[g];
        if (mk) {
          e[h] = min(nS - 1, 32 * g + __ffs(mk) - 2);
          found = true;
        }
      }
      if (lane + 32 * h < nS) sz = max(sz, e[h] - a[h] + 1);
    }
    const int M = int(__reduce_max_sync(kFull, unsigned(sz)));
    int c[H];
#pragma unroll
    for (int h = 0; h < H; ++h) c[h] = 0;
    for (int r = 0; r < M; ++r) {
#pragma unroll
      for (int h = 0; h < H; ++h) {
        // member r of this element's cluster (positions past it are skipped)
        const int pq = min(a[h] + r, 32 * H - 1);
        double x = 0.0;
        int y = 0;
#pragma unroll
        for (int g = 0; g < H; ++g) {
          const double xg = __shfl_sync(kFull, dd[g], pq & 31);
          const int yg = __shfl_sync(kFull, jj[g], pq & 31);
          if (g == (pq >> 5)) x = xg, y = yg;
        }
        if (a[h] + r <= e[h] && lex_less(x, y, dd[h], jj[h])) ++c[h];
      }
    }
#pragma unroll
    for (int h = 0; h < H; ++h)
      if (lane + 32 * h < nS) rk[h] = a[h] + c[h];
  }
  // a tie across the k-th slot: the k-th and (k+1)-th exact values are equal
  if (nS > k) {
#pragma unroll
    for (int h = 0; h < H; ++h) {
      if (lane + 32 * h < nS && rk[h] == k - 1)
        sh.hmax[0] = __double2loint(dd[h]), sh.hmax[1] = __double2hiint(dd[h]);
      if (lane + 32 * h < nS && rk[h] == k)
        sh.hmax[2] = __double2loint(dd[h]), sh.hmax[3] = __double2hiint(dd[h]);
    }
    __syncwarp();
    const bool tie = sh.hmax[0] == sh.hmax[2] && sh.hmax[1] == sh.hmax[3];
    __syncwarp();
    if (tie) {
      if (STATS && lane == 0) ++sh.wc[kWcReplays];
      return false;
    }
  }
  const int i = b.sidx[p];
  int *row = b.out_nn + fr.out_base + (long long)i * k;
  double *drow = b.out_d2 ? b.out_d2 + fr.out_base + (long long)i * k : nullptr;
#pragma unroll
  for (int h = 0; h < H; ++h) {
    if (lane + 32 * h < nS && rk[h] < k) {
      row[rk[h]] = jj[h];
      if (drow) drow[rk[h]] = dd[h];
    }
  }
  if (b.stop_log && lane == 0) b.stop_log[p] = int8_t(Rs);
  if (STATS && lane == 0) sh.wc[kWcInserts] += unsigned(k);
  return true;
}

// Step 2 of the select walk for the candidates of buffer entries
// [o, o + total) of source p: the stop reach R* (0 when no reach up to the
// proposal qualifies from this gather).
template <int SN, bool STATS>
__device__ int sel_reach(const BatchBuffers &b, long long p, int lane, SelShared<SN> &sh,
                         const FrameDesc &fr, int o, int total, int Rp, bool partial) {
  const int k = fr.k;
  const double cell_min = fr.cell_min;
  // exact distance of buffer entry i (absolute index)
  auto exact = [&](int i) -> double {
    const uint2 tm = sh.tm[i];
    const int t = int(tm.x);
    const double *sh3 = fr.shift27[tm.y >> 8];
    return dist2_shifted(b.sx[p], b.sy[p], b.sz[p], b.sx[t], b.sy[t], b.sz[t], sh3[0], sh3[1],
                         sh3[2]);
  };
  int Rs = 0;
  // 2. stop reach: key counts packed 16 bits per reach (reaches 1-4 | 5-8)
  const float inv_c = 1.f / float(cell_min);
  const float eps_r = fr.sel_epsr[Rp];
  unsigned long long klo = 0, khi = 0;
  unsigned in_rho = 0;  // first gather: candidates with exact distance <= rho2
  // the level-1 histogram of step 3 for R* = R_p (the common case) on the way
  // (not needed when the sorted selection takes the buffer)
  const bool use_hist = !sorted_fits<SN>(total);
  const float spec_hi = partial ? fr.sel_rho_bhi[Rp] : fr.sel_bhi[Rp];
  const float spec_scale = 32.f / spec_hi;
  if (use_hist) sh.hist[lane] = 0;
  __syncwarp();
  for (int i = lane; i < total; i += 32) {
    const float d32 = sh.d[o + i];
    if (use_hist && d32 <= spec_hi) atomicAdd(&sh.hist[min(31, int(d32 * spec_scale))], 1);
    const int s = int(sh.tm[o + i].y & 255u);
    // sqrt error 2^-22 rr: inside the 16 u (R + 2) of eps_r beside the rest of
    // the FP32 evaluation (about 1.5 u rr)
    const float rr = sqrt_approx(d32) * inv_c;
    const float rc = ceilf(rr);
    int bR;
    double dex = -1.0;
    if (rr <= 1.f - eps_r) {
      bR = 1;
    } else if (rc - rr < eps_r || rr - (rc - 1.f) < eps_r) {
      dex = exact(o + i);
      if (STATS) atomicAdd(&sh.wc[kWcRerank], 1ull);
      int R = max(1, int(rc) - 1);
      while (R <= Rp && !(dex <= stop_bound(R, cell_min))) ++R;
      bR = R;
    } else {
      bR = int(rc);
    }
    if (partial) {
      if (d32 <= fr.sel_rho_lo[Rp]) {
        ++in_rho;
      } else if (!(d32 > fr.sel_rho_hi[Rp])) {
        if (dex < 0.0) {
          dex = exact(o + i);
          if (STATS) atomicAdd(&sh.wc[kWcRerank], 1ull);
        }
        in_rho += dex <= fr.sel_rho2[Rp] ? 1u : 0u;
      }
    }
    const int key = max(s, bR);
    if (key <= Rp) {
      const unsigned long long one = 1ull << (16 * ((key - 1) & 3));
      if (key <= 4)
        klo += one;
      else
        khi += one;
    }
  }
  const unsigned c12 = __reduce_add_sync(kFull, unsigned(klo));
  const unsigned c34 = __reduce_add_sync(kFull, unsigned(klo >> 32));
  unsigned c56 = 0, c78 = 0;  // keys above 4 exist only when R_p > 4
  if (Rp > 4) {
    c56 = __reduce_add_sync(kFull, unsigned(khi));
    c78 = __reduce_add_sync(kFull, unsigned(khi >> 32));
  }
  {
    // reaches below R_p are exact in both gathers; R_p itself from the
    // whole ball, or from the candidates within rho2 after the first
    unsigned cum = 0;
#pragma unroll
    for (int R = 1; R <= 8; ++R) {
      const unsigned w = R <= 2 ? c12 : (R <= 4 ? c34 : (R <= 6 ? c56 : c78));
      cum += (R & 1) ? (w & 0xffffu) : (w >> 16);
      if (Rs == 0 && (partial ? R < Rp : R <= Rp) && cum >= unsigned(k)) Rs = R;
    }
  }
  if (Rs == 0 && partial && __reduce_add_sync(kFull, in_rho) >= unsigned(k)) Rs = Rp;
  return Rs;
}

// Steps 3-4 of the select walk for the candidates of buffer entries
// [o, o + total) of source p with stop reach Rs: writes the row, or returns
// false when the source must go to the literal replay.
template <int SN, bool STATS>
__device__ bool sel_finish(const BatchBuffers &b, long long p, int lane, SelShared<SN> &sh,
                           const FrameDesc &fr, int o, int total, int Rs, int Rp, bool partial) {
  const int k = fr.k;
  // exact distance of buffer entry i (absolute index)
  auto exact = [&](int i) -> double {
    const uint2 tm = sh.tm[i];
    const int t = int(tm.x);
    const double *sh3 = fr.shift27[tm.y >> 8];
    return dist2_shifted(b.sx[p], b.sy[p], b.sz[p], b.sx[t], b.sy[t], b.sz[t], sh3[0], sh3[1],
                         sh3[2]);
  };
  if (Rs < Rp)
    { if (STATS && lane == 0) ++sh.wc[kWcOver]; }
  else
    { if (STATS && lane == 0) ++sh.wc[kWcExact]; }
  if (STATS && lane == 0) sh.wc[kWcShells] += unsigned(Rs);
  if (sorted_fits<SN>(total))
    return select_sorted<2, SN, STATS>(b, p, lane, sh, fr, o, total, Rs, Rp, partial);

  // 3. select: two-level histogram over candidates of shells <= R* within
  // B(R*) (within rho2 when the first gather settled R* = R_p)
  const float Bs_hi = (partial && Rs == Rp) ? fr.sel_rho_bhi[Rp] : fr.sel_bhi[Rs];
  const float beta_s = fr.sel_beta[Rs];  // candidates of shells <= R* have offsets <= R*
  const float scale = 32.f / Bs_hi;
  sh.hmax[lane] = 0u;
  __syncwarp();
  if (Rs != Rp) {  // the histogram built with the stop reach assumed R* = R_p
    sh.hist[lane] = 0;
    __syncwarp();
    for (int i = lane; i < total; i += 32) {
      const float d32 = sh.d[o + i];
      if (int(sh.tm[o + i].y & 255u) <= Rs && d32 <= Bs_hi)
        atomicAdd(&sh.hist[min(31, int(d32 * scale))], 1);
    }
    __syncwarp();
  }
  int bstar, need;
  {
    const int c = sh.hist[lane];
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const unsigned reach = __ballot_sync(kFull, incl >= k);
    if (!reach) return false;  // cannot happen: R* guarantees k candidates within B(R*)
    bstar = __ffs(reach) - 1;
    need = k - (__shfl_sync(kFull, incl, bstar) - __shfl_sync(kFull, c, bstar));
  }
  __syncwarp();
  sh.hist[lane] = 0;
  __syncwarp();
  for (int i = lane; i < total; i += 32) {
    const float d32 = sh.d[o + i];
    if (int(sh.tm[o + i].y & 255u) > Rs || !(d32 <= Bs_hi)) continue;
    const float x = d32 * scale;
    if (min(31, int(x)) != bstar) continue;
    const int sub = min(31, int((x - float(bstar)) * 32.f));
    atomicAdd(&sh.hist[sub], 1);
    atomicMax(&sh.hmax[sub], __float_as_uint(d32));
  }
  __syncwarp();
  float T;
  {
    const int c = sh.hist[lane];
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const unsigned reach = __ballot_sync(kFull, incl >= need);
    if (!reach) return false;  // cannot happen
    const int b2 = __ffs(reach) - 1;
    // buckets below bstar hold smaller values than every value of bstar
    T = __uint_as_float(__reduce_max_sync(kFull, lane <= b2 ? sh.hmax[lane] : 0u));
  }
  const float TS = fminf(__fadd_ru(T, __fmul_ru(3.f, __fmaf_ru(T, 8.f * kU32, beta_s))), Bs_hi);

  // S = shells <= R*, d32 <= TS: buffer positions compacted first, then every
  // lane recomputes its S elements in exact FP64 at once
  int nS = 0;
  for (int i0 = 0; i0 < total; i0 += 32) {
    const int i = i0 + lane;
    const bool in = i < total && int(sh.tm[o + i].y & 255u) <= Rs && sh.d[o + i] <= TS;
    const unsigned m = __ballot_sync(kFull, in);
    if (nS + __popc(m) > 32 * SN) return false;  // S larger than the row buffer
    if (in) sh.si[nS + __popc(m & lanemask_lt())] = o + i;
    nS += __popc(m);
  }
  __syncwarp();
  if (nS < k) return false;  // cannot happen: T bounds k candidates
  if (STATS && lane == 0) sh.wc[kWcRerank] += unsigned(nS);
  double ed[SN];
  int ej[SN];
#pragma unroll
  for (int h = 0; h < SN; ++h) {
    const int q = lane + 32 * h;
    ed[h] = pinf();
    ej[h] = 0x7fffffff;
    if (q < nS) {
      const int i = sh.si[q];
      ed[h] = exact(i);
      ej[h] = b.sidx[sh.tm[i].x];
      sh.sd[q] = ed[h];
      sh.sj[q] = ej[h];
    }
  }
  __syncwarp();
  // 4. rank of each element in (d2, index) order; the first k are the row.
  // Element q sits in lane q % 32, group q / 32. A group of many elements
  // counts in one pass over S, each lane for its own element; a group of a
  // few (the elements past 32 when S barely exceeds k = 32) is ranked one
  // element at a time by the whole warp: every lane compares its elements
  // with it and a warp sum adds the comparisons up. (Empty slots hold
  // (+inf, INT_MAX) and never count.)
  int rk[SN];
#pragma unroll
  for (int h = 0; h < SN; ++h) {
    rk[h] = 0;
    const int cnt = min(nS - 32 * h, 32);
    if (cnt <= 0) continue;
    if (cnt >= 16) {
      int e = 0;
      for (; e + 2 <= nS; e += 2) {
        const double d0 = sh.sd[e], d1 = sh.sd[e + 1];
        const int j0 = sh.sj[e], j1 = sh.sj[e + 1];
        rk[h] += (lex_less(d0, j0, ed[h], ej[h]) ? 1 : 0) + (lex_less(d1, j1, ed[h], ej[h]) ? 1 : 0);
      }
      if (e < nS) rk[h] += lex_less(sh.sd[e], sh.sj[e], ed[h], ej[h]) ? 1 : 0;
    } else {
      for (int q = 32 * h; q < 32 * h + cnt; ++q) {
        const double dq = sh.sd[q];
        const int jq = sh.sj[q];
        int c = 0;
#pragma unroll
        for (int g = 0; g < SN; ++g) c += lex_less(ed[g], ej[g], dq, jq) ? 1 : 0;
        const int r = int(__reduce_add_sync(kFull, unsigned(c)));
        if (lane == q - 32 * h) rk[h] = r;
      }
    }
  }
  const FrameDesc &frr = fr;
  const int i = b.sidx[p];
  int *row = b.out_nn + frr.out_base + (long long)i * k;
  double *drow = b.out_d2 ? b.out_d2 + frr.out_base + (long long)i * k : nullptr;
#pragma unroll
  for (int h = 0; h < SN; ++h) {
    if (lane + 32 * h < nS) {
      if (rk[h] == k - 1) sh.hmax[0] = __double2loint(ed[h]), sh.hmax[1] = __double2hiint(ed[h]);
      if (rk[h] == k) sh.hmax[2] = __double2loint(ed[h]), sh.hmax[3] = __double2hiint(ed[h]);
    }
  }
  __syncwarp();
  // a tie across the k-th slot: the k-th and (k+1)-th values are equal
  if (nS > k && sh.hmax[0] == sh.hmax[2] && sh.hmax[1] == sh.hmax[3]) {
    if (STATS && lane == 0) ++sh.wc[kWcReplays];
    return false;
  }
#pragma unroll
  for (int h = 0; h < SN; ++h) {
    if (lane + 32 * h < nS && rk[h] < k) {
      row[rk[h]] = ej[h];
      if (drow) drow[rk[h]] = ed[h];
    }
  }
  if (b.stop_log && lane == 0) b.stop_log[p] = int8_t(Rs);
  if (STATS && lane == 0) sh.wc[kWcInserts] += unsigned(k);
  return true;
}

// One source; false: the source must go to the literal replay. STATS: count
// the walk statistics (lc_gpu_set_stats; they cost about 3 % of the walk).
template <int SN, bool STATS, bool ONE>
__device__ bool select_source(const BatchBuffers &b, long long p, int lane, SelShared<SN> &sh,
                              const FrameDesc &fr1) {
  const int f = ONE || b.nframes == 1 ? 0 : frame_of_sorted(b, p);
  const FrameDesc &fr = ONE ? fr1 : b.frames[f];
  int Rp = b.proposal[p];
  const int k = fr.k;
  const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
  if ((b.frame_flags[f] & kFrameNaN) || Rp <= 0 || Rp > 8 || Rp > fr.max_reach || k > 16 * SN ||
      2 * Rp + 1 > nx || 2 * Rp + 1 > ny || 2 * Rp + 1 > nz)
    return false;
  const float4 r = b.rec[p];
  const int ix = __float_as_int(r.w);
  int iy, iz;
  const uint32_t yz = b.syz ? b.syz[p] : kNoYZ;
  if (yz != kNoYZ) {
    iy = int(yz & 0xFFFFu);
    iz = int(yz >> 16);
  } else {
    const uint32_t lc = b.scell[p];
    const uint32_t qy = quot(lc, uint32_t(nx), fr.inv_nx);
    const uint32_t iz_ = quot(lc, uint32_t(nx) * uint32_t(ny), fr.inv_nxy);
    iy = int(qy - iz_ * uint32_t(ny));
    iz = int(iz_);
  }
  const long long cb = fr.cell_base;
  const float plx = r.x, ply = r.y, plz = r.z;
  const float fa = fr.nhinv[0] * plx + fr.nhinv[1] * ply + fr.nhinv[2] * plz;
  const float fb = fr.nhinv[3] * plx + fr.nhinv[4] * ply + fr.nhinv[5] * plz;
  const float fc = fr.nhinv[6] * plx + fr.nhinv[7] * ply + fr.nhinv[8] * plz;
  const float ev0 = fr.ev[0], ev1 = fr.ev[1], ev2 = fr.ev[2];
  const unsigned long long pxy = f2_pack(plx, ply), exy = f2_pack(ev0, ev1);
  const int p32 = p <= 0x7fffffffLL ? int(p) : -1;  // candidate positions are ints
  // The first gather covers only rho2 = max(B(R_p - 1), q B(R_p)): every
  // candidate of the reaches below R_p, and usually the k nearest. It
  // settles R* = R_p when at least k candidates lie within rho2 (their
  // distances are then at most rho2, and everything within rho2 is here);
  // otherwise the whole ball B(R_p) is gathered again. A gather that
  // overflows the buffer starts over at R_p - 1 (any proposal gives the same
  // rows; a long one in a dense region holds more candidates than the buffer).
  int total = 0, Rs = 0;
  bool partial = false;
retry:
  for (int pass = fr.sel_rho_thr[Rp] < fr.sel_thr[Rp] ? 0 : 1; pass < 2; ++pass) {
  partial = pass == 0;
  const float thr = partial ? fr.sel_rho_thr[Rp] : fr.sel_thr[Rp];
  const float qlim = partial ? fr.sel_rho_qlim[Rp] : fr.sel_qlim[Rp];

  // 1. gather
  const int W = 2 * Rp + 1;
  const float invW = 1.f / float(W);
  const int nrow = W * W;
  total = 0;
  const unsigned lt = lanemask_lt();
  for (int r0 = 0; r0 < nrow; r0 += 32) {
    const int row = r0 + lane;
    int lenA = 0, lenB = 0, pruned = 0, startA = 0, sB = 0, wrapB = 0, wbc = 0, syz = 0;
    float Dx = 0.f, Dy = 0.f, Dz = 0.f;
    if (row < nrow) {
      const int qz = int((float(row) + 0.5f) * invW);  // exact: row < 289, W <= 17
      const int dy = row - qz * W - Rp, dz = qz - Rp;
      // row (dy, dz): offsets D_b in [dy - fb, dy + 1 - fb], D_c likewise
      const float lo1 = float(dy) - fb, lo2 = float(dz) - fc;
      const float hi1 = lo1 + 1.f, hi2 = lo2 + 1.f;
      const float gb = fmaxf(0.f, fmaxf(lo1, -hi1)), gc = fmaxf(0.f, fmaxf(lo2, -hi2));
      const float Q = qlim - (gb * gb + gc * gc);
      if (Q >= 0.f) {
        const float r01 = fr.sel_r01, r02 = fr.sel_r02;
        const float cmin = -(fmaxf(r01 * lo1, r01 * hi1) + fmaxf(r02 * lo2, r02 * hi2));
        const float cmax = -(fminf(r01 * lo1, r01 * hi1) + fminf(r02 * lo2, r02 * hi2));
        const float hm = sqrt_approx(fr.sel_ls00 * Q) * 1.0001f + 1e-4f;
        // cells dx with [dx - fa, dx + 1 - fa] meeting [cmin - hm, cmax + hm]:
        // dx <= cmax + hm + fa and dx >= cmin - hm + fa - 1 (with margins)
        const int dxh = int(floorf(fminf(cmax + hm + fa + 1e-4f, float(Rp))));
        const int dxl = -int(floorf(fminf(1.f - (cmin - hm) - fa + 1e-4f, float(Rp))));
        pruned = W - max(0, dxh - dxl + 1);
        int cy = iy + dy, wb = 0, cz = iz + dz, wc = 0;
        if (cy < 0) { cy += ny; wb = -1; } else if (cy >= ny) { cy -= ny; wb = 1; }
        if (cz < 0) { cz += nz; wc = -1; } else if (cz >= nz) { cz -= nz; wc = 1; }
        const int rowbase = (cz * ny + cy) * nx;
        const uint32_t *o = b.off + cb + rowbase;
        const int xl = ix + dxl, xh = ix + dxh;  // empty when dxl > dxh
        // the cells inside the box, then the ones across the x boundary (one
        // side only: the range spans at most 2 Rp + 1 <= nx cells)
        const int a0 = max(xl, 0), a1 = min(xh, nx - 1);
        if (a0 <= a1) {
          startA = int(o[a0]);
          lenA = int(o[a1 + 1]) - startA;
        }
        if (xl < 0 && xl <= xh) {
          const int b1 = min(xh, -1);
          sB = int(o[xl + nx]);
          lenB = int(o[b1 + nx + 1]) - sB;
          wrapB = -1;
        } else if (xh >= nx && xl <= xh) {
          const int b0 = max(xl, nx);
          sB = int(o[b0 - nx]);
          lenB = int(o[xh - nx + 1]) - sB;
          wrapB = 1;
        }
        wbc = (wb + 1) * 3 + (wc + 1);
        const float fdy = float(dy), fdz = float(dz);
        Dx = fdy * fr.ev[3] + fdz * fr.ev[6];
        Dy = fdy * fr.ev[4] + fdz * fr.ev[7];
        Dz = fdy * fr.ev[5] + fdz * fr.ev[8];
        syz = max(1, max(abs(dy), abs(dz)));
      } else {
        pruned = W;
      }
    }
    const int len = lenA + lenB;
    if (STATS) {
      const unsigned pr = __reduce_add_sync(kFull, unsigned(pruned));
      if (lane == 0) sh.wc[kWcPruned] += pr;
    }
    const unsigned hasA = __ballot_sync(kFull, lenA > 0), hasB = __ballot_sync(kFull, lenB > 0);
    if (!(hasA | hasB)) continue;
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const int tot = __shfl_sync(kFull, incl, 31);
    const int excl = incl - len;  // first candidate position of the row
    const int exclB = excl + lenA;
    if (STATS && lane == 0) sh.wc[kWcPairs] += unsigned(tot);  // the source itself included
    __syncwarp();
    {
      // the row's runs as segments, in candidate order
      const int si = __popc(hasA & lt) + __popc(hasB & lt);
      if (lenA > 0) {
        SelSeg sg;
        sg.excl = excl;
        sg.start = startA;
        sg.xoff = -ix;
        sg.meta = uint32_t(9 + wbc) << 8;
        sg.Dx = Dx, sg.Dy = Dy, sg.Dz = Dz, sg.syz = syz;
        sh.segs[si] = sg;
      }
      if (lenB > 0) {
        SelSeg sg;
        sg.excl = exclB;
        sg.start = sB;
        sg.xoff = -ix + wrapB * nx;
        sg.meta = uint32_t((wrapB + 1) * 9 + wbc) << 8;
        sg.Dx = Dx, sg.Dy = Dy, sg.Dz = Dz, sg.syz = syz;
        sh.segs[si + (lenA > 0 ? 1 : 0)] = sg;
      }
    }
    __syncwarp();
    // kSelWin 32-candidate windows per trip, so that their loads are in
    // flight together; the segment of candidate g is the last one starting
    // at or before g: one OR-reduction of the segment starts in the window
    int before = 0;  // segments that start before the window
    const unsigned le = lt | (1u << lane);
    auto starts_in = [&](int w0) -> unsigned {
      unsigned bits = 0;
      if (lenA > 0 && excl >= w0 && excl < w0 + 32) bits |= 1u << (excl - w0);
      if (lenB > 0 && exclB >= w0 && exclB < w0 + 32) bits |= 1u << (exclB - w0);
      return __reduce_or_sync(kFull, bits);
    };
    for (int g0 = 0; g0 < tot; g0 += 32 * kSelWin) {
      int owner[kSelWin];
#pragma unroll
      for (int w = 0; w < kSelWin; ++w) {
        const unsigned sw = starts_in(g0 + 32 * w);
        owner[w] = before + __popc(sw & le) - 1;
        before += __popc(sw);
      }
      int t[kSelWin];
      bool live[kSelWin];
#pragma unroll
      for (int w = 0; w < kSelWin; ++w) {
        const int g = g0 + 32 * w + lane;
        live[w] = g < tot;
        t[w] = 0;
        if (live[w]) {
          const SelSeg &S = sh.segs[owner[w]];
          t[w] = S.start + (g - S.excl);
          live[w] = t[w] != p32;
        }
      }
      float4 q[kSelWin];
#pragma unroll
      for (int w = 0; w < kSelWin; ++w)
        q[w] = live[w] ? b.rec[t[w]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int w = 0; w < kSelWin; ++w) {
        bool keep = false;
        float d32 = 0.f;
        uint32_t mm = 0;
        if (live[w]) {
          const SelSeg &S = sh.segs[owner[w]];
          const int dx = __float_as_int(q[w].w) + S.xoff;  // the candidate cell's x offset
          const float fdx = float(dx);
          float ex, ey;  // (q.x - plx) + fmaf(fdx, ev0, S.Dx), and y likewise
          offset_xy(q[w].x, q[w].y, pxy, fdx, exy, S.Dx, S.Dy, ex, ey);
          const float ez = (q[w].z - plz) + fmaf(fdx, ev2, S.Dz);
          d32 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
          keep = !(d32 > thr);
          mm = uint32_t(max(abs(dx), S.syz)) | S.meta;
        }
        const unsigned km = __ballot_sync(kFull, keep);
        const int nk = __popc(km);
        if (total + nk > kSelCap) {
          if (Rp <= 1) return false;
          --Rp;
          if (STATS && lane == 0) ++sh.wc[kWcRegather];
          __syncwarp();
          goto retry;
        }
        if (keep) {
          const int pos = total + __popc(km & lt);
          sh.d[pos] = d32;
          sh.tm[pos] = make_uint2(uint32_t(t[w]), mm);
        }
        total += nk;
      }
    }
  }
  __syncwarp();

  Rs = sel_reach<SN, STATS>(b, p, lane, sh, fr, 0, total, Rp, partial);
  if (Rs != 0) break;
  if (!partial) {
    if (STATS && lane == 0) ++sh.wc[kWcUnder];
    return false;
  }
  if (STATS && lane == 0) ++sh.wc[kWcRegather];
  __syncwarp();
  }  // gathers
  return sel_finish<SN, STATS>(b, p, lane, sh, fr, 0, total, Rs, Rp, partial);
}

// grab: consecutive sources a warp takes from the work queue at a time
// (they share most candidates, which then stay in L1).
// ONE: a single frame, passed as fr1 (read from the constant bank) instead
// of b.frames[0].
template <int SN, bool STATS, int WARPS, bool ONE>
__global__ void __launch_bounds__(WARPS * 32, sel_warps_per_sm<SN>() / WARPS)
    k_select_walk(BatchBuffers b, int grab, const __grid_constant__ FrameDesc fr1) {
  extern __shared__ __align__(16) unsigned char sel_smem[];
  SelShared<SN> &sh = reinterpret_cast<SelShared<SN> *>(sel_smem)[threadIdx.x >> 5];
  const long long total = walk_sources(b);
  const int lane = threadIdx.x & 31;
  if (lane < kWcSlots) sh.wc[lane] = 0;
  __syncwarp();
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(b.work, uint32_t(grab));
    base = __shfl_sync(kFull, base, 0);
    if ((long long)base >= total) break;
    const long long end = min(total, (long long)base + grab);
    for (long long src = base; src < end; ++src) {
      const long long p = walk_source_at(b, src);
      if (p < 0) continue;
      const unsigned long long tie = STATS ? sh.wc[kWcReplays] : 0ull;
      if (!select_source<SN, STATS, ONE>(b, p, lane, sh, fr1)) {
        if (STATS && lane == 0 && sh.wc[kWcReplays] == tie) ++sh.wc[kWcFallback];
        if (lane == 0) push_replay(b, p);
      }
      __syncwarp();
    }
  }
  if (STATS && lane == 0) {
    unsigned long long *c = reinterpret_cast<unsigned long long *>(b.counters);
    atomicAdd(&c[kCntPairs], sh.wc[kWcPairs]);
    atomicAdd(&c[kCntPruned], sh.wc[kWcPruned]);
    atomicAdd(&c[kCntRerank], sh.wc[kWcRerank]);
    atomicAdd(&c[kCntInserts], sh.wc[kWcInserts]);
    atomicAdd(&c[kCntShells], sh.wc[kWcShells]);
    atomicAdd(&c[kCntReplays], sh.wc[kWcReplays] + sh.wc[kWcFallback]);
    atomicAdd(&c[kCntPropUnder], sh.wc[kWcUnder]);
    atomicAdd(&c[kCntPropOver], sh.wc[kWcOver]);
    atomicAdd(&c[kCntPropExact], sh.wc[kWcExact]);
    atomicAdd(&c[kCntFallback], sh.wc[kWcFallback]);
    atomicAdd(&c[kCntRevisit], sh.wc[kWcRegather]);
  }
}

int sm_count();

template <int SN, bool STATS, int WARPS, bool ONE>
cudaError_t launch_select_as(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  const size_t smem = sizeof(SelShared<SN>) * WARPS;
  cudaError_t e = cudaFuncSetAttribute(k_select_walk<SN, STATS, WARPS, ONE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_select_walk<SN, STATS, WARPS, ONE>,
                                                WARPS * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = w.grid > 0 ? w.grid : sm_count() * per_sm;
  const int grab = w.grab == 8 || w.grab == 32 ? w.grab : 16;
  k_select_walk<SN, STATS, WARPS, ONE><<<grid, WARPS * 32, smem, s>>>(b, grab, w.frame1);
  return cudaGetLastError();
}

template <int SN, int WARPS>
cudaError_t launch_select_w(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  const bool one = w.one && b.nframes == 1;
  if (w.stats)
    return one ? launch_select_as<SN, true, WARPS, true>(b, w, s)
               : launch_select_as<SN, true, WARPS, false>(b, w, s);
  return one ? launch_select_as<SN, false, WARPS, true>(b, w, s)
             : launch_select_as<SN, false, WARPS, false>(b, w, s);
}

// The select walk in the block shape w.warps asks for (one of the two its S
// size allows; anything else takes the default).
template <int SN>
cudaError_t launch_select(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  constexpr int W = sel_default_warps<SN>();
  return w.warps == W / 2 ? launch_select_w<SN, W / 2>(b, w, s) : launch_select_w<SN, W>(b, w, s);
}

// Warp-parallel literal replay of the reference heap for one source (finite
// coordinates). The warp evaluates the reference visit sequence 32
// candidates at a time -- shells ascending, offsets in lexicographic order
// (src/knearest.rs:436-445), occupants in descending point index -- and
// applies KHeap::push in that order: the first k candidates fill slots 0..k-1;
// afterwards a candidate replaces the first slot holding the maximum only
// when it is strictly smaller, which is a no-op otherwise. Slots are
// distributed: slot s lives in lane s % 32, register s / 32. With finite
// values "first slot with the maximum" is the parallel argmax (largest
// value, then smallest slot), so the result is the reference's exactly.

// Offset e of shell R in the reference's lexicographic order.
__device__ __forceinline__ void lex_offset(int R, int e, int &dx, int &dy, int &dz) {
  if (R == 1) {
    dx = e / 9 - 1;
    dy = (e / 3) % 3 - 1;
    dz = e % 3 - 1;
    return;
  }
  const int w = 2 * R + 1;
  const int full = w * w, part = 8 * R;
  if (e < full) {
    dx = -R;
    dy = e / w - R;
    dz = e % w - R;
    return;
  }
  e -= full;
  if (e < (2 * R - 1) * part) {
    const int slab = e / part;
    int r = e - slab * part;
    dx = -R + 1 + slab;
    if (r < w) {
      dy = -R;
      dz = r - R;
      return;
    }
    r -= w;
    if (r < 2 * (2 * R - 1)) {
      dy = -R + 1 + r / 2;
      dz = (r & 1) ? R : -R;
      return;
    }
    r -= 2 * (2 * R - 1);
    dy = R;
    dz = r - R;
    return;
  }
  e -= (2 * R - 1) * part;
  dx = R;
  dy = e / w - R;
  dz = e % w - R;
}

template <int KPL>
struct ReplayHeap {
  double d[KPL];
  int j[KPL];
};

// First slot holding the maximum value among the n filled slots.
template <int KPL>
__device__ __forceinline__ void heap_argmax(const ReplayHeap<KPL> &H, int lane, int n, double &wmax,
                                            int &widx) {
  double bd = -pinf();
  int bs = 0x7fffffff;
#pragma unroll
  for (int r = 0; r < KPL; ++r) {
    const int slot = r * 32 + lane;
    if (slot < n && (H.d[r] > bd || (H.d[r] == bd && slot < bs))) {
      bd = H.d[r];
      bs = slot;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double od = __shfl_xor_sync(kFull, bd, o);
    const int os = __shfl_xor_sync(kFull, bs, o);
    if (od > bd || (od == bd && os < bs)) {
      bd = od;
      bs = os;
    }
  }
  wmax = bd;
  widx = bs;
}

template <int KPL>
__device__ void warp_replay(const BatchBuffers &b, const FrameDesc &fr, long long p, int lane) {
  const int k = fr.k;
  const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
  const uint32_t lc = b.scell[p];
  const int ix = int(lc % uint32_t(nx));
  const int iy = int((lc / uint32_t(nx)) % uint32_t(ny));
  const int iz = int(lc / (uint32_t(nx) * uint32_t(ny)));
  const double px = b.sx[p], py = b.sy[p], pz = b.sz[p];
  const long long cb = fr.cell_base;
  ReplayHeap<KPL> H;
#pragma unroll
  for (int r = 0; r < KPL; ++r) {
    H.d[r] = pinf();
    H.j[r] = 0x7fffffff;
  }
  int n = 0, widx = 0;
  double wmax = pinf();
  for (int R = 1; R <= fr.max_reach; ++R) {
    const bool dedupe = 2 * R + 1 > nx || 2 * R + 1 > ny || 2 * R + 1 > nz;
    const int E = R == 1 ? 27 : 24 * R * R + 2;
    for (int e0 = 0; e0 < E; e0 += 32) {
      const int e = e0 + lane;
      int a1 = 0, nc = 0, wa = 0, wb = 0, wc = 0;
      if (e < E) {
        int dx, dy, dz, cx, cy, cz;
        lex_offset(R, e, dx, dy, dz);
        wrap_axis(ix + dx, nx, cx, wa);
        wrap_axis(iy + dy, ny, cy, wb);
        wrap_axis(iz + dz, nz, cz, wc);
        const long long c = cb + ((long long)cz * ny + cy) * (long long)nx + cx;
        const int a0 = int(b.off[c]);
        a1 = int(b.off[c + 1]);
        nc = a1 - a0;
      }
      int incl = nc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
      }
      const int tot = __shfl_sync(kFull, incl, 31);
      const int excl = incl - nc;
      for (int g0 = 0; g0 < tot; g0 += 32) {
        const int g = g0 + lane;
        int owner = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int v = __shfl_sync(kFull, incl, owner + step - 1);
          if (v <= g) owner += step;
        }
        owner &= 31;
        const int oa1 = __shfl_sync(kFull, a1, owner);
        const int oex = __shfl_sync(kFull, excl, owner);
        const int owa = __shfl_sync(kFull, wa, owner);
        const int owb = __shfl_sync(kFull, wb, owner);
        const int owc = __shfl_sync(kFull, wc, owner);
        const long long t = (long long)oa1 - 1 - (g - oex);  // descending point index
        bool valid = g < tot && t != p;
        double d = 0.0;
        int j = 0;
        if (valid) {
          double shx, shy, shz;
          lattice_shift(fr, owa, owb, owc, shx, shy, shz);
          d = dist2_shifted(px, py, pz, b.sx[t], b.sy[t], b.sz[t], shx, shy, shz);
          j = b.sidx[t];
        }
        unsigned vm = __ballot_sync(kFull, valid);
        if (dedupe) {
          // index repeats possible: push one candidate at a time
          while (vm) {
            const int src = __ffs(vm) - 1;
            vm &= vm - 1;
            const double x = shfl_d(d, src);
            const int jx = __shfl_sync(kFull, j, src);
            int hit = -1;
#pragma unroll
            for (int r = 0; r < KPL; ++r) {
              const int slot = r * 32 + lane;
              const unsigned hm = __ballot_sync(kFull, slot < n && H.j[r] == jx);
              if (hm) hit = r * 32 + __ffs(hm) - 1;
            }
            if (hit >= 0) {
              const double old = shfl_d(H.d[hit >> 5], hit & 31);
              if (x < old) {
                if ((hit & 31) == lane) H.d[hit >> 5] = x;
                if (n >= k) heap_argmax(H, lane, n, wmax, widx);
              }
              continue;
            }
            if (n < k) {
              if ((n & 31) == lane) {
                H.d[n >> 5] = x;
                H.j[n >> 5] = jx;
              }
              ++n;
              if (n == k) heap_argmax(H, lane, n, wmax, widx);
              continue;
            }
            if (x < wmax) {
              if ((widx & 31) == lane) {
                H.d[widx >> 5] = x;
                H.j[widx >> 5] = jx;
              }
              heap_argmax(H, lane, n, wmax, widx);
            }
          }
          continue;
        }
        // fill: the first k - n valid candidates append in order
        if (n < k) {
          const int cntv = __popc(vm);
          const int take = min(cntv, k - n);
#pragma unroll
          for (int r = 0; r < KPL; ++r) {
            const int slot = r * 32 + lane;
            const int rank = slot - n;
            const bool mine = rank >= 0 && rank < take;
            const int src = mine ? int(__fns(vm, 0, rank + 1)) : lane;
            const double vd = shfl_d(d, src);
            const int vj = __shfl_sync(kFull, j, src);
            if (mine) {
              H.d[r] = vd;
              H.j[r] = vj;
            }
          }
          n += take;
          // drop the appended lanes: the first `take` set bits of vm
          for (int q = 0; q < take; ++q) vm &= vm - 1;
          if (n == k) heap_argmax(H, lane, n, wmax, widx);
        }
        // replacements in lane order
        while (vm) {
          const unsigned cm = __ballot_sync(kFull, ((vm >> lane) & 1u) && d < wmax);
          if (!cm) break;
          const int src = __ffs(cm) - 1;
          vm &= (src == 31) ? 0u : ~((2u << src) - 1u);  // lanes up to src are done
          const double x = shfl_d(d, src);
          const int jx = __shfl_sync(kFull, j, src);
          if ((widx & 31) == lane) {
            H.d[widx >> 5] = x;
            H.j[widx >> 5] = jx;
          }
          heap_argmax(H, lane, n, wmax, widx);
        }
      }
    }
    if (n >= k && wmax <= stop_bound(R, fr.cell_min)) break;
  }
  // KHeap::finish: ascending (total_cmp, index)
  if (KPL == 1) {
    double sdv = lane < n ? H.d[0] : pinf();
    int sjv = lane < n ? H.j[0] : 0x7fffffff;
    warp_sort_pairs(sdv, sjv, lane);
    H.d[0] = sdv;
    H.j[0] = sjv;
  } else {
    // small k-lists beyond 32: gather to lane 0 order through insertion by rank
    double rd[KPL];
    int rj[KPL];
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int slot = r * 32 + lane;
      rd[r] = slot < n ? H.d[r] : pinf();
      rj[r] = slot < n ? H.j[r] : 0x7fffffff;
    }
    // rank of every slot = number of slots ordered before it
    int rank[KPL];
#pragma unroll
    for (int r = 0; r < KPL; ++r) rank[r] = 0;
    for (int src = 0; src < 32; ++src) {
#pragma unroll
      for (int r2 = 0; r2 < KPL; ++r2) {
        const double od = shfl_d(rd[r2], src);
        const int oj = __shfl_sync(kFull, rj[r2], src);
#pragma unroll
        for (int r = 0; r < KPL; ++r) rank[r] += lex_less(od, oj, rd[r], rj[r]) ? 1 : 0;
      }
    }
    const int i = b.sidx[p];
    int *row = b.out_nn + fr.out_base + (long long)i * k;
    double *drow = b.out_d2 ? b.out_d2 + fr.out_base + (long long)i * k : nullptr;
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int slot = r * 32 + lane;
      if (slot < n) {
        row[rank[r]] = rj[r];
        if (drow) drow[rank[r]] = rd[r];
      }
    }
    for (int pos = n + lane; pos < k; pos += 32) {
      row[pos] = -1;
      if (drow) drow[pos] = qnan();
    }
    return;
  }
  const int i = b.sidx[p];
  int *row = b.out_nn + fr.out_base + (long long)i * k;
  double *drow = b.out_d2 ? b.out_d2 + fr.out_base + (long long)i * k : nullptr;
  if (lane < k) {
    const bool ok = lane < n;
    row[lane] = ok ? H.j[0] : -1;
    if (drow) drow[lane] = ok ? H.d[0] : qnan();
  }
}

// ONE: a single frame, passed as fr1 (read from the constant bank).
// Blocks per SM of the literal replay: 16 at 64 registers; 11 at 80 for
// k-lists past 128 (KPL = 8), which would spill more at 64.
template <int KPL>
constexpr int replay_blocks_per_sm() { return KPL >= 8 ? 11 : 16; }

template <int KPL, bool ONE>
__global__ void __launch_bounds__(64, replay_blocks_per_sm<KPL>())
    k_replay_warp(BatchBuffers b, const __grid_constant__ FrameDesc fr1) {
  long long cnt = *b.replay_count;
  if (cnt > b.replay_cap) cnt = b.replay_cap;
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long q = warp; q < cnt; q += nwarps) {
    const long long p = b.replay_list[q];
    const int f = ONE || b.nframes == 1 ? 0 : frame_of_sorted(b, p);
    const FrameDesc &fr = ONE ? fr1 : b.frames[f];
    if ((b.frame_flags[f] & kFrameNaN) || fr.k > 32 * KPL) {
      // NaN comparisons follow the reference's sequential scans: one thread
      if (lane == 0 && warp < b.replay_threads) {
        double *hd = b.replay_d + warp * b.kmax;
        int *hi = b.replay_i + warp * b.kmax;
        const int m = replay_walk(b, fr, p, hd, hi, 1);
        write_row(b, fr, b.sidx[p], hd, hi, 1, m);
      }
      __syncwarp();
      continue;
    }
    warp_replay<KPL>(b, fr, p, lane);
    __syncwarp();
  }
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <int MODE, int KPL>
cudaError_t launch_team(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_team_walk<MODE, KPL>, 256, 0);
  if (per_sm < 1) per_sm = 1;
  const int grid = w.grid > 0 ? w.grid : sm_count() * per_sm;
  k_team_walk<MODE, KPL><<<grid, 256, 0, s>>>(b);
  return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_team_k(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  if (b.kmax <= 32) return launch_team<MODE, 1>(b, w, s);
  if (b.kmax <= 64) return launch_team<MODE, 2>(b, w, s);
  if (b.kmax <= 128) return launch_team<MODE, 4>(b, w, s);
  return launch_team<MODE, 8>(b, w, s);
}

template <int MODE, int BLOCK>
cudaError_t launch_mode(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  const size_t sm = walk_smem_bytes(MODE, BLOCK, b.kmax);
  cudaError_t e = cudaFuncSetAttribute(k_walk<MODE, BLOCK>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess) return e;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk<MODE, BLOCK>, BLOCK, sm);
  if (per_sm < 1) per_sm = 1;
  const int grid = w.grid > 0 ? w.grid : sm_count() * per_sm;
  k_walk<MODE, BLOCK><<<grid, BLOCK, sm, s>>>(b);
  return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_block(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  switch (w.block) {
    case 32: return launch_mode<MODE, 32>(b, w, s);
    case 64: return launch_mode<MODE, 64>(b, w, s);
    case 128: return launch_mode<MODE, 128>(b, w, s);
    case 256: return launch_mode<MODE, 256>(b, w, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

size_t walk_smem_bytes(int mode, int block, int kmax) {
  (void)mode;
  return size_t(block) * size_t(kmax) * (sizeof(double) + sizeof(int));
}

int walk_max_block(int mode, int kmax) {
  // keep the heap under ~100 KB per block so two blocks share an SM
  const size_t budget = 100 * 1024;
  int blk = 256;
  while (blk > 32 && walk_smem_bytes(mode, blk, kmax) > budget) blk >>= 1;
  return blk;
}

cudaError_t launch_walk(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  if (w.mode == kModeReplayAll) {
    k_queue_all<<<sm_count() * 4, 256, 0, s>>>(b);
    return cudaGetLastError();
  }
  if (w.tpp == 32 && w.mode == kModeLearned && b.kmax <= 64 && b.proposal)
    return b.kmax <= 32 ? launch_select<2>(b, w, s) : launch_select<4>(b, w, s);
  if (w.tpp == 32 && b.kmax <= 256) {
    switch (w.mode) {
      case kModeFastF32: return launch_team_k<kModeFastF32>(b, w, s);
      case kModeLearned: return launch_team_k<kModeLearned>(b, w, s);
      default: return launch_team_k<kModePlainF64>(b, w, s);
    }
  }
  switch (w.mode) {
    case kModeFastF32: return launch_block<kModeFastF32>(b, w, s);
    case kModeLearned: return launch_block<kModeLearned>(b, w, s);
    default: return launch_block<kModePlainF64>(b, w, s);
  }
}

namespace {
constexpr int kPartBlock = 256, kPartItems = 8;  // a block partitions 2048 sorted positions

// Row range of sorted position p: its output row (point units) against the cuts.
__device__ __forceinline__ int range_of(const BatchBuffers &b, const RowCuts &rc, long long p) {
  const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
  const long long row = b.frames[f].pt_base + b.sidx[p];
  int r = 0;
#pragma unroll
  for (int c = 1; c < kMaxRowRanges; ++c) r += (c < rc.nr && row >= rc.cut[c]) ? 1 : 0;
  return r;
}

// Per block and range: how many of the block's sorted positions fall in the
// range (range-major, so that one scan gives every block's stable offsets).
__global__ void __launch_bounds__(kPartBlock)
    k_part_count(BatchBuffers b, RowCuts rc, uint32_t *__restrict__ cnt, int nblk) {
  __shared__ uint32_t s_cnt[kMaxRowRanges];
  if (threadIdx.x < kMaxRowRanges) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const long long total = b.off[b.ncells];
  const long long base = (long long)blockIdx.x * kPartBlock * kPartItems;
#pragma unroll
  for (int i = 0; i < kPartItems; ++i) {
    const long long p = base + i * kPartBlock + threadIdx.x;
    if (p < total) atomicAdd(&s_cnt[range_of(b, rc, p)], 1u);
  }
  __syncthreads();
  if (threadIdx.x < rc.nr) cnt[(long long)threadIdx.x * nblk + blockIdx.x] = s_cnt[threadIdx.x];
}

// Stable scatter: positions in ascending order within each range.
__global__ void __launch_bounds__(kPartBlock)
    k_part_scatter(BatchBuffers b, RowCuts rc, const uint32_t *__restrict__ off, int nblk,
                   int *__restrict__ order) {
  constexpr int kWarps = kPartBlock / 32;
  __shared__ uint32_t s_run[kMaxRowRanges];
  __shared__ uint32_t s_w[kWarps][kMaxRowRanges];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < kMaxRowRanges) s_run[threadIdx.x] = 0;
  const long long total = b.off[b.ncells];
  const long long base = (long long)blockIdx.x * kPartBlock * kPartItems;
  unsigned lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  for (int i = 0; i < kPartItems; ++i) {
    const long long p = base + i * kPartBlock + threadIdx.x;
    const int r = p < total ? range_of(b, rc, p) : -1;
    int rank = 0;
    for (int c = 0; c < rc.nr; ++c) {
      const unsigned m = __ballot_sync(0xffffffffu, r == c);
      if (r == c) rank = __popc(m & lt);
      if (lane == 0) s_w[warp][c] = __popc(m);
    }
    __syncthreads();
    if (r >= 0) {
      uint32_t pos = off[(long long)r * nblk + blockIdx.x] + s_run[r] + uint32_t(rank);
      for (int w = 0; w < warp; ++w) pos += s_w[w][r];
      order[pos] = int(p);
    }
    __syncthreads();
    if (threadIdx.x < rc.nr) {
      uint32_t add = 0;
      for (int w = 0; w < kWarps; ++w) add += s_w[w][threadIdx.x];
      s_run[threadIdx.x] += add;
    }
    __syncthreads();
  }
}

// ---- a search split across ranks (one process per GPU, inputs replicated)
// Expected work of sorted source p: its cell's occupancy times its proposed
// cube in units of the 3x3x3 cube (shell 2 without a proposal), plus one,
// capped so that the prefix over all sources fits 32 bits; zero past the
// active sources.
__global__ void k_shard_weights(BatchBuffers b, uint32_t *__restrict__ w, uint32_t cap) {
  const long long total = b.off[b.ncells];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < b.npts;
       p += (long long)gridDim.x * blockDim.x) {
    uint32_t v = 0;
    if (p < total) {
      const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
      const long long c = b.frames[f].cell_base + (long long)b.scell[p];
      const uint32_t occ = min(b.off[c + 1] - b.off[c], 64u);
      int R = b.proposal ? int(b.proposal[p]) : 2;
      R = R <= 0 ? 2 : min(R, 8);
      const uint32_t cube = uint32_t((2 * R + 1) * (2 * R + 1) * (2 * R + 1));
      v = 1u + min(cap - 1u, occ * cube / 27u);
    }
    w[p] = v;
  }
}

// cut = this rank's [lo, hi): lo is the first sorted position whose prefix
// weight reaches rank / world of the total (hi likewise for rank + 1), so
// consecutive ranks' ranges meet and together cover every active source.
__global__ void k_shard_cut(BatchBuffers b, const uint32_t *__restrict__ pre, int rank, int world,
                            uint32_t *__restrict__ cut) {
  if (threadIdx.x > 1) return;
  const long long total = b.off[b.ncells];
  const unsigned long long W = pre[b.npts];
  const int r = rank + int(threadIdx.x);
  if (r >= world) {
    cut[1] = uint32_t(total);
    return;
  }
  const unsigned long long target = W * (unsigned long long)r / (unsigned long long)world;
  long long lo = 0, hi = total;  // first p in [0, total] with pre[p] >= target
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if ((unsigned long long)pre[mid] >= target)
      hi = mid;
    else
      lo = mid + 1;
  }
  cut[threadIdx.x] = uint32_t(lo);
}

__global__ void k_shard_owned(BatchBuffers b, const uint32_t *__restrict__ cut, int rank,
                              int *__restrict__ owned) {
  const long long lo = cut[0], hi = cut[1];
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < hi; p += stride) {
    const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
    owned[b.frames[f].pt_base + b.sidx[p]] = 1;
  }
  if (rank == 0)
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < b.npts; i += stride)
      if (b.cell_of[i] == kInactive) owned[i] = 1;
}
}  // namespace

cudaError_t launch_shard_split(const BatchBuffers &b, int rank, int world, uint32_t *w,
                               uint32_t *pre, unsigned long long *tile_state,
                               uint32_t *tile_counter, uint32_t *cut, cudaStream_t s) {
  if (world < 1 || rank < 0 || rank >= world || b.npts <= 0) return cudaErrorInvalidValue;
  const unsigned long long per = 0xFFFFFFFFull / (unsigned long long)b.npts;
  const uint32_t cap = uint32_t(per < 1 ? 1 : (per > 64 ? 64 : per));
  const int g = int(std::min<long long>((b.npts + 255) / 256, (long long)sm_count() * 8));
  k_shard_weights<<<g, 256, 0, s>>>(b, w, cap);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  BatchBuffers sb;  // prefix of the weights over the sorted positions
  sb.count = w;
  sb.off = pre;
  sb.ncells = b.npts;
  sb.tile_state = tile_state;
  sb.tile_counter = tile_counter;
  sb.status = b.status;
  if ((e = cudaMemsetAsync(tile_state, 0, size_t(scan_tiles(sb.ncells)) * sizeof(unsigned long long),
                           s)) != cudaSuccess ||
      (e = cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), s)) != cudaSuccess)
    return e;
  if ((e = launch_scan(sb, s)) != cudaSuccess) return e;
  k_shard_cut<<<1, 32, 0, s>>>(b, pre, rank, world, cut);
  return cudaGetLastError();
}

cudaError_t launch_shard_owned(const BatchBuffers &b, const uint32_t *cut, int rank, int *owned,
                               cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(owned, 0, size_t(b.npts) * sizeof(int), s);
  if (e != cudaSuccess) return e;
  const int g = int(std::min<long long>((b.npts + 255) / 256, (long long)sm_count() * 8));
  k_shard_owned<<<g, 256, 0, s>>>(b, cut, rank, owned);
  return cudaGetLastError();
}

long long range_partition_blocks(long long sources) {
  const long long per = (long long)kPartBlock * kPartItems;
  return std::max<long long>(1, (sources + per - 1) / per);
}

cudaError_t launch_range_partition(const BatchBuffers &b, const RowCuts &cuts, uint32_t *cnt,
                                   uint32_t *off, unsigned long long *tile_state,
                                   uint32_t *tile_counter, int *order, cudaStream_t s) {
  // b.npts bounds the active sources: the grid covers them all
  const int nblk = int(range_partition_blocks(b.npts));
  k_part_count<<<nblk, kPartBlock, 0, s>>>(b, cuts, cnt, nblk);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  BatchBuffers sb;  // the cell-count scan over the range-major block counts
  sb.count = cnt;
  sb.off = off;
  sb.ncells = (long long)cuts.nr * nblk;
  sb.tile_state = tile_state;
  sb.tile_counter = tile_counter;
  sb.status = b.status;
  if ((e = cudaMemsetAsync(tile_state, 0, size_t(scan_tiles(sb.ncells)) * sizeof(unsigned long long),
                           s)) != cudaSuccess ||
      (e = cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), s)) != cudaSuccess)
    return e;
  if ((e = launch_scan(sb, s)) != cudaSuccess) return e;
  k_part_scatter<<<nblk, kPartBlock, 0, s>>>(b, cuts, off, nblk, order);
  return cudaGetLastError();
}

template <int KPL>
void launch_replay_kpl(const BatchBuffers &b, int grid, const FrameDesc *one, cudaStream_t s) {
  if (one && b.nframes == 1)
    k_replay_warp<KPL, true><<<grid, 64, 0, s>>>(b, *one);
  else
    k_replay_warp<KPL, false><<<grid, 64, 0, s>>>(b, FrameDesc{});
}

cudaError_t launch_replay(const BatchBuffers &b, cudaStream_t s, const FrameDesc *one) {
  if (b.replay_threads <= 0) return cudaSuccess;
  if (b.kmax <= 256) {
    // one warp per queued source; NaN frames take one thread of the warp
    // 2-warp blocks, 16 per SM at 64 registers: the replay is bound by
    // latency, so more warps (4M: 0.29 -> 0.25 ms at k = 32 against 11 per SM
    // at 80 registers, 0.69 -> 0.58 ms at k = 64)
    const int per_sm = b.kmax <= 128 ? replay_blocks_per_sm<4>() : replay_blocks_per_sm<8>();
    const int warps = std::max(1, std::min(b.replay_threads, sm_count() * 2 * per_sm));
    const int grid = (warps + 1) / 2;
    if (b.kmax <= 32)
      launch_replay_kpl<1>(b, grid, one, s);
    else if (b.kmax <= 64)
      launch_replay_kpl<2>(b, grid, one, s);
    else if (b.kmax <= 128)
      launch_replay_kpl<4>(b, grid, one, s);
    else
      launch_replay_kpl<8>(b, grid, one, s);
    return cudaGetLastError();
  }
  const int block = 128;
  const int grid = (b.replay_threads + block - 1) / block;
  k_replay<<<grid, block, 0, s>>>(b);
  return cudaGetLastError();
}

}  // namespace lc

namespace lc {

// Offsets of shells 1..rmax, each shell sorted near-first by |d|^2 in bin
// units (ties by lexicographic order). Shell 1 (the whole 3x3x3 cube)
// occupies [0, 27), shell R > 1 [(2R-1)^3, (2R+1)^3); the walk's result
// does not depend on this order.
void build_shell_table(int rmax, uint32_t *out) {
  size_t o = 0;
  for (int R = 1; R <= rmax; ++R) {
    struct Off {
      int d2, dx, dy, dz;
    };
    std::vector<Off> v;
    for (int dx = -R; dx <= R; ++dx)
      for (int dy = -R; dy <= R; ++dy)
        for (int dz = -R; dz <= R; ++dz) {
          const int m = std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz)));
          if (m != R && !(R == 1 && m == 0)) continue;
          v.push_back({dx * dx + dy * dy + dz * dz, dx, dy, dz});
        }
    std::stable_sort(v.begin(), v.end(), [](const Off &a, const Off &b) { return a.d2 < b.d2; });
    for (const Off &x : v)
      out[o++] = uint32_t(x.dx + 512) | (uint32_t(x.dy + 512) << 10) | (uint32_t(x.dz + 512) << 20);
  }
}

}  // namespace lc
