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
// The walk below detects that case (a rejected or evicted value equal to
// the final k-th value) and sends the source to k_replay, which re-runs the
// reference push sequence literally: shells ascending, offsets in
// lexicographic order, occupants in descending point index.
#include <cuda/atomic>

#include "lc_kernels.h"

namespace lc {

namespace {

constexpr unsigned kFull = 0xffffffffu;

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

// Max-heap of (d, idx) in shared memory, one slot every S words.
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
  long long pairs = 0, inserts = 0, shells = 0, replays = 0, pruned = 0;
};

__device__ __forceinline__ void flush_counters(const BatchBuffers &b, LocalCounters &c) {
  long long v[5] = {c.pairs, c.inserts, c.shells, c.replays, c.pruned};
  const int slot[5] = {kCntPairs, kCntInserts, kCntShells, kCntReplays, kCntPruned};
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    long long x = v[t];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(kFull, x, d);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd((unsigned long long *)&b.counters[slot[t]],
                                                 (unsigned long long)x);
  }
}

// ------------------------------------------------------------------------
// Plain FP64 walk: one thread per source, shells in order, exact stop rule.
__device__ void walk_source_f64(const BatchBuffers &b, long long p, double *hd, int *hi, int S,
                                LocalCounters &cnt) {
  const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
  const FrameDesc &fr = b.frames[f];
  if (b.frame_flags[f] & kFrameNaN) {
    push_replay(b, p);
    ++cnt.replays;
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
  int n = 0;
  double rej = __longlong_as_double(0x7ff0000000000000ll);  // +inf
  const int max_reach = fr.max_reach;
  for (int R = 1; R <= max_reach; ++R) {
    const bool dedupe = 2 * R + 1 > nx || 2 * R + 1 > ny || 2 * R + 1 > nz;
    ++cnt.shells;
    for_each_shell_offset(R, [&](int dx, int dy, int dz) {
      int cx, cy, cz, wa, wb, wc;
      wrap_axis(ix + dx, nx, cx, wa);
      wrap_axis(iy + dy, ny, cy, wb);
      wrap_axis(iz + dz, nz, cz, wc);
      const long long c = cb + ((long long)cz * ny + cy) * (long long)nx + cx;
      const uint32_t a0 = off[c], a1 = off[c + 1];
      if (a0 == a1) return;
      double shx, shy, shz;
      lattice_shift(fr, wa, wb, wc, shx, shy, shz);
      for (uint32_t t = a0; t < a1; ++t) {
        if ((long long)t == p) continue;
        const double d = dist2_shifted(px, py, pz, b.sx[t], b.sy[t], b.sz[t], shx, shy, shz);
        ++cnt.pairs;
        if (dedupe) {
          const int j = b.sidx[t];
          int s = 0;
          for (; s < n; ++s)
            if (hi[s * S] == j) break;
          if (s < n) {
            if (d < hd[s * S]) {
              hd[s * S] = d;
              if (n >= k) heap_sift_down(hd, hi, S, s, n);
            }
            continue;
          }
        }
        if (n < k) {
          hd[n * S] = d;
          hi[n * S] = b.sidx[t];
          ++n;
          ++cnt.inserts;
          if (n == k) heap_build(hd, hi, S, n);
        } else if (d < hd[0]) {
          rej = fmin(rej, hd[0]);
          hd[0] = d;
          hi[0] = b.sidx[t];
          heap_sift_down(hd, hi, S, 0, n);
          ++cnt.inserts;
        } else {
          rej = fmin(rej, d);
        }
      }
    });
    if (n >= k && hd[0] <= stop_bound(R, fr.cell_min)) break;
  }
  if (n >= k && !(rej > hd[0])) {
    // a value equal to the k-th was left out: the kept subset of the tie
    // depends on the reference push order
    push_replay(b, p);
    ++cnt.replays;
    return;
  }
  if (n < k) heap_build(hd, hi, S, n);
  heap_sort(hd, hi, S, n);
  write_row(b, fr, b.sidx[p], hd, hi, S, n);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_walk_f64(BatchBuffers b) {
  extern __shared__ double smem[];
  double *hd = smem + threadIdx.x;
  int *hi = reinterpret_cast<int *>(smem + (size_t)b.kmax * BLOCK) + threadIdx.x;
  const long long total = b.off[b.ncells];
  const int lane = threadIdx.x & 31;
  LocalCounters cnt;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(b.work, 32u);
    base = __shfl_sync(kFull, base, 0);
    if ((long long)base >= total) break;
    const long long p = (long long)base + lane;
    if (p < total) walk_source_f64(b, p, hd, hi, BLOCK, cnt);
    __syncwarp();
  }
  flush_counters(b, cnt);
}

// ------------------------------------------------------------------------
// Exact replay of the reference push sequence for one source.
__device__ void replay_source(const BatchBuffers &b, long long p, double *hd, int *hi) {
  const int f = b.nframes == 1 ? 0 : frame_of_sorted(b, p);
  const FrameDesc &fr = b.frames[f];
  const int k = fr.k;
  const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
  const uint32_t lc = b.scell[p];
  const int ix = int(lc % uint32_t(nx));
  const int iy = int((lc / uint32_t(nx)) % uint32_t(ny));
  const int iz = int(lc / (uint32_t(nx) * uint32_t(ny)));
  const double px = b.sx[p], py = b.sy[p], pz = b.sz[p];
  const long long cb = fr.cell_base;
  int n = 0;
  for (int R = 1; R <= fr.max_reach; ++R) {
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
        // KHeap::push, src/knearest.rs:106-129
        int s = 0;
        for (; s < n; ++s)
          if (hi[s] == j) break;
        if (s < n) {
          if (d < hd[s]) hd[s] = d;
          continue;
        }
        if (n < k) {
          hd[n] = d;
          hi[n] = j;
          ++n;
          continue;
        }
        int w = 0;
        for (int u = 1; u < n; ++u)
          if (hd[u] > hd[w]) w = u;
        if (d < hd[w]) {
          hd[w] = d;
          hi[w] = j;
        }
      }
    });
    if (n >= k) {
      double worst = hd[0];
      for (int u = 1; u < n; ++u)
        if (hd[u] > worst) worst = hd[u];
      if (worst <= stop_bound(R, fr.cell_min)) break;
    }
  }
  // KHeap::finish: sort by (total_cmp, idx), src/knearest.rs:146-158
  for (int a = 1; a < n; ++a) {
    const double kd = hd[a];
    const int ki = hi[a];
    const long long kk = total_key(kd);
    int q = a;
    while (q > 0) {
      const long long pk = total_key(hd[q - 1]);
      if (pk > kk || (pk == kk && hi[q - 1] > ki)) {
        hd[q] = hd[q - 1];
        hi[q] = hi[q - 1];
        --q;
      } else {
        break;
      }
    }
    hd[q] = kd;
    hi[q] = ki;
  }
  write_row(b, fr, b.sidx[p], hd, hi, 1, n);
}

__global__ void __launch_bounds__(128) k_replay(BatchBuffers b) {
  long long cnt = *b.replay_count;
  if (cnt > b.replay_cap) cnt = b.replay_cap;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= b.replay_threads) return;
  double *hd = b.replay_d + tid * b.kmax;
  int *hi = b.replay_i + tid * b.kmax;
  for (long long q = tid; q < cnt; q += b.replay_threads) replay_source(b, b.replay_list[q], hd, hi);
}

// Every source of the batch through the exact replay (large k, or on request).
__global__ void k_queue_all(BatchBuffers b) {
  const long long total = b.off[b.ncells];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < total;
       p += (long long)gridDim.x * blockDim.x)
    b.replay_list[p] = int(p);
  if (blockIdx.x == 0 && threadIdx.x == 0) *b.replay_count = uint32_t(total);
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <int BLOCK>
cudaError_t launch_f64(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s) {
  const size_t sm = walk_smem_bytes(w.mode, BLOCK, b.kmax);
  cudaError_t e = cudaFuncSetAttribute(k_walk_f64<BLOCK>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess) return e;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_f64<BLOCK>, BLOCK, sm);
  if (per_sm < 1) per_sm = 1;
  const int grid = w.grid > 0 ? w.grid : sm_count() * per_sm;
  k_walk_f64<BLOCK><<<grid, BLOCK, sm, s>>>(b);
  return cudaGetLastError();
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
  switch (w.block) {
    case 32: return launch_f64<32>(b, w, s);
    case 64: return launch_f64<64>(b, w, s);
    case 128: return launch_f64<128>(b, w, s);
    case 256: return launch_f64<256>(b, w, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_replay(const BatchBuffers &b, cudaStream_t s) {
  if (b.replay_threads <= 0) return cudaSuccess;
  const int block = 128;
  const int grid = (b.replay_threads + block - 1) / block;
  k_replay<<<grid, block, 0, s>>>(b);
  return cudaGetLastError();
}

}  // namespace lc
