// Fold, bin, histogram, scan and stable cell-sorted placement (sm_100a).
//
// These are the HBM-bound stages in front of the walk. They replace the
// fold/bin and linked-list build of the reference search
// (src/knearest.rs:399-428). The reference keeps a per-cell linked list
// that it traverses in descending point index. Here the points are stored
// cell-major in SoA arrays, ascending by point index inside each cell, so a
// cell is one contiguous range of the sorted arrays.
#include <cuda/atomic>

#include <algorithm>

#include "lc_kernels.h"

namespace lc {

namespace {

__device__ __forceinline__ int frame_of_point(const FrameDesc *__restrict__ fr, int nf,
                                              long long g) {
  int lo = 0, hi = nf - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (fr[mid].pt_base <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// fold + bin + histogram: grid-stride over points, two per thread per trip
// (their coordinate loads and histogram atomics in flight together). ONE: a
// single frame, passed as fr1 (read from the constant bank).
template <bool ONE>
__global__ void __launch_bounds__(256)
    k_fold_bin(const double *__restrict__ xyz, const int *__restrict__ mask,
               const FrameDesc *__restrict__ frames, int nframes, long long npts,
               uint32_t *__restrict__ cell_of, uint32_t *__restrict__ arank,
               uint32_t *__restrict__ count, int *__restrict__ frame_flags,
               const __grid_constant__ FrameDesc fr1) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long g0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; g0 < npts;
       g0 += 2 * stride) {
    const long long gg[2] = {g0, g0 + stride};
    double r[2][3];
    bool act[2];
    int fi[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const long long g = gg[u];
      act[u] = g < npts;
      fi[u] = 0;
      if (!act[u]) continue;
      fi[u] = ONE || nframes == 1 ? 0 : frame_of_point(frames, nframes, g);
      const FrameDesc &fr = ONE ? fr1 : frames[fi[u]];
      if (fr.dead || (fr.has_mask && mask[fr.mask_base + (g - fr.pt_base)] == 0)) {
        cell_of[g] = kInactive;
        act[u] = false;
        continue;
      }
      r[u][0] = xyz[3 * g + 0];
      r[u][1] = xyz[3 * g + 1];
      r[u][2] = xyz[3 * g + 2];
    }
    uint32_t c[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      c[u] = 0;
      if (!act[u]) continue;
      const FrameDesc &fr = ONE ? fr1 : frames[fi[u]];
      double s0, s1, s2;
      fractional(fr, r[u][0], r[u][1], r[u][2], s0, s1, s2);
      if (s0 != s0 || s1 != s1 || s2 != s2) atomicOr(&frame_flags[fi[u]], kFrameNaN);
      const int cx = bin_of(s0, fr.nx);
      const int cy = bin_of(s1, fr.ny);
      const int cz = bin_of(s2, fr.nz);
      c[u] = uint32_t(fr.cell_base + ((long long)cz * fr.ny + cy) * (long long)fr.nx + cx);
    }
    uint32_t rk[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) rk[u] = act[u] ? atomicAdd(&count[c[u]], 1u) : 0u;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (!act[u]) continue;
      cell_of[gg[u]] = c[u];
      arank[gg[u]] = rk[u];
    }
  }
}

// ---------------------------------------------------------------- scan
// Single-pass exclusive scan with decoupled look-back (Merrill & Garland).
// Tile ids come from an atomic counter in launch order, so a tile only ever
// waits on tiles that have already started; every wait is still bounded
// (spin_limit loads, kSpinLimit when it is 0) and reports kStatusScanTimeout
// instead of hanging. A tile whose wait runs out sums its exclusive prefix
// straight from the counts of the cells before it, so the offsets stay right
// and no later kernel reads past its buffers. silent_tile >= 0 keeps that
// tile from publishing its state, so that its successor's wait runs out: a
// failure-detection test hook (lc_gpu_set_scan_limit), -1 in searches.
constexpr unsigned long long kFlagA = 1ull << 62;  // aggregate published
constexpr unsigned long long kFlagP = 2ull << 62;  // inclusive prefix published
constexpr unsigned long long kValMask = (1ull << 62) - 1;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ unsigned long long load_acquire(unsigned long long *p) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*p);
  return r.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void store_release(unsigned long long *p, unsigned long long v) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*p);
  r.store(v, cuda::memory_order_release);
}

// ncells is the size of the cell arrays. With live set, only the first
// *live cells are in use (a device-planned batch, whose mesh the host never
// reads): the scan covers those and also writes the total to off[ncells],
// where every consumer reads it. Blocks take tiles until none are left, so
// a grid smaller than the tile count is fine.
__global__ void __launch_bounds__(kScanBlock)
    k_scan_cells(const uint32_t *__restrict__ count, uint32_t *__restrict__ off, long long ncells,
                 const long long *__restrict__ live, unsigned long long *__restrict__ tile_state,
                 uint32_t *__restrict__ tile_counter, int *__restrict__ status, int spin_limit,
                 long long silent_tile) {
  const int limit = spin_limit > 0 ? spin_limit : kSpinLimit;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kScanBlock / 32];
  __shared__ unsigned long long s_excl;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long nlive = live ? *live : ncells;
  const long long ntiles = (nlive + kScanTile - 1) / kScanTile;
  for (;;) {
    __syncthreads();  // the previous tile's shared values are consumed
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= ntiles) return;
    const long long base = tile * kScanTile + (long long)tid * kScanItems;
    uint32_t v[kScanItems];
    if (base + kScanItems <= nlive) {
      const uint4 *src = reinterpret_cast<const uint4 *>(count + base);
#pragma unroll
      for (int m = 0; m < kScanItems / 4; ++m) {
        const uint4 a = src[m];
        v[4 * m + 0] = a.x; v[4 * m + 1] = a.y; v[4 * m + 2] = a.z; v[4 * m + 3] = a.w;
      }
    } else {
#pragma unroll
      for (int m = 0; m < kScanItems; ++m) v[m] = (base + m < nlive) ? count[base + m] : 0u;
    }
    uint32_t tsum = 0;
#pragma unroll
    for (int m = 0; m < kScanItems; ++m) tsum += v[m];
    // inclusive warp scan of thread sums
    uint32_t x = tsum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < kScanBlock / 32 ? s_warp[lane] : 0u;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
        if (lane >= d) w += y;
      }
      if (lane < kScanBlock / 32) s_warp[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const uint32_t agg = s_warp[kScanBlock / 32 - 1];
    const uint32_t texcl = (warp ? s_warp[warp - 1] : 0u) + x - tsum;

    if (warp == 0) {
      // publish this tile's aggregate, then look back 32 predecessors at a time
      const bool publish = tile != silent_tile;
      if (lane == 0 && publish) store_release(&tile_state[tile], (tile == 0 ? kFlagP : kFlagA) | agg);
      unsigned long long excl = 0;
      if (tile > 0) {
        long long end = tile;  // predecessors [end-32, end)
        bool done = false, timeout = false;
        while (!done && !timeout) {
          const long long t = end - 1 - lane;
          unsigned long long w = kFlagP;  // before tile 0: an empty prefix
          if (t >= 0) {
            int spins = 0;
            w = load_acquire(&tile_state[t]);
            while ((w >> 62) == 0 && spins < limit) {
              ++spins;
              w = load_acquire(&tile_state[t]);
            }
          }
          const unsigned invalid = __ballot_sync(0xffffffffu, (w >> 62) == 0);
          if (invalid) {
            timeout = true;
            break;
          }
          const unsigned pm = __ballot_sync(0xffffffffu, (w >> 62) == 2);
          const int stop = pm ? (__ffs(pm) - 1) : 31;
          unsigned long long val = (lane <= stop) ? (w & kValMask) : 0ull;
#pragma unroll
          for (int d = 16; d > 0; d >>= 1) val += __shfl_xor_sync(0xffffffffu, val, d);
          excl += val;
          if (pm) done = true;
          end -= 32;
        }
        if (timeout) {
          // the counts are final (the histogram kernel has finished): sum them
          unsigned long long sum = 0;
          for (long long c = lane; c < tile * kScanTile; c += 32) sum += count[c];
#pragma unroll
          for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
          excl = sum;
          if (lane == 0) atomicOr(status, kStatusScanTimeout);
        }
        if (lane == 0 && publish)
          store_release(&tile_state[tile], kFlagP | ((excl + agg) & kValMask));
      }
      if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    uint32_t run = uint32_t(s_excl) + texcl;
    if (base + kScanItems <= nlive) {
      uint32_t o[kScanItems];
#pragma unroll
      for (int m = 0; m < kScanItems; ++m) {
        o[m] = run;
        run += v[m];
      }
      uint4 *dst = reinterpret_cast<uint4 *>(off + base);
#pragma unroll
      for (int m = 0; m < kScanItems / 4; ++m)
        dst[m] = make_uint4(o[4 * m + 0], o[4 * m + 1], o[4 * m + 2], o[4 * m + 3]);
    } else {
#pragma unroll
      for (int m = 0; m < kScanItems; ++m) {
        if (base + m < nlive) off[base + m] = run;
        run += v[m];
      }
    }
    // the thread that owns the last cell also writes the total
    if (base <= nlive - 1 && nlive - 1 < base + kScanItems) {
      off[nlive] = run;
      if (nlive != ncells) off[ncells] = run;
    }
  }
}

// Zeroes the cell counts and scan tile states of a device-planned batch
// (its first *live cells).
__global__ void k_zero_live(uint32_t *__restrict__ count, unsigned long long *__restrict__ tile_state,
                            const long long *__restrict__ live) {
  const long long n = *live, tiles = (n + kScanTile - 1) / kScanTile;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    count[i] = 0u;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += stride)
    tile_state[t] = 0ull;
}

// Arrival slots: tmp[off[c] + arank[g]] = (g, c, folded coordinates of g).
// The coordinates are read here in point order (coalesced) and folded
// again (the same fractional / cartesian expressions as the bin), so the
// stable placement after this reads its slots as one stream and gathers
// nothing by point id. The output rows of masked points are filled here
// with -1 / NaN (src/knearest.rs:293-296). Two points per thread per trip:
// their loads, and then their dependent cell-offset loads, are in flight
// together. ONE: a single frame, passed as fr1.
template <bool ONE>
__global__ void __launch_bounds__(256)
    k_place_slots(const double *__restrict__ xyz, const FrameDesc *__restrict__ frames,
                  int nframes, const uint32_t *__restrict__ cell_of,
                  const uint32_t *__restrict__ arank, const uint32_t *__restrict__ off,
                  PlaceSlot *__restrict__ tmp, long long npts, long long ncells,
                  int *__restrict__ out_nn, double *__restrict__ out_d2, int *__restrict__ status,
                  const __grid_constant__ FrameDesc fr1) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long total = off[ncells];
  for (long long g0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; g0 < npts;
       g0 += 2 * stride) {
    const long long gg[2] = {g0, g0 + stride};
    uint32_t c[2], rk[2];
    double r[2][3];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const long long g = gg[u];
      c[u] = g < npts ? cell_of[g] : kInactive;
      rk[u] = 0u;
      if (c[u] == kInactive) continue;
      rk[u] = arank[g];
      r[u][0] = xyz[3 * g + 0];
      r[u][1] = xyz[3 * g + 1];
      r[u][2] = xyz[3 * g + 2];
    }
    long long pos[2];
#pragma unroll
    for (int u = 0; u < 2; ++u)
      pos[u] = c[u] != kInactive && c[u] < ncells ? (long long)off[c[u]] + rk[u] : -1;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const long long g = gg[u];
      if (g >= npts) continue;
      if (c[u] == kInactive) {
        const int f = ONE || nframes == 1 ? 0 : frame_of_point(frames, nframes, g);
        const FrameDesc &fr = ONE ? fr1 : frames[f];
        const long long i = g - fr.pt_base;
        int *row = out_nn + fr.out_base + i * fr.k;
        for (int s = 0; s < fr.k; ++s) row[s] = -1;
        if (out_d2) {
          double *drow = out_d2 + fr.out_base + i * fr.k;
          const double nan = __longlong_as_double(0x7ff8000000000000ll);
          for (int s = 0; s < fr.k; ++s) drow[s] = nan;
        }
        continue;
      }
      if (pos[u] < 0 || pos[u] >= total) {
        atomicOr(status, kStatusBadIndex);
        continue;
      }
      const int f = ONE || nframes == 1 ? 0 : frame_of_point(frames, nframes, g);
      const FrameDesc &fr = ONE ? fr1 : frames[f];
      double s0, s1, s2, q0, q1, q2;
      fractional(fr, r[u][0], r[u][1], r[u][2], s0, s1, s2);
      cartesian(fr, s0, s1, s2, q0, q1, q2);
      // two 16-byte stores: (g, c, q0) and (q1, q2)
      double2 *w = reinterpret_cast<double2 *>(tmp + pos[u]);
      const unsigned long long gc = (unsigned long long)c[u] << 32 | uint32_t(g);
      w[0] = make_double2(__longlong_as_double((long long)gc), q0);
      w[1] = make_double2(q1, q2);
    }
  }
}

// Stable placement, one thread per sorted slot: the point g arriving at
// slot pos of cell c lands at off[c] + (number of points of c with a
// smaller id), so the order inside a cell is by point id (the reference
// bins points in id order). The slot carries the point's cell and folded
// coordinates, so the kernel reads its slots, the cell offsets and the
// ids of the cell's other slots in sorted order, with no gather by id; the
// writes of the sorted SoA records stay within the cell's few slots, so a
// warp's stores remain coalesced.
template <bool ONE>
__global__ void __launch_bounds__(256, ONE ? 4 : 3)
    k_place_records(const FrameDesc *__restrict__ frames, int nframes, long long npts,
                    long long ncells, const uint32_t *__restrict__ off,
                    const PlaceSlot *__restrict__ tmp, double *__restrict__ sx,
                    double *__restrict__ sy, double *__restrict__ sz, int *__restrict__ sidx,
                    uint32_t *__restrict__ scell, float4 *__restrict__ rec,
                    uint32_t *__restrict__ syz, int *__restrict__ status,
                    const __grid_constant__ FrameDesc fr1) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long total = off[ncells];
  for (long long p0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; p0 < total;
       p0 += 2 * stride) {
    long long pos[2] = {p0, p0 + stride};
    bool live[2];
    uint32_t g[2], c[2];
    double q[2][3];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      live[u] = pos[u] < total;
      g[u] = 0u;
      c[u] = kInactive;
      if (!live[u]) continue;
      const double2 *w = reinterpret_cast<const double2 *>(tmp + pos[u]);
      const double2 w0 = w[0], w1 = w[1];
      const unsigned long long gc = (unsigned long long)__double_as_longlong(w0.x);
      g[u] = uint32_t(gc);
      c[u] = uint32_t(gc >> 32);
      q[u][0] = w0.y;
      q[u][1] = w1.x;
      q[u][2] = w1.y;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (!live[u]) continue;
      if (c[u] >= ncells || (long long)g[u] >= npts) {
        atomicOr(status, kStatusBadIndex);
        continue;
      }
      const uint32_t a = off[c[u]], e = off[c[u] + 1];
      uint32_t rk = 0;
      for (uint32_t t = a; t < e; ++t) rk += tmp[t].g < g[u] ? 1u : 0u;
      const long long dst = (long long)a + rk;
      if (dst >= (long long)e) {
        atomicOr(status, kStatusBadIndex);
        continue;
      }
      const int f = ONE || nframes == 1 ? 0 : frame_of_point(frames, nframes, g[u]);
      const FrameDesc &fr = ONE ? fr1 : frames[f];
      const double q0 = q[u][0], q1 = q[u][1], q2 = q[u][2];
      sx[dst] = q0;
      sy[dst] = q1;
      sz[dst] = q2;
      const int i = int((long long)g[u] - fr.pt_base);
      sidx[dst] = i;
      const uint32_t lc = uint32_t(c[u] - fr.cell_base);
      scell[dst] = lc;
      // FP32 offset from the lower cell corner H (c / n) + origin.
      const int cx = int(lc % uint32_t(fr.nx));
      const int cy = int((lc / uint32_t(fr.nx)) % uint32_t(fr.ny));
      const int cz = int(lc / (uint32_t(fr.nx) * uint32_t(fr.ny)));
      const double f0 = double(cx) / fr.nx, f1 = double(cy) / fr.ny, f2 = double(cz) / fr.nz;
      const double c0 = fr.h[0] * f0 + fr.h[3] * f1 + fr.h[6] * f2 + fr.origin[0];
      const double c1 = fr.h[1] * f0 + fr.h[4] * f1 + fr.h[7] * f2 + fr.origin[1];
      const double c2 = fr.h[2] * f0 + fr.h[5] * f1 + fr.h[8] * f2 + fr.origin[2];
      rec[dst] = make_float4(float(q0 - c0), float(q1 - c1), float(q2 - c2), __int_as_float(cx));
      if (syz)
        syz[dst] = fr.ny <= 0xFFFF && fr.nz <= 0xFFFF ? uint32_t(cy) | (uint32_t(cz) << 16) : kNoYZ;
    }
  }
}

__global__ void k_count_active(const int *__restrict__ mask, long long n,
                               unsigned long long *__restrict__ out) {
  unsigned long long local = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    local += mask[i] != 0;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) local += __shfl_xor_sync(0xffffffffu, local, d);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

// The rows of a search whose mesh is too fine, after k_count_active: with
// no active point every slot becomes -1 / NaN, as the reference fills the
// rows before it returns for an all-masked search (src/knearest.rs:293-296,
// 370-375); otherwise the status word gets kStatusPlanTooFine and nothing
// is written.
__global__ void k_fill_if_inactive(const unsigned long long *__restrict__ active,
                                   int *__restrict__ out_nn, double *__restrict__ out_d2,
                                   long long need, int *__restrict__ status) {
  if (*active != 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, kStatusPlanTooFine);
    return;
  }
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < need;
       i += (long long)gridDim.x * blockDim.x) {
    out_nn[i] = -1;
    if (out_d2) out_d2[i] = nan;
  }
}

int grid_for(long long n, int block) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (n + block - 1) / block;
  const long long cap = (long long)sms * 16;
  return int(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

long long scan_tiles(long long ncells) { return (ncells + kScanTile - 1) / kScanTile; }

cudaError_t launch_fold_bin(const BatchBuffers &b, cudaStream_t s, const FrameDesc *one) {
  if (b.npts <= 0) return cudaSuccess;
  const int grid = grid_for(b.npts, 256);
  if (one && b.nframes == 1)
    k_fold_bin<true><<<grid, 256, 0, s>>>(b.xyz, b.mask, b.frames, b.nframes, b.npts, b.cell_of,
                                          b.arank, b.count, b.frame_flags, *one);
  else
    k_fold_bin<false><<<grid, 256, 0, s>>>(b.xyz, b.mask, b.frames, b.nframes, b.npts, b.cell_of,
                                           b.arank, b.count, b.frame_flags, FrameDesc{});
  return cudaGetLastError();
}

cudaError_t launch_scan(const BatchBuffers &b, cudaStream_t s) {
  long long grid = scan_tiles(b.ncells);
  if (b.live_cells) {
    // the live tile count is only known on the device: blocks loop
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    grid = std::min<long long>(grid, (long long)sms * 4);
  }
  k_scan_cells<<<unsigned(grid), kScanBlock, 0, s>>>(b.count, b.off, b.ncells, b.live_cells,
                                                      b.tile_state, b.tile_counter, b.status,
                                                      b.scan_spin_limit, b.scan_silent_tile);
  return cudaGetLastError();
}

cudaError_t launch_zero_live(const BatchBuffers &b, cudaStream_t s) {
  k_zero_live<<<grid_for(b.ncells, 256), 256, 0, s>>>(b.count, b.tile_state, b.live_cells);
  return cudaGetLastError();
}

cudaError_t launch_place(const BatchBuffers &b, cudaStream_t s, const FrameDesc *one) {
  if (b.npts <= 0) return cudaSuccess;
  const int g = grid_for(b.npts, 256);
  const bool single = one && b.nframes == 1;
  const FrameDesc fr1 = single ? *one : FrameDesc{};
  if (single)
    k_place_slots<true><<<g, 256, 0, s>>>(b.xyz, b.frames, b.nframes, b.cell_of, b.arank, b.off,
                                          b.tmp, b.npts, b.ncells, b.out_nn, b.out_d2, b.status,
                                          fr1);
  else
    k_place_slots<false><<<g, 256, 0, s>>>(b.xyz, b.frames, b.nframes, b.cell_of, b.arank, b.off,
                                           b.tmp, b.npts, b.ncells, b.out_nn, b.out_d2, b.status,
                                           fr1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (single)
    k_place_records<true><<<g, 256, 0, s>>>(b.frames, b.nframes, b.npts, b.ncells, b.off, b.tmp,
                                            b.sx, b.sy, b.sz, b.sidx, b.scell, b.rec, b.syz,
                                            b.status, fr1);
  else
    k_place_records<false><<<g, 256, 0, s>>>(b.frames, b.nframes, b.npts, b.ncells, b.off, b.tmp,
                                             b.sx, b.sy, b.sz, b.sidx, b.scell, b.rec, b.syz,
                                             b.status, fr1);
  return cudaGetLastError();
}

cudaError_t launch_count_active(const int *mask, long long n, unsigned long long *out,
                                cudaStream_t s) {
  k_count_active<<<grid_for(n, 256), 256, 0, s>>>(mask, n, out);
  return cudaGetLastError();
}

cudaError_t launch_masked_too_fine(const int *mask, long long n, unsigned long long *active,
                                   int *out_nn, double *out_d2, long long need, int *status,
                                   cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(active, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  if ((e = launch_count_active(mask, n, active, s)) != cudaSuccess) return e;
  k_fill_if_inactive<<<grid_for(need, 256), 256, 0, s>>>(active, out_nn, out_d2, need, status);
  return cudaGetLastError();
}

}  // namespace lc
