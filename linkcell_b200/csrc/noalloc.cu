// lc_gpu_knearest_noalloc: one search that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application that hands all of
// the GPU's memory to its own pool allocator at start-up and forbids other
// allocations, a real-time loop in which an allocation may block or fail at
// the wrong moment, or a plug-in that runs inside a framework which owns the
// device allocator. For them this entry point keeps every scratch buffer of
// the search (cell histogram and offsets, arrival slots, the cell-sorted
// point records, the scan's tile states, counters and the replay heaps) in
// one file-scope static __device__ array of fixed size. Every GPU that loads
// the library holds that array until the process exits. The caller still
// passes the inputs and the outputs.
//
// Limits: at most kNoAllocMaxPoints points, kNoAllocMaxCells linked cells
// and k <= kNoAllocMaxK; larger searches are rejected with an error. All
// calls share the one array and leave their contents in it, so calls that
// overlap on the GPU (on different streams, or from different host threads
// without ordering) race and must not be issued.
//
// Every call, with the caller's device current, looks up the array's device
// address with cudaGetSymbolAddress (the array's name in host code only
// stands in for the symbol; it is not a device pointer). The first call on a
// device also loads this library's kernels there (that is its set-up), so it
// should come before any stream capture. Looking the address up again on
// every call keeps it right after a cudaDeviceReset, which gives the array a
// new context.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <limits>

#include "../../include/linkcell_gpu.h"
#include "lc_kernels.h"
#include "workspace.h"

namespace lc {
// Error slot of the device C ABI (capi.cu).
void set_gpu_error_message(const char *msg);
}  // namespace lc

namespace {

constexpr long long kNoAllocMaxPoints = 65536;
constexpr long long kNoAllocMaxCells = 65536;
constexpr int kNoAllocMaxK = 64;
constexpr int kNoAllocReplayThreads = 256;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of each buffer inside the scratch array.
struct Layout {
  size_t frame, counters, small, cell_of, arank, tmp, count, off, tile_state, sx, sy, sz, sidx,
      scell, rec, replay_list, replay_d, replay_i, total;
};

constexpr Layout make_layout() {
  Layout l{};
  size_t o = 0;
  const size_t P = size_t(kNoAllocMaxPoints), C = size_t(kNoAllocMaxCells);
  const size_t tiles = (C + lc::kScanTile - 1) / lc::kScanTile;
  l.frame = o; o += align256(sizeof(lc::FrameDesc));
  l.counters = o; o += align256(sizeof(long long) * lc::kNumCounters);
  // tile counter, work, replay count, status, frame flags; words 6-7: the
  // active-point count of a masked search on a too-fine mesh
  l.small = o; o += align256(8 * sizeof(uint32_t));
  l.cell_of = o; o += align256(P * 4);
  l.arank = o; o += align256(P * 4);
  l.tmp = o; o += align256(P * sizeof(lc::PlaceSlot));
  l.count = o; o += align256(C * 4);
  l.off = o; o += align256((C + 1) * 4);
  l.tile_state = o; o += align256(tiles * 8);
  l.sx = o; o += align256(P * 8);
  l.sy = o; o += align256(P * 8);
  l.sz = o; o += align256(P * 8);
  l.sidx = o; o += align256(P * 4);
  l.scell = o; o += align256(P * 4);
  l.rec = o; o += align256(P * 16);
  l.replay_list = o; o += align256(P * 4);
  l.replay_d = o; o += align256(size_t(kNoAllocReplayThreads) * kNoAllocMaxK * 8);
  l.replay_i = o; o += align256(size_t(kNoAllocReplayThreads) * kNoAllocMaxK * 4);
  l.total = o;
  return l;
}

constexpr Layout kLayout = make_layout();

// About 6.7 MB per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kLayout.total];

// Device address of the scratch array in the current device's context.
cudaError_t scratch_base(unsigned char **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<unsigned char *>(p);
  return cudaSuccess;
}

int fail(const char *msg) {
  lc::set_gpu_error_message(msg);
  return 1;
}

int fail_cuda(cudaError_t e) {
  lc::set_gpu_error_message(cudaGetErrorString(e));
  return 1;
}

}  // namespace

extern "C" int lc_gpu_knearest_noalloc(const double *xyz, size_t n, const struct lc_cell *simbox,
                                       size_t k, const int *mask, double cell_hint, int *out_nn,
                                       double *out_d2, void *stream, int wait) {
  if (!xyz || !simbox || !out_nn) return fail("null pointer");
  if (n == 0) return fail("no points");
  if (k == 0) return fail("k must be at least 1");
  if ((long long)n > kNoAllocMaxPoints) return fail("no-alloc search supports at most 65536 points");
  if (k > size_t(kNoAllocMaxK)) return fail("no-alloc search supports k <= 64");
  const double rows[9] = {simbox->ax, simbox->ay, simbox->az, simbox->bx, simbox->by,
                          simbox->bz, simbox->cx, simbox->cy, simbox->cz};
  const double origin[3] = {simbox->ox, simbox->oy, simbox->oz};
  lc::FrameDesc fd;
  const lc::Code pc = lc::plan_frame(rows, origin, cell_hint, int(k), fd);
  if (pc == lc::Code::BadCell) return fail("bad cell");
  const long long ncells = pc == lc::Code::Ok ? (long long)fd.nx * fd.ny * fd.nz : 0;
  const char *mesh_error = pc == lc::Code::TooFine ? "too many cells"
                           : ncells > kNoAllocMaxCells
                               ? "no-alloc search supports at most 65536 cells"
                               : nullptr;
  if (mesh_error && !mask) return fail(mesh_error);

  unsigned char *base = nullptr;
  cudaError_t e = scratch_base(&base);
  if (e != cudaSuccess) return fail_cuda(e);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Layout &L = kLayout;
  uint32_t *small = reinterpret_cast<uint32_t *>(base + L.small);

  if (mesh_error) {
    // The reference returns -1 / NaN rows for an all-masked search before it
    // sizes the mesh (src/knearest.rs:370-375): the mask is checked on the
    // device, and this call waits for that check whatever wait says.
    int *status = reinterpret_cast<int *>(small + 3);
    unsigned long long *active = reinterpret_cast<unsigned long long *>(small + 6);
    int st = 0;
    if ((e = cudaMemsetAsync(status, 0, sizeof(int), s)) != cudaSuccess ||
        (e = lc::launch_masked_too_fine(mask, (long long)n, active, out_nn, out_d2,
                                        (long long)(n * k), status, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return fail_cuda(e);
    if (st != 0) return fail(mesh_error);
    lc::set_gpu_error_message(nullptr);
    return 0;
  }
  fd.n = (long long)n;
  fd.has_mask = mask ? 1 : 0;
  fd.mask_base = 0;
  fd.out_base = 0;
  fd.pt_base = 0;
  fd.cell_base = 0;

  lc::BatchBuffers b;
  b.xyz = xyz;
  b.mask = mask;
  b.frames = reinterpret_cast<const lc::FrameDesc *>(base + L.frame);
  b.nframes = 1;
  b.npts = (long long)n;
  b.ncells = ncells;
  b.cell_of = reinterpret_cast<uint32_t *>(base + L.cell_of);
  b.arank = reinterpret_cast<uint32_t *>(base + L.arank);
  b.tmp = reinterpret_cast<lc::PlaceSlot *>(base + L.tmp);
  b.count = reinterpret_cast<uint32_t *>(base + L.count);
  b.off = reinterpret_cast<uint32_t *>(base + L.off);
  b.tile_state = reinterpret_cast<unsigned long long *>(base + L.tile_state);
  b.tile_counter = small + 0;
  b.work = small + 1;
  b.replay_count = small + 2;
  b.status = reinterpret_cast<int *>(small + 3);
  b.frame_flags = reinterpret_cast<int *>(small + 4);
  b.sx = reinterpret_cast<double *>(base + L.sx);
  b.sy = reinterpret_cast<double *>(base + L.sy);
  b.sz = reinterpret_cast<double *>(base + L.sz);
  b.sidx = reinterpret_cast<int *>(base + L.sidx);
  b.scell = reinterpret_cast<uint32_t *>(base + L.scell);
  b.rec = reinterpret_cast<float4 *>(base + L.rec);
  b.out_nn = out_nn;
  b.out_d2 = out_d2;
  b.replay_list = reinterpret_cast<int *>(base + L.replay_list);
  b.replay_cap = (long long)n;
  b.replay_d = reinterpret_cast<double *>(base + L.replay_d);
  b.replay_i = reinterpret_cast<int *>(base + L.replay_i);
  b.replay_threads = kNoAllocReplayThreads;
  b.kmax = int(k);
  b.counters = reinterpret_cast<long long *>(base + L.counters);

  // The array keeps the previous call's contents: reset everything that
  // must start at zero, and the frame description.
  const long long tiles = lc::scan_tiles(ncells);
  if ((e = cudaMemcpyAsync(base + L.frame, &fd, sizeof(fd), cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (e = cudaMemsetAsync(small, 0, 8 * sizeof(uint32_t), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(b.count, 0, size_t(ncells) * 4, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(b.tile_state, 0, size_t(tiles) * 8, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(b.counters, 0, sizeof(long long) * lc::kNumCounters, s)) !=
          cudaSuccess)
    return fail_cuda(e);

  lc::WalkLaunch wl;
  wl.mode = lc::kModeFastF32;
  wl.kmax = int(k);
  wl.block = lc::walk_max_block(wl.mode, int(k));
  if ((e = lc::launch_fold_bin(b, s)) != cudaSuccess || (e = lc::launch_scan(b, s)) != cudaSuccess ||
      (e = lc::launch_place(b, s)) != cudaSuccess || (e = lc::launch_walk(b, wl, s)) != cudaSuccess ||
      (e = lc::launch_replay(b, s)) != cudaSuccess)
    return fail_cuda(e);
  if (wait) {
    int st = 0;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess ||
        (e = cudaMemcpy(&st, b.status, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess)
      return fail_cuda(e);
    if (st != 0) return fail("device search failed");
  }
  lc::set_gpu_error_message(nullptr);
  return 0;
}
