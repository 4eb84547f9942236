// Launch wrappers of the sm_100a kernels of the linked-cell k-nearest
// search. Host code (workspace.cu) calls only these; every pointer is a
// device pointer and every launch goes on the given stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lc_types.h"

namespace lc {

// Device buffers of one batch. Sizes: P = points in the batch, C = cells
// in the batch, F = frames.
constexpr uint32_t kNoYZ = 0xFFFFFFFFu;

// A point at its arrival slot inside its cell: the point id, the batch cell
// and the folded FP64 coordinates, 32 bytes (two 16-byte words).
struct __align__(16) PlaceSlot {
  uint32_t g, c;
  double q0, q1, q2;
};
static_assert(sizeof(PlaceSlot) == 32, "PlaceSlot is two 16-byte words");

struct BatchBuffers {
  const double *xyz = nullptr;   // P*3, frame-major, caller's
  const int *mask = nullptr;     // caller's; frames index it with mask_base
  const FrameDesc *frames = nullptr;  // F
  int nframes = 0;
  long long npts = 0;            // P
  long long ncells = 0;          // C (cell arrays' size)
  // device-planned batch: the cells in use (first *live_cells), else null
  const long long *live_cells = nullptr;
  uint32_t *cell_of = nullptr;   // P: batch cell id or kInactive
  uint32_t *arank = nullptr;     // P: arrival rank inside the cell (atomics)
  PlaceSlot *tmp = nullptr;      // P: the point at its arrival slot
  uint32_t *count = nullptr;     // C
  uint32_t *off = nullptr;       // C+1: exclusive scan of count
  unsigned long long *tile_state = nullptr;  // scan tiles
  uint32_t *tile_counter = nullptr;
  int *status = nullptr;         // StatusBits
  int *frame_flags = nullptr;    // F
  // cell-sorted (stable: ascending point id inside a cell) source arrays
  double *sx = nullptr, *sy = nullptr, *sz = nullptr;  // folded FP64 SoA
  int *sidx = nullptr;           // index of the point inside its frame
  uint32_t *scell = nullptr;     // cell id inside the frame
  float4 *rec = nullptr;         // FP32 offset from the cell corner; w: the cell's x index (int bits)
  // optional: the cell's y | z << 16 (kNoYZ where the frame has more than
  // 65535 cells along y or z), read by the select walk instead of dividing scell
  uint32_t *syz = nullptr;
  // outputs (caller's)
  int *out_nn = nullptr;
  double *out_d2 = nullptr;
  // walk bookkeeping
  uint32_t *work = nullptr;      // work-queue cursor
  int *replay_list = nullptr;    // sorted positions that need the exact replay
  uint32_t *replay_count = nullptr;
  long long replay_cap = 0;
  double *replay_d = nullptr;    // replay heap scratch: replay_threads * kmax
  int *replay_i = nullptr;
  int replay_threads = 0;
  int kmax = 0;
  long long *counters = nullptr; // walk statistics (see WalkCounters)
  const int8_t *proposal = nullptr;  // learned walk: proposed shell per sorted source (0: none)
  int8_t *stop_log = nullptr;        // optional: settled shell per sorted source (training)
  const uint32_t *shell_table = nullptr;  // near-first shell offsets, shells 1..shell_rmax
  int shell_rmax = 0;
  // optional source order: when set, the walk visits sorted positions
  // src_order[*src_lo .. *src_hi) instead of all of them (the bounds are
  // device values, written by the kernels that built the order); with
  // src_lo / src_hi but no src_order, the sorted positions *src_lo ..
  // *src_hi themselves (one rank's share of a split search)
  const int *src_order = nullptr;
  const uint32_t *src_lo = nullptr, *src_hi = nullptr;
  // scan look-back: loads a wait may take (0: the default bound) and a tile
  // that never publishes (-1: none); failure-detection tests only
  int scan_spin_limit = 0;
  long long scan_silent_tile = -1;
};

// Sources a walk launch visits, and the sorted position of the q-th.
__device__ __forceinline__ long long walk_sources(const BatchBuffers &b) {
  return b.src_lo ? (long long)*b.src_hi - (long long)*b.src_lo : (long long)b.off[b.ncells];
}
__device__ __forceinline__ long long walk_source_at(const BatchBuffers &b, long long q) {
  return b.src_order ? (long long)b.src_order[*b.src_lo + q]
                     : (b.src_lo ? (long long)*b.src_lo + q : q);
}

// Walk statistics accumulated on the device (counters[...]).
enum WalkCounters : int {
  kCntPairs = 0,      // candidate distances evaluated
  kCntInserts = 1,    // heap insertions
  kCntReplays = 2,    // sources sent to the exact replay
  kCntShells = 3,     // shells walked (sum over sources)
  kCntPruned = 4,     // stencil cells skipped by the distance bound
  kCntRerank = 5,     // FP64 recomputations in the FP32 walk
  kCntPropUnder = 6,  // learned proposal too short
  kCntPropOver = 7,   // learned proposal too long
  kCntPropExact = 8,  // learned proposal equal to the settled shell
  kCntRevisit = 9,    // shells walked again after a short proposal
  kCntFallback = 10,  // cube-select sources sent to the literal replay (not ties)
  kNumCounters = 16
};

constexpr int kShellTableRmax = 16;

constexpr int kScanBlock = 256;
constexpr int kScanItems = 16;  // a multiple of 4 (16-byte loads and stores)
constexpr int kScanTile = kScanBlock * kScanItems;

long long scan_tiles(long long ncells);

// fold + bin + cell histogram (one pass over the points).
// one: the batch's single frame as the host holds it (read by the kernel from
// its parameters), or nullptr to read the frames from device memory.
cudaError_t launch_fold_bin(const BatchBuffers &b, cudaStream_t s, const FrameDesc *one = nullptr);
// exclusive scan of the histogram (single-pass decoupled look-back).
cudaError_t launch_scan(const BatchBuffers &b, cudaStream_t s);
// Zeroes counts and scan tile states of the live cells (device-planned batches).
cudaError_t launch_zero_live(const BatchBuffers &b, cudaStream_t s);
// stable cell-sorted placement: arrival slots, then in-cell rank by point id.
cudaError_t launch_place(const BatchBuffers &b, cudaStream_t s, const FrameDesc *one = nullptr);

// Walk modes.
enum WalkMode : int {
  kModePlainF64 = 0,   // shell-by-shell FP64 walk
  kModeFastF32 = 1,    // FP32 candidates + FP64 rerank, shell-by-shell
  kModeLearned = 2,    // FP32 + learned shell proposal (cube opened at once)
  kModeReplayAll = 3,  // every source through the exact sequential replay
};

struct WalkLaunch {
  int mode = kModePlainF64;
  int tpp = 1;      // threads per source: 1 (heap in shared memory) or 32 (warp team)
  int block = 128;
  int grid = 0;
  int kmax = 32;
  int prune = 1;
  bool stats = false;  // the learned select walk counts its statistics
  const int8_t *proposal = nullptr;  // per sorted source proposed shell (learned mode)
  // select walk shape: warps per block (k <= 32: 8 or 4; k <= 64: 4 or 2;
  // 0 = the default) and sources per work grab (8, 16 or 32; 0 = 16)
  int warps = 0;
  int grab = 0;
  // A single frame whose description the host holds (not device-planned, no
  // CUDA graph, which would replay the launch with this copy): the select
  // walk takes it as a kernel parameter and reads it from the constant bank.
  bool one = false;
  FrameDesc frame1{};
};

// Walk shapes the autotuner times for the select walk of k <= kmax.
constexpr int kSelGrabs[3] = {8, 16, 32};
inline int sel_warps_for(int kmax, int i) { return kmax <= 32 ? (i ? 4 : 8) : (i ? 2 : 4); }

cudaError_t launch_walk(const BatchBuffers &b, const WalkLaunch &w, cudaStream_t s);
cudaError_t launch_replay(const BatchBuffers &b, cudaStream_t s, const FrameDesc *one = nullptr);
// order[pt_base + index] = sorted position of each active source (order is
// pre-filled with -1 for masked points).
// Output-row ranges of a host-pointer search: row cuts cut[0] = 0 <
// cut[1] < ... < cut[nr] (point units).
constexpr int kMaxRowRanges = 12;
struct RowCuts {
  long long cut[kMaxRowRanges + 1];
  int nr;
};
// Sorted positions partitioned by the row range of their source, cell order
// kept inside each range: order[off[r * nblk] .. off[(r + 1) * nblk]) are
// range r's. cnt and off (nr * nblk + 1 entries) are scratch of
// range_partition_blocks(); tile_state (scan tiles of nr * nblk) and
// tile_counter serve the scan.
long long range_partition_blocks(long long sources);
cudaError_t launch_range_partition(const BatchBuffers &b, const RowCuts &cuts, uint32_t *cnt,
                                   uint32_t *off, unsigned long long *tile_state,
                                   uint32_t *tile_counter, int *order, cudaStream_t s);
// One rank's share of a search split across ranks that hold the same
// inputs: the sorted sources are cut into world contiguous ranges of equal
// expected work (weight of a source: its cell's occupancy times its proposed
// cube, plus one), and cut[0], cut[1] get rank's range. w (npts words), pre
// (npts + 1), tile_state (scan tiles of npts) and tile_counter are scratch.
cudaError_t launch_shard_split(const BatchBuffers &b, int rank, int world, uint32_t *w,
                               uint32_t *pre, unsigned long long *tile_state,
                               uint32_t *tile_counter, uint32_t *cut, cudaStream_t s);
// owned[i] = 1 for every point whose row this rank wrote: its sources in
// [cut[0], cut[1]), and on rank 0 every masked point (-1 / NaN rows on every
// rank). owned has npts entries, zeroed here.
cudaError_t launch_shard_owned(const BatchBuffers &b, const uint32_t *cut, int rank, int *owned,
                               cudaStream_t s);
// CSR of the entries within a cutoff of n x k rows (sorted ascending, -1 /
// NaN padded): counts and row_off are rows + 1 scratch words, tile_state /
// tile_counter the scan's scratch; row_ptr gets rows + 1 offsets, col /
// dist2 the first cap kept entries.
cudaError_t launch_csr(const int *nn, const double *d2, long long rows, int k, double cutoff,
                       uint32_t *counts, uint32_t *row_off, unsigned long long *tile_state,
                       uint32_t *tile_counter, int *status, int *row_ptr, int *col,
                       double *dist2, long long cap, cudaStream_t s);
size_t walk_smem_bytes(int mode, int block, int kmax);
// Near-first shell-offset table for shells 1..rmax ((2 rmax + 1)^3 entries).
void build_shell_table(int rmax, uint32_t *out);
int walk_max_block(int mode, int kmax);
cudaError_t walk_prepare(int mode, int kmax, int block);  // sets the dynamic smem attribute

// Counts active points (used to tell an all-masked batch from a bad mesh).
cudaError_t launch_count_active(const int *mask, long long n, unsigned long long *out,
                                cudaStream_t s);
// A mesh too fine for the bin caps with a length-n mask: counts the active
// points into *active; none: the need output slots become -1 / NaN; some:
// kStatusPlanTooFine goes into *status (which the caller zeroed).
cudaError_t launch_masked_too_fine(const int *mask, long long n, unsigned long long *active,
                                   int *out_nn, double *out_d2, long long need, int *status,
                                   cudaStream_t s);

}  // namespace lc
