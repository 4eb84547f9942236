// Host-side planning and the device workspace of the linked-cell k-nearest
// search. The C ABI (capi.cpp) and the C++ class linkcell::gpu::Workspace
// are thin layers over WorkspaceImpl.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "lc_kernels.h"
#include "lc_types.h"

namespace lc {

// Why a call failed. Each public API family maps these to its own strings.
enum class Code {
  Ok = 0,
  NoPoints,      // n == 0 or n_frames == 0
  ZeroK,         // k == 0
  NullPointer,
  Overflow,      // n * k does not fit
  BadCell,       // singular or non-positive cell
  TooFine,       // linked-cell mesh exceeds the bin caps
  BadCellN,      // device cell is not 3, 9 or 12 doubles
  NoDevice,      // no CUDA device
  Cuda,          // a CUDA runtime call failed (message in detail)
  DeviceStatus,  // a kernel reported a status bit
  TooLarge,      // batch exceeds the 32-bit point / cell indexing
};

// The reference's messages for the CPU C ABI (src/error.rs:24-36,
// src/capi.rs:201-203).
const char *cpu_message(Code c);
// The reference's messages for the device C ABI (src/gpu/knearest.cpp,
// src/gpu/capi.cpp).
const char *gpu_message(Code c);

// Cell::from_vectors + the mesh of search() (src/cell.rs:97-124,
// src/knearest.rs:377-397,430) into a FrameDesc. rows = a, b, c (9 doubles)
// and origin (3 doubles). hint <= 0 or NaN selects the default edge 3.0.
Code plan_frame(const double *rows, const double *origin, double cell_hint, int k, FrameDesc &fd);
// Fraction of B(R_p) the select walk's first gather covers, for k.
double select_rho_q(int k);
// Plans the shared cell of a device-cell batch on the device (no host
// read of the cell) and writes the frame table of nframes frames of n
// points; *live_cells gets the batch's cell count. Rejections leave
// kStatusPlanBadCell / kStatusPlanTooFine in status.
cudaError_t launch_plan_device_cell(const double *cell, int cell_n, long long n, int nframes, int k,
                                    double hint, const int *mask, FrameDesc *frames,
                                    long long *live_cells, int *status, cudaStream_t s);
// Device address of page-locked host memory, or null.
void *mapped_host(const void *p);

// A walk design and shape: threads per source (32 or 1) and, for the cube
// select walk, warps per block and sources per work grab (0: default).
struct WalkShape {
  int tpp = 32, warps = 0, grab = 0;
};

// Options that pick the walk.
struct WalkOptions {
  // the learned walk: results equal every other mode's, and it is the fastest
  int mode = kModeLearned;
  int tpp = 32;    // threads per source: 32 (warp team) or 1 (one thread, heap in shared memory)
  int block = 0;   // 0: autotune / default
  int sel_warps = 0;  // select walk warps per block (lc_gpu_set_walk_shape), 0: autotune
  int sel_grab = 0;   // select walk sources per grab (or LINKCELL_GRAB), 0: autotune
  int prune = 1;
  int fixed_proposal = 0;  // learned walk: > 0 proposes this shell for every source
  int log_shells = 0;      // record the settled shell of every source (training data)
  bool tpp_forced = false; // tpp set explicitly (API or LINKCELL_TPP): no autotuning
  bool autotune = true;    // time the walk designs on the first batch of each kind
  bool graph = false;      // capture the launch sequence in a CUDA graph and replay it
  bool stats = false;      // the learned select walk counts its statistics (lc_gpu_stats)
  // failure-detection tests (lc_gpu_set_scan_limit): the scan's wait bound
  // (0: default) and a scan tile that never publishes (-1: none)
  int scan_spin_limit = 0;
  long long scan_silent_tile = -1;
};

struct Stats {
  long long counters[kNumCounters] = {};
  double ms_total = 0.0;   // fold .. replay, device time
  double ms_prep = 0.0;    // fold + bin + scan + placement
  double ms_walk = 0.0;    // shell proposals + the walk kernel(s)
  double ms_propose = 0.0; // shell proposals alone (learned mode)
  double ms_replay = 0.0;  // exact replay of tied sources
};

class WorkspaceImpl {
 public:
  WorkspaceImpl();
  ~WorkspaceImpl();
  WorkspaceImpl(const WorkspaceImpl &) = delete;
  WorkspaceImpl &operator=(const WorkspaceImpl &) = delete;

  cudaStream_t stream();
  void set_stream(cudaStream_t s);  // nullptr: back to the workspace's own stream
  Code wait(std::string &detail);

  // Runs one batch. frames[f] carries the plan (plan_frame) plus pt_base,
  // cell_base (filled here), out_base and mask_base. xyz, mask, outputs are
  // device pointers.
  Code run(std::vector<FrameDesc> &frames, const double *xyz, const int *mask, int *out_nn,
           double *out_d2, bool wait, std::string &detail);

  // A mesh too fine for the bin caps with a length-n device mask. The
  // reference returns -1 / NaN rows for an all-masked search before it sizes
  // the mesh (src/knearest.rs:370-375), so the mask is checked on the device:
  // no active point fills the need output slots; any active point reports
  // TooFine when the call waits (else at the next wait()).
  Code too_fine_masked(const int *mask, long long n, int *out_nn, double *out_d2, long long need,
                       bool wait, std::string &detail);

  // Device-cell batch without a host read of the cell: nframes frames of n
  // points sharing the cell at the device pointer cell (cell_n = 3, 9 or 12
  // doubles), planned on the device at every launch (and every graph
  // replay). The cell arrays are sized for the largest mesh a cell may have
  // (kMaxCellsPerFrame per frame), so nframes is at most kDeviceCellFrames.
  // A rejected cell reports BadCell / TooFine when the batch is waited for.
  static constexpr int kDeviceCellFrames = 16;
  Code run_device_cell(const double *cell, int cell_n, long long n, int nframes, int k,
                       double hint, const double *xyz, const int *mask, int *out_nn,
                       double *out_d2, bool wait, std::string &detail);

  // One rank's share of a search split across world ranks that hold the
  // same inputs: the prep runs whole, the walk covers this rank's range of
  // sorted sources (split by expected work), and owned (device, one int per
  // point) marks the rows this rank wrote. Graphs are not used for it.
  Code run_shard(std::vector<FrameDesc> &frames, const double *xyz, const int *mask, int *out_nn,
                 double *out_d2, int *owned, int rank, int world, bool wait, std::string &detail);

  WalkOptions opts;
  bool collect_stats = true;
  int last_tpp = 0;          // walk design of the last batch
  WalkShape last_shape;      // design and shape of the last batch's walk
  std::vector<WalkShape> trial_shapes_;  // the candidates the last autotuning timed
  int last_host_rows = 0;  // how the last host-pointer search returned its rows (0 copy, 1 ranges, 2 mapped)
  int graph_captures = 0;    // CUDA graphs captured so far
  // Counters and phase times of the last run (waits for it to finish).
  Code fetch_stats(Stats &out, std::string &detail);

  // Host-pointer convenience used by the CPU-compatible C ABI: copies in,
  // runs, copies out, waits.
  Code run_host(std::vector<FrameDesc> &frames, const double *xyz, size_t xyz_n, const int *mask,
                size_t mask_n, int *out_nn, double *out_d2, size_t out_n, std::string &detail);

  // Device-side view of the last batch (diagnostics and tests).
  const BatchBuffers &buffers() const { return bb_; }

  // Learned proposals: copy the MLP parameters (host floats) in.
  Code set_model(const float *params, size_t n, float tau, std::string &detail);
  bool has_model() const { return has_model_; }
  // Proposed shells of the last learned search for the sorted sources
  // first, first + stride, ... (host buffer).
  Code proposals(int8_t *out, long long cap, long long stride, long long first, long long &rows,
                 std::string &detail);
  // Training rows of the last logged search (device X / y buffers).
  Code training_rows(float *X, int *y, long long cap, long long stride, long long first,
                     long long &rows, std::string &detail);

 private:
  template <class T>
  struct Buf {
    T *p = nullptr;
    size_t cap = 0;
  };
  template <class T>
  cudaError_t grow(Buf<T> &b, size_t n);
  Code enqueue(BatchBuffers &b, const WalkLaunch &wl, int nf, size_t C, long long tiles,
               cudaStream_t s, bool timed, std::string &detail);

  struct GraphKey {
    long long npts = -1, ncells = -1;
    int nf = 0, kmax = 0;
    const void *xyz = nullptr, *mask = nullptr, *nn = nullptr, *d2 = nullptr;
    int mode = 0, tpp = 0, block = 0, model = 0, fixed = 0, log = 0, stats = 0;
    const void *dcell = nullptr;  // device-planned batch: its cell and launch constants
    int cell_n = 0;
    double hint = 0.0;
    int spin = 0;
    long long silent = -1;
    bool operator==(const GraphKey &o) const {
      return npts == o.npts && ncells == o.ncells && nf == o.nf && kmax == o.kmax && xyz == o.xyz &&
             mask == o.mask && nn == o.nn && d2 == o.d2 && mode == o.mode && tpp == o.tpp &&
             block == o.block && model == o.model && fixed == o.fixed && log == o.log &&
             stats == o.stats &&
             dcell == o.dcell && cell_n == o.cell_n && hint == o.hint && spin == o.spin &&
             silent == o.silent;
    }
  };
  // the device-cell batch being enqueued (run_device_cell)
  struct DeviceCell {
    bool on = false;
    const double *cell = nullptr;
    int cell_n = 0;
    long long n = 0;
    int nframes = 0, k = 0;
    double hint = 0.0;
  };
  DeviceCell dcell_;
  Buf<long long> live_;
  GraphKey graph_key_;
  cudaGraphExec_t graph_exec_ = nullptr;
  bool graph_total_ = false;
  std::map<int, WalkShape> tuned_;
  FrameDesc *h_frames_ = nullptr;
  size_t h_frames_cap_ = 0;
  cudaEvent_t ev_done_ = nullptr;
  // host-pointer searches with page-locked outputs: 1 = row ranges copied back
  // while the next range is searched, 2 = rows written to mapped host memory,
  // 0 = one copy at the end (LINKCELL_HOST_ROWS)
  int host_rows_ = 1;
  static constexpr long long kMinRangeRows = 16384;  // shortest row range
  struct Pipe {
    bool on = false, done = false;
    int *host_nn = nullptr;
    double *host_d2 = nullptr;
  };
  Pipe pipe_;
  Buf<int> order_;
  cudaStream_t copy_stream_ = nullptr;
  cudaEvent_t range_ev_[kMaxRowRanges + 1] = {};
  Buf<uint32_t> part_cnt_, part_off_;
  Buf<unsigned long long> part_tiles_;
  Code walk_in_row_ranges(BatchBuffers &b, const WalkLaunch &wl, cudaStream_t s, bool timed,
                          std::string &detail);
  struct Shard {
    bool on = false;
    int rank = 0, world = 1;
    int *owned = nullptr;
  };
  Shard shard_;
  Buf<uint32_t> shard_cut_;
  Code walk_shard(BatchBuffers &b, const WalkLaunch &wl, cudaStream_t s, bool timed,
                  std::string &detail);
  Buf<uint32_t> csr_counts_, csr_off_;

 public:
  // CSR of the entries of n x k rows (device) within cutoff; waits.
  Code neighbors_within(const int *nn, const double *d2, size_t rows, size_t k, double cutoff,
                        int *row_ptr, int *col, double *dist2, size_t cap, size_t &nnz,
                        std::string &detail);

 private:
  bool done_pending_ = false;
  void release_all();
  Code read_status(std::string &detail);  // the status word of the last batch

  int device_ = -1;
  cudaStream_t own_ = nullptr;
  cudaStream_t user_ = nullptr;
  bool user_set_ = false;
  cudaStream_t last_stream_ = nullptr;  // stream of the last batch

  Buf<uint32_t> cell_of_, arank_, count_, off_, tile_counter_, work_, replay_count_;
  Buf<PlaceSlot> tmp_;
  Buf<unsigned long long> tile_state_;
  Buf<int> status_, frame_flags_, sidx_, replay_list_, replay_i_;
  Buf<uint32_t> scell_;
  Buf<double> sx_, sy_, sz_, replay_d_;
  Buf<float4> rec_;
  Buf<uint32_t> syz_;  // learned walk: the cell's y | z << 16 per sorted point
  Buf<FrameDesc> frames_;
  Buf<long long> counters_;
  Buf<int8_t> proposal_, cell_prop_, stop_log_;
  Buf<float> model_;
  Buf<uint4> model_image_;  // the inference kernel's operand image of model_
  Buf<uint32_t> shell_table_;
  bool shell_table_ready_ = false;
  bool has_model_ = false;
  bool model_tried_ = false;  // the shipped network was looked for once
  bool load_default_model();
  float tau_ = 0.9f;
  // host-pointer staging
  Buf<double> h_xyz_, h_d2_;
  Buf<int> h_mask_, h_nn_;
  Buf<unsigned long long> active_;
  BatchBuffers bb_;
  cudaEvent_t ev_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // prep | propose | walk | replay
  bool timed_ = false;
};

}  // namespace lc
