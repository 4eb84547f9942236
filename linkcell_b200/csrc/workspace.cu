// Launch sequence of one batch and the device workspace around it (the
// cell planning is in plan.cu).
#include "workspace.h"

#include "lc_mlp.h"

#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

namespace lc {

const char *cpu_message(Code c) {
  switch (c) {
    case Code::Ok: return "";
    case Code::NoPoints: return "no points";
    case Code::ZeroK: return "k must be at least 1";
    case Code::NullPointer: return "null pointer";
    case Code::Overflow: return "n * k overflows";
    case Code::BadCell: return "singular or non-positive cell";
    case Code::TooFine: return "linked-cell mesh is too fine";
    case Code::BadCellN: return "device cell must have 3, 9, or 12 doubles";
    case Code::NoDevice: return "no CUDA device available";
    case Code::Cuda: return "CUDA error";
    case Code::DeviceStatus: return "device search failed";
    case Code::TooLarge: return "batch too large for 32-bit indexing";
  }
  return "unknown error";
}

const char *gpu_message(Code c) {
  switch (c) {
    case Code::BadCell: return "bad cell";          // src/gpu/knearest.cpp:731
    case Code::TooFine: return "too many cells";    // src/gpu/knearest.cpp:756
    case Code::NoDevice: return "CUDA driver or nvrtc not loaded";
    default: return cpu_message(c);
  }
}

// Device address of page-locked host memory, or null (pageable, device or
// unknown memory).
void *mapped_host(const void *p) {
  if (!p) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

// ------------------------------------------------------------ workspace
WorkspaceImpl::WorkspaceImpl() {
  // Environment overrides: LINKCELL_MODE (walk mode), LINKCELL_BLOCK
  // (threads per block of the walk), as the reference honours LINKCELL_TPP /
  // LINKCELL_BLOCK (src/gpu/knearest.cpp:948-960).
  if (const char *m = std::getenv("LINKCELL_MODE")) {
    const int v = std::atoi(m);
    if (v >= 0 && v <= 3) opts.mode = v;
  }
  if (const char *t = std::getenv("LINKCELL_TPP")) {
    const int v = std::atoi(t);
    if (v == 1 || v == 32) {
      opts.tpp = v;
      opts.tpp_forced = true;
    }
  }
  if (const char *z = std::getenv("LINKCELL_HOST_ROWS")) {
    const int v = std::atoi(z);
    if (v >= 0 && v <= 2) host_rows_ = v;
  }
  if (const char *b = std::getenv("LINKCELL_BLOCK")) {
    const int v = std::atoi(b);
    if (v == 32 || v == 64 || v == 128 || v == 256) opts.block = v;
  }
  if (const char *g = std::getenv("LINKCELL_GRAB")) {
    const int v = std::atoi(g);
    if (v == 8 || v == 16 || v == 32) opts.sel_grab = v;
  }
  cudaGetDevice(&device_);
  cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking);
  for (auto &e : ev_) cudaEventCreate(&e);
  cudaEventCreateWithFlags(&ev_done_, cudaEventDisableTiming);
}

WorkspaceImpl::~WorkspaceImpl() {
  if (own_) cudaStreamSynchronize(own_);
  if (user_set_ && user_) cudaStreamSynchronize(user_);
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (copy_stream_) {
    cudaStreamSynchronize(copy_stream_);
    cudaStreamDestroy(copy_stream_);
  }
  for (auto &e : range_ev_)
    if (e) cudaEventDestroy(e);
  release_all();
  if (h_frames_) cudaFreeHost(h_frames_);
  if (ev_done_) cudaEventDestroy(ev_done_);
  for (auto &e : ev_)
    if (e) cudaEventDestroy(e);
  if (own_) cudaStreamDestroy(own_);
}

cudaStream_t WorkspaceImpl::stream() { return user_set_ ? user_ : own_; }

void WorkspaceImpl::set_stream(cudaStream_t s) {
  user_ = s;
  user_set_ = s != nullptr;
}

Code WorkspaceImpl::wait(std::string &detail) {
  const cudaError_t e = cudaStreamSynchronize(stream());
  if (e != cudaSuccess) {
    detail = cudaGetErrorString(e);
    return Code::Cuda;
  }
  if (!done_pending_) return Code::Ok;
  // the last batch ran without a wait: its status word is reported here
  done_pending_ = false;
  return read_status(detail);
}

template <class T>
cudaError_t WorkspaceImpl::grow(Buf<T> &b, size_t n) {
  if (n <= b.cap && b.p) return cudaSuccess;
  size_t want = std::max<size_t>(n, 16);
  want = want + want / 8;  // headroom against small repeated growth
  if (b.p) {
    // the previous batch may still read the old buffer on another stream
    if (last_stream_ && last_stream_ != stream()) {
      cudaError_t se = cudaStreamSynchronize(last_stream_);
      if (se != cudaSuccess) return se;
    }
    cudaError_t e = cudaFreeAsync(b.p, stream());
    if (e != cudaSuccess) return e;
    b.p = nullptr;
    b.cap = 0;
  }
  void *p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, want * sizeof(T), stream());
  if (e != cudaSuccess) return e;
  b.p = static_cast<T *>(p);
  b.cap = want;
  return cudaSuccess;
}

void WorkspaceImpl::release_all() {
  auto rel = [&](auto &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
  };
  rel(cell_of_); rel(arank_); rel(tmp_); rel(count_); rel(off_); rel(tile_counter_);
  rel(work_); rel(replay_count_); rel(tile_state_); rel(status_); rel(frame_flags_);
  rel(sidx_); rel(replay_list_); rel(replay_i_); rel(scell_); rel(sx_); rel(sy_); rel(sz_);
  rel(replay_d_); rel(rec_); rel(frames_); rel(counters_); rel(h_xyz_); rel(h_d2_);
  rel(h_mask_); rel(h_nn_); rel(active_); rel(proposal_); rel(cell_prop_); rel(stop_log_);
  rel(order_); rel(csr_counts_); rel(csr_off_); rel(live_); rel(part_cnt_); rel(part_off_);
  rel(part_tiles_); rel(shard_cut_);
  rel(model_); rel(model_image_); rel(shell_table_); rel(syz_);
  shell_table_ready_ = false;
}

#define LC_TRY(expr)                        \
  do {                                      \
    const cudaError_t e_ = (expr);          \
    if (e_ != cudaSuccess) {                \
      detail = cudaGetErrorString(e_);      \
      return Code::Cuda;                    \
    }                                       \
  } while (0)

Code WorkspaceImpl::run(std::vector<FrameDesc> &frames, const double *xyz, const int *mask,
                        int *out_nn, double *out_d2, bool wait, std::string &detail) {
  const int nf = int(frames.size());
  long long npts = 0, ncells = 0, ptiles = 0;
  int kmax = 1;
  for (auto &fd : frames) {
    fd.pt_base = npts;
    fd.cell_base = ncells;
    fd.tile_base = ptiles;  // shell-proposal tiles
    ptiles += proposal_tiles(fd.nx, fd.ny, fd.nz);
    npts += fd.n;
    ncells += (long long)fd.nx * fd.ny * fd.nz;
    kmax = std::max(kmax, fd.k);
  }
  // 32-bit point ids and cell ids (kInactive is reserved)
  if (npts >= 0xFFFFFFF0LL || ncells >= 0xFFFFFFF0LL) return Code::TooLarge;
  const cudaStream_t s = stream();
  const size_t P = size_t(npts), C = size_t(ncells);
  struct LastStream {
    cudaStream_t &slot, s;
    ~LastStream() { slot = s; }
  } last_guard{last_stream_, s};
  const long long tiles = scan_tiles(ncells);

  // ---- 1. buffers (grow-only; nothing is allocated once they fit)
  LC_TRY(grow(cell_of_, P));
  LC_TRY(grow(arank_, P));
  LC_TRY(grow(tmp_, P));
  LC_TRY(grow(count_, C));
  LC_TRY(grow(off_, C + 1));
  LC_TRY(grow(tile_state_, size_t(tiles)));
  LC_TRY(grow(tile_counter_, 1));
  LC_TRY(grow(work_, 1));
  LC_TRY(grow(replay_count_, 1));
  LC_TRY(grow(status_, 1));
  LC_TRY(grow(frame_flags_, size_t(nf)));
  LC_TRY(grow(sidx_, P));
  LC_TRY(grow(scell_, P));
  LC_TRY(grow(sx_, P));
  LC_TRY(grow(sy_, P));
  LC_TRY(grow(sz_, P));
  LC_TRY(grow(rec_, P));
  LC_TRY(grow(replay_list_, P));
  LC_TRY(grow(frames_, size_t(nf)));
  LC_TRY(grow(counters_, size_t(kNumCounters)));
  if (dcell_.on) LC_TRY(grow(live_, 1));
  if (opts.log_shells) LC_TRY(grow(stop_log_, P));
  if (opts.mode == kModeLearned && !has_model_ && opts.fixed_proposal <= 0 && !model_tried_) {
    model_tried_ = true;
    load_default_model();  // the shipped network, when it can be found
  }
  // without a network (or fixed proposal) the learned mode is the FP32 walk
  const bool learned =
      opts.mode == kModeLearned && kmax <= 256 && (opts.fixed_proposal > 0 || has_model_);
  if (learned) {
    LC_TRY(grow(proposal_, P));
    LC_TRY(grow(syz_, P));
    if (opts.fixed_proposal <= 0 && has_model_) LC_TRY(grow(cell_prop_, C));
  }
  if (!shell_table_ready_) {
    const int rmax = kShellTableRmax;
    const size_t entries = size_t(2 * rmax + 1) * (2 * rmax + 1) * (2 * rmax + 1);
    std::vector<uint32_t> h(entries);
    build_shell_table(rmax, h.data());
    LC_TRY(grow(shell_table_, entries));
    LC_TRY(cudaMemcpyAsync(shell_table_.p, h.data(), entries * sizeof(uint32_t),
                           cudaMemcpyHostToDevice, s));
    LC_TRY(cudaStreamSynchronize(s));
    shell_table_ready_ = true;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
  const int replay_threads = int(std::min<long long>(
      std::max<long long>(1, npts), std::max<long long>(sms * 32, std::min<long long>(
                                                                     sms * 256,
                                                                     (256LL << 20) / (kmax * 12)))));
  LC_TRY(grow(replay_d_, size_t(replay_threads) * kmax));
  LC_TRY(grow(replay_i_, size_t(replay_threads) * kmax));
  // pinned staging of the frame table (the previous batch may still read it)
  if (done_pending_) {
    LC_TRY(cudaEventSynchronize(ev_done_));
    done_pending_ = false;
  }
  if (size_t(nf) > h_frames_cap_) {
    if (h_frames_) cudaFreeHost(h_frames_);
    h_frames_ = nullptr;
    h_frames_cap_ = 0;
    void *hp = nullptr;
    LC_TRY(cudaMallocHost(&hp, sizeof(FrameDesc) * size_t(nf) * 2));
    h_frames_ = static_cast<FrameDesc *>(hp);
    h_frames_cap_ = size_t(nf) * 2;
  }
  std::memcpy(h_frames_, frames.data(), sizeof(FrameDesc) * size_t(nf));

  // ---- 2. device view of the batch
  BatchBuffers &b = bb_;
  b = BatchBuffers();
  b.xyz = xyz;
  b.mask = mask;
  b.frames = frames_.p;
  b.nframes = nf;
  b.npts = npts;
  b.ncells = ncells;
  b.live_cells = dcell_.on ? live_.p : nullptr;
  b.cell_of = cell_of_.p;
  b.arank = arank_.p;
  b.tmp = tmp_.p;
  b.count = count_.p;
  b.off = off_.p;
  b.tile_state = tile_state_.p;
  b.tile_counter = tile_counter_.p;
  b.status = status_.p;
  b.frame_flags = frame_flags_.p;
  b.sx = sx_.p;
  b.sy = sy_.p;
  b.sz = sz_.p;
  b.sidx = sidx_.p;
  b.scell = scell_.p;
  b.rec = rec_.p;
  b.syz = learned ? syz_.p : nullptr;
  b.out_nn = out_nn;
  b.out_d2 = out_d2;
  b.work = work_.p;
  b.replay_list = replay_list_.p;
  b.replay_count = replay_count_.p;
  b.replay_cap = npts;
  b.replay_d = replay_d_.p;
  b.replay_i = replay_i_.p;
  b.replay_threads = replay_threads;
  b.kmax = kmax;
  b.counters = counters_.p;
  b.shell_table = shell_table_.p;
  b.shell_rmax = kShellTableRmax;
  b.stop_log = opts.log_shells ? stop_log_.p : nullptr;
  b.proposal = learned ? proposal_.p : nullptr;
  b.scan_spin_limit = opts.scan_spin_limit;
  b.scan_silent_tile = opts.scan_silent_tile;

  // ---- 3. walk configuration: overrides, else the autotuned choice
  WalkLaunch wl;
  wl.mode = kmax > 256 ? int(kModeReplayAll) : opts.mode;
  wl.kmax = kmax;
  wl.prune = opts.prune;
  wl.stats = opts.stats;
  // a single host-planned frame goes to the select walk as a kernel
  // parameter (not under a graph: its replays would keep the captured copy)
  wl.one = nf == 1 && !dcell_.on && !opts.graph;
  if (wl.one) wl.frame1 = frames[0];
  const int kclass = kmax <= 32 ? 0 : (kmax <= 64 ? 1 : (kmax <= 128 ? 2 : 3));
  const int tkey = (wl.mode * 4 + kclass) * 2 + (nf > 1 ? 1 : 0);
  const bool select = wl.mode == kModeLearned && kmax <= 64 && learned;  // the cube select walk
  auto set_shape = [&](const WalkShape &sh) {
    wl.tpp = sh.tpp;
    const int maxblk = walk_max_block(wl.mode, kmax);
    wl.block = opts.block > 0 ? std::min(opts.block, maxblk) : maxblk;
    wl.warps = sh.warps;
    wl.grab = sh.grab;
  };
  bool done = false;  // the batch's results are already in place
  const bool forced = opts.tpp_forced || opts.sel_warps > 0 || opts.sel_grab > 0;
  if (forced || !opts.autotune || wl.mode == kModeReplayAll) {
    // overrides (API or LINKCELL_TPP / LINKCELL_BLOCK / LINKCELL_GRAB); the
    // rest at its default
    int warps = opts.sel_warps;
    if (warps == 0 && opts.block > 0 && select &&
        (opts.block / 32 == sel_warps_for(kmax, 0) || opts.block / 32 == sel_warps_for(kmax, 1)))
      warps = opts.block / 32;
    set_shape(WalkShape{opts.tpp_forced ? opts.tpp : 32, warps, opts.sel_grab});
  } else if (tuned_.count(tkey)) {
    set_shape(tuned_[tkey]);
  } else {
    // time every candidate design and shape once on this batch (their
    // results are identical) and keep the fastest for every later batch of
    // this kind: warp per source (for the select walk, in two block sizes and
    // three work-grab sizes) and thread per source
    std::vector<WalkShape> cand;
    if (select)
      for (int wi = 0; wi < 2; ++wi)
        for (int g : kSelGrabs) cand.push_back(WalkShape{32, sel_warps_for(kmax, wi), g});
    else
      cand.push_back(WalkShape{32, 0, 0});
    cand.push_back(WalkShape{1, 0, 0});
    std::vector<float> ms(cand.size(), 0.f);
    const bool piping = pipe_.on;
    pipe_.on = false;  // the trials run whole searches
    for (size_t c = 0; c < cand.size(); ++c) {
      set_shape(cand[c]);
      const Code rc = enqueue(b, wl, nf, C, tiles, s, true, detail);
      if (rc != Code::Ok) return rc;
      LC_TRY(cudaEventSynchronize(ev_[3]));
      LC_TRY(cudaEventElapsedTime(&ms[c], ev_[1], ev_[2]));
    }
    pipe_.on = piping;
    size_t best = 0;
    for (size_t c = 1; c < cand.size(); ++c)
      if (ms[c] < ms[best]) best = c;
    tuned_[tkey] = cand[best];
    set_shape(cand[best]);
    trial_shapes_ = cand;
    done = best + 1 == cand.size() && !opts.graph;  // the last run used the winner
    if (!done && !opts.graph) {
      const Code rc = enqueue(b, wl, nf, C, tiles, s, collect_stats, detail);
      if (rc != Code::Ok) return rc;
      done = true;
    }
    timed_ = true;
    graph_total_ = false;
  }
  last_tpp = wl.tpp;
  last_shape = WalkShape{wl.tpp,
                         wl.tpp == 32 && select ? (wl.warps ? wl.warps : sel_warps_for(kmax, 0)) : 0,
                         wl.tpp == 32 && select ? (wl.grab ? wl.grab : 16) : 0};

  // ---- 4. enqueue: direct launches, or a CUDA graph replayed while the
  // batch signature (sizes, pointers, configuration) stays the same
  if (done) {
    // autotuning left this batch's results and stats in place
  } else if (opts.graph) {
    const GraphKey key{npts, ncells, nf, kmax, xyz, mask, out_nn, out_d2, wl.mode, wl.tpp,
                       wl.block + 1024 * wl.warps + 65536 * wl.grab, has_model_ ? 1 : 0,
                       opts.fixed_proposal, opts.log_shells,
                       opts.stats ? 1 : 0, dcell_.on ? dcell_.cell : nullptr,
                       dcell_.on ? dcell_.cell_n : 0,
                       dcell_.on ? dcell_.hint : 0.0, opts.scan_spin_limit,
                       opts.scan_silent_tile};
    if (!graph_exec_ || !(key == graph_key_)) {
      if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
      graph_exec_ = nullptr;
      cudaGraph_t g = nullptr;
      LC_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const Code c = enqueue(b, wl, nf, C, tiles, s, false, detail);
      const cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (c != Code::Ok) {
        if (g) cudaGraphDestroy(g);
        return c;
      }
      LC_TRY(ce);
      const cudaError_t ie = cudaGraphInstantiate(&graph_exec_, g, 0);
      cudaGraphDestroy(g);
      LC_TRY(ie);
      graph_key_ = key;
      ++graph_captures;
    }
    LC_TRY(cudaEventRecord(ev_[0], s));
    LC_TRY(cudaGraphLaunch(graph_exec_, s));
    LC_TRY(cudaEventRecord(ev_[3], s));
    timed_ = false;
    graph_total_ = true;
  } else {
    const Code c = enqueue(b, wl, nf, C, tiles, s, collect_stats, detail);
    if (c != Code::Ok) return c;
    timed_ = collect_stats;
    graph_total_ = false;
  }
  LC_TRY(cudaEventRecord(ev_done_, s));
  done_pending_ = true;
  if (!wait) return Code::Ok;
  LC_TRY(cudaStreamSynchronize(s));
  done_pending_ = false;
  return read_status(detail);
}

Code WorkspaceImpl::read_status(std::string &detail) {
  if (!status_.p) return Code::Ok;
  int st = 0;
  LC_TRY(cudaMemcpy(&st, status_.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (st & kStatusPlanBadCell) return Code::BadCell;
  if (st & kStatusPlanTooFine) return Code::TooFine;
  if (st != 0) {
    detail = "device status " + std::to_string(st);
    return Code::DeviceStatus;
  }
  return Code::Ok;
}

Code WorkspaceImpl::too_fine_masked(const int *mask, long long n, int *out_nn, double *out_d2,
                                    long long need, bool wait, std::string &detail) {
  const cudaStream_t s = stream();
  if (done_pending_) {
    LC_TRY(cudaEventSynchronize(ev_done_));
    done_pending_ = false;
  }
  LC_TRY(grow(active_, 1));
  LC_TRY(grow(status_, 1));
  LC_TRY(cudaMemsetAsync(status_.p, 0, sizeof(int), s));
  LC_TRY(launch_masked_too_fine(mask, n, active_.p, out_nn, out_d2, need, status_.p, s));
  LC_TRY(cudaEventRecord(ev_done_, s));
  last_stream_ = s;
  done_pending_ = true;
  if (!wait) return Code::Ok;
  LC_TRY(cudaStreamSynchronize(s));
  done_pending_ = false;
  return read_status(detail);
}

Code WorkspaceImpl::run_shard(std::vector<FrameDesc> &frames, const double *xyz, const int *mask,
                              int *out_nn, double *out_d2, int *owned, int rank, int world,
                              bool wait, std::string &detail) {
  if (world < 1 || rank < 0 || rank >= world || !owned) return Code::NullPointer;
  long long P = 0;
  for (const auto &fd : frames) P += fd.n;
  LC_TRY(grow(part_cnt_, size_t(P)));
  LC_TRY(grow(part_off_, size_t(P) + 1));
  LC_TRY(grow(part_tiles_, size_t(scan_tiles(P))));
  LC_TRY(grow(shard_cut_, 2));
  const bool graph = opts.graph;
  opts.graph = false;
  shard_ = Shard{true, rank, world, owned};
  const Code c = run(frames, xyz, mask, out_nn, out_d2, wait, detail);
  shard_ = Shard();
  opts.graph = graph;
  return c;
}

Code WorkspaceImpl::walk_shard(BatchBuffers &b, const WalkLaunch &wl, cudaStream_t s, bool timed,
                               std::string &detail) {
  LC_TRY(launch_shard_split(b, shard_.rank, shard_.world, part_cnt_.p, part_off_.p, part_tiles_.p,
                            tile_counter_.p, shard_cut_.p, s));
  if (timed) LC_TRY(cudaEventRecord(ev_[4], s));
  BatchBuffers br = b;
  br.src_lo = shard_cut_.p;
  br.src_hi = shard_cut_.p + 1;
  LC_TRY(launch_walk(br, wl, s));
  if (timed) LC_TRY(cudaEventRecord(ev_[2], s));
  LC_TRY(launch_replay(br, s, wl.one ? &wl.frame1 : nullptr));
  LC_TRY(launch_shard_owned(b, shard_cut_.p, shard_.rank, shard_.owned, s));
  if (timed) LC_TRY(cudaEventRecord(ev_[3], s));
  return Code::Ok;
}

Code WorkspaceImpl::run_device_cell(const double *cell, int cell_n, long long n, int nframes,
                                    int k, double hint, const double *xyz, const int *mask,
                                    int *out_nn, double *out_d2, bool wait, std::string &detail) {
  if (nframes < 1 || nframes > kDeviceCellFrames) return Code::TooLarge;
  // host-side placeholders: sizes only; the device planner writes the table
  std::vector<FrameDesc> frames(static_cast<size_t>(nframes));
  for (auto &fd : frames) {
    std::memset(&fd, 0, sizeof(fd));
    fd.n = n;
    fd.k = k;
    fd.nx = int(kMaxCellsPerFrame);
    fd.ny = fd.nz = 1;
    fd.has_mask = mask ? 1 : 0;
  }
  dcell_ = DeviceCell{true, cell, cell_n, n, nframes, k, hint};
  const Code c = run(frames, xyz, mask, out_nn, out_d2, wait, detail);
  dcell_.on = false;
  return c;
}

Code WorkspaceImpl::enqueue(BatchBuffers &b, const WalkLaunch &wl, int nf, size_t C,
                            long long tiles, cudaStream_t s, bool timed, std::string &detail) {
  if (!dcell_.on) {
    LC_TRY(cudaMemcpyAsync(frames_.p, h_frames_, sizeof(FrameDesc) * size_t(nf),
                           cudaMemcpyHostToDevice, s));
    LC_TRY(cudaMemsetAsync(count_.p, 0, C * sizeof(uint32_t), s));
    LC_TRY(cudaMemsetAsync(tile_state_.p, 0, size_t(tiles) * sizeof(unsigned long long), s));
  }
  LC_TRY(cudaMemsetAsync(tile_counter_.p, 0, sizeof(uint32_t), s));
  LC_TRY(cudaMemsetAsync(work_.p, 0, sizeof(uint32_t), s));
  LC_TRY(cudaMemsetAsync(replay_count_.p, 0, sizeof(uint32_t), s));
  LC_TRY(cudaMemsetAsync(status_.p, 0, sizeof(int), s));
  LC_TRY(cudaMemsetAsync(frame_flags_.p, 0, sizeof(int) * size_t(nf), s));
  LC_TRY(cudaMemsetAsync(counters_.p, 0, sizeof(long long) * kNumCounters, s));
  if (timed) LC_TRY(cudaEventRecord(ev_[0], s));
  if (dcell_.on) {
    // the frame table and the live cell count come from the device cell
    LC_TRY(launch_plan_device_cell(dcell_.cell, dcell_.cell_n, dcell_.n, dcell_.nframes, dcell_.k,
                                   dcell_.hint, b.mask, frames_.p, live_.p, status_.p, s));
    LC_TRY(launch_zero_live(b, s));
  }
  const FrameDesc *one = wl.one ? &wl.frame1 : nullptr;
  LC_TRY(launch_fold_bin(b, s, one));
  LC_TRY(launch_scan(b, s));
  LC_TRY(launch_place(b, s, one));
  if (timed) LC_TRY(cudaEventRecord(ev_[1], s));
  if (b.proposal) {
    // shell proposals per sorted source (part of the walk phase)
    const size_t P = size_t(b.npts);
    if (opts.fixed_proposal > 0) {
      LC_TRY(cudaMemsetAsync(proposal_.p, std::min(opts.fixed_proposal, 127), P, s));
    } else if (has_model_) {
      LC_TRY(mlp_propose(model_image_.p, b, cell_prop_.p, proposal_.p, tau_, s));
    } else {
      LC_TRY(cudaMemsetAsync(proposal_.p, 0, P, s));
    }
  }
  if (pipe_.on && !pipe_.done) return walk_in_row_ranges(b, wl, s, timed, detail);
  if (shard_.on) return walk_shard(b, wl, s, timed, detail);
  if (timed) LC_TRY(cudaEventRecord(ev_[4], s));
  LC_TRY(launch_walk(b, wl, s));
  if (timed) LC_TRY(cudaEventRecord(ev_[2], s));
  LC_TRY(launch_replay(b, s, wl.one ? &wl.frame1 : nullptr));
  if (timed) LC_TRY(cudaEventRecord(ev_[3], s));
  return Code::Ok;
}

// The shipped shell-proposal network: LINKCELL_MODEL, else data/shell_mlp.f32
// beside this shared library. File: "LCMLP001", i32 n, f32 tau, i32 meta
// length, meta bytes, n f32 parameters (little-endian).
bool WorkspaceImpl::load_default_model() {
  std::string path;
  if (const char *e = std::getenv("LINKCELL_MODEL")) {
    path = e;
  } else {
    Dl_info info;
    if (!dladdr(reinterpret_cast<void *>(&mapped_host), &info) || !info.dli_fname) return false;
    path = info.dli_fname;
    const size_t slash = path.rfind('/');
    path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) +
           "/data/shell_mlp.f32";
  }
  FILE *fh = std::fopen(path.c_str(), "rb");
  if (!fh) return false;
  char magic[8];
  int32_t n = 0, ml = 0;
  float tau = 0.f;
  bool ok = std::fread(magic, 1, 8, fh) == 8 && std::memcmp(magic, "LCMLP001", 8) == 0 &&
            std::fread(&n, 4, 1, fh) == 1 && std::fread(&tau, 4, 1, fh) == 1 &&
            std::fread(&ml, 4, 1, fh) == 1 && n == kMlpParams && ml >= 0 && ml < (1 << 20) &&
            std::fseek(fh, ml, SEEK_CUR) == 0;
  std::vector<float> params(ok ? size_t(n) : 0);
  ok = ok && std::fread(params.data(), 4, size_t(n), fh) == size_t(n);
  std::fclose(fh);
  if (!ok || !(tau > 0.f && tau <= 1.f)) return false;
  std::string detail;
  return set_model(params.data(), params.size(), tau, detail) == Code::Ok;
}

Code WorkspaceImpl::set_model(const float *params, size_t n, float tau, std::string &detail) {
  if (n != size_t(kMlpParams)) {
    detail = "model must have " + std::to_string(kMlpParams) + " parameters";
    return Code::DeviceStatus;
  }
  LC_TRY(grow(model_, n));
  LC_TRY(grow(model_image_, (mlp_image_bytes() + 15) / 16));
  LC_TRY(cudaMemcpyAsync(model_.p, params, n * sizeof(float), cudaMemcpyHostToDevice, stream()));
  LC_TRY(mlp_pack(model_.p, model_image_.p, stream()));
  LC_TRY(cudaStreamSynchronize(stream()));
  has_model_ = true;
  tau_ = tau;
  return Code::Ok;
}

Code WorkspaceImpl::training_rows(float *X, int *y, long long cap, long long stride,
                                  long long first, long long &rows, std::string &detail) {
  rows = 0;
  if (!bb_.stop_log || !bb_.off) {
    detail = "no logged search";
    return Code::DeviceStatus;
  }
  uint32_t total = 0;
  LC_TRY(cudaStreamSynchronize(stream()));
  LC_TRY(cudaMemcpy(&total, bb_.off + bb_.ncells, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (stride < 1) stride = 1;
  if (first < 0 || first >= (long long)total) return Code::Ok;
  const long long avail = ((long long)total - first + stride - 1) / stride;
  rows = std::min(avail, cap);
  LC_TRY(mlp_training_rows(bb_, bb_.stop_log, stride, first, X, y, rows, stream()));
  LC_TRY(cudaStreamSynchronize(stream()));
  return Code::Ok;
}

Code WorkspaceImpl::proposals(int8_t *out, long long cap, long long stride, long long first,
                              long long &rows, std::string &detail) {
  rows = 0;
  if (!bb_.proposal || !bb_.off) {
    detail = "no learned search";
    return Code::DeviceStatus;
  }
  uint32_t total = 0;
  LC_TRY(cudaStreamSynchronize(stream()));
  LC_TRY(cudaMemcpy(&total, bb_.off + bb_.ncells, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (stride < 1) stride = 1;
  if (first < 0 || first >= (long long)total) return Code::Ok;
  const long long avail = ((long long)total - first + stride - 1) / stride;
  rows = std::min(avail, cap);
  LC_TRY(cudaMemcpy2D(out, 1, bb_.proposal + first, size_t(stride), 1, size_t(rows),
                      cudaMemcpyDeviceToHost));
  return Code::Ok;
}

Code WorkspaceImpl::fetch_stats(Stats &out, std::string &detail) {
  out = Stats();
  if (!counters_.p) return Code::Ok;
  if (graph_total_) {
    LC_TRY(cudaEventSynchronize(ev_[3]));
    float t = 0.f;
    LC_TRY(cudaEventElapsedTime(&t, ev_[0], ev_[3]));
    out.ms_total = t;
  } else if (timed_) {
    LC_TRY(cudaEventSynchronize(ev_[3]));
    float a = 0.f, b = 0.f, c = 0.f, t = 0.f, q = 0.f;
    LC_TRY(cudaEventElapsedTime(&a, ev_[0], ev_[1]));
    LC_TRY(cudaEventElapsedTime(&b, ev_[1], ev_[2]));
    LC_TRY(cudaEventElapsedTime(&c, ev_[2], ev_[3]));
    LC_TRY(cudaEventElapsedTime(&t, ev_[0], ev_[3]));
    LC_TRY(cudaEventElapsedTime(&q, ev_[1], ev_[4]));
    out.ms_prep = a;
    out.ms_walk = b;
    out.ms_propose = q;
    out.ms_replay = c;
    out.ms_total = t;
  } else {
    LC_TRY(cudaStreamSynchronize(stream()));
  }
  LC_TRY(cudaMemcpy(out.counters, counters_.p, sizeof(long long) * kNumCounters,
                    cudaMemcpyDeviceToHost));
  return Code::Ok;
}

Code WorkspaceImpl::run_host(std::vector<FrameDesc> &frames, const double *xyz, size_t xyz_n,
                             const int *mask, size_t mask_n, int *out_nn, double *out_d2,
                             size_t out_n, std::string &detail) {
  const cudaStream_t s = stream();
  // Output rows land in a random order, so a finished search cannot be
  // copied back in pieces while it runs. With page-locked output buffers
  // the search is cut into row ranges instead: the walk visits the sources
  // of one range of output rows at a time (in cell order inside the range)
  // and a copy engine brings each finished range back while the next one is
  // searched (host_rows 1, the default). host_rows 2 has the kernels write
  // the rows straight into the mapped host buffers; pageable buffers (or
  // host_rows 0) take one copy back at the end.
  const bool locked = mapped_host(out_nn) && (!out_d2 || mapped_host(out_d2));
  const int how = locked ? host_rows_ : 0;
  int *map_nn = nullptr;
  double *map_d2 = nullptr;
  if (how == 2) {
    map_nn = static_cast<int *>(mapped_host(out_nn));
    map_d2 = out_d2 ? static_cast<double *>(mapped_host(out_d2)) : nullptr;
  }
  LC_TRY(grow(h_xyz_, xyz_n));
  if (!map_nn) {
    LC_TRY(grow(h_nn_, out_n));
    if (out_d2) LC_TRY(grow(h_d2_, out_n));
  }
  if (mask) LC_TRY(grow(h_mask_, mask_n));
  LC_TRY(cudaMemcpyAsync(h_xyz_.p, xyz, xyz_n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (mask)
    LC_TRY(cudaMemcpyAsync(h_mask_.p, mask, mask_n * sizeof(int), cudaMemcpyHostToDevice, s));
  pipe_ = Pipe();
  if (how == 1 && !opts.graph) {
    pipe_.on = true;
    pipe_.host_nn = out_nn;
    pipe_.host_d2 = out_d2;
  }
  const Code c = run(frames, h_xyz_.p, mask ? h_mask_.p : nullptr, map_nn ? map_nn : h_nn_.p,
                     out_d2 ? (map_nn ? map_d2 : h_d2_.p) : nullptr, false, detail);
  const bool piped = pipe_.done;
  pipe_ = Pipe();
  if (c != Code::Ok) return c;
  last_host_rows = map_nn ? 2 : (piped ? 1 : 0);
  if (!map_nn && !piped) {
    LC_TRY(cudaMemcpyAsync(out_nn, h_nn_.p, out_n * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (out_d2)
      LC_TRY(cudaMemcpyAsync(out_d2, h_d2_.p, out_n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  LC_TRY(cudaStreamSynchronize(s));
  done_pending_ = false;
  return read_status(detail);
}

Code WorkspaceImpl::neighbors_within(const int *nn, const double *d2, size_t rows, size_t k,
                                     double cutoff, int *row_ptr, int *col, double *dist2,
                                     size_t cap, size_t &nnz, std::string &detail) {
  nnz = 0;
  if (rows == 0) return Code::Ok;
  if (rows * k >= size_t(0x7fffffff)) return Code::TooLarge;
  const cudaStream_t s = stream();
  LC_TRY(grow(csr_counts_, rows));
  LC_TRY(grow(csr_off_, rows + 1));
  LC_TRY(grow(tile_state_, size_t(scan_tiles((long long)rows))));
  LC_TRY(grow(tile_counter_, 1));
  LC_TRY(grow(status_, 1));
  LC_TRY(cudaMemsetAsync(status_.p, 0, sizeof(int), s));
  LC_TRY(launch_csr(nn, d2, (long long)rows, int(k), cutoff, csr_counts_.p, csr_off_.p,
                    tile_state_.p, tile_counter_.p, status_.p, row_ptr, col, dist2,
                    (long long)cap, s));
  int total = 0, st = 0;
  LC_TRY(cudaMemcpyAsync(&total, row_ptr + rows, sizeof(int), cudaMemcpyDeviceToHost, s));
  LC_TRY(cudaMemcpyAsync(&st, status_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  LC_TRY(cudaStreamSynchronize(s));
  if (st != 0) {
    detail = "device status " + std::to_string(st);
    return Code::DeviceStatus;
  }
  nnz = size_t(total);
  return Code::Ok;
}

// The walk and replay of run_host's pipelined path: row range r of the
// output goes back on the copy stream as soon as its sources are done.
Code WorkspaceImpl::walk_in_row_ranges(BatchBuffers &b, const WalkLaunch &wl, cudaStream_t s,
                                       bool timed, std::string &detail) {
  const long long rows = b.npts;
  // First output element of point row r (frames are contiguous in points and
  // in outputs, each with its own k), from the host copy of the frame table.
  const int nf = b.nframes;
  auto elem_at = [&](long long r) -> size_t {
    int lo = 0, hi = nf - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (h_frames_[mid].pt_base <= r)
        lo = mid;
      else
        hi = mid - 1;
    }
    const FrameDesc &f = h_frames_[lo];
    return size_t(f.out_base + std::min<long long>(r - f.pt_base, f.n) * f.k);
  };
  // The copy engine starts after a short first range (1/32 of the rows).
  // Later ranges double, so each is walked before the copies ahead of it
  // finish, up to 1/8 of the rows, so that little is left to copy after the
  // last walk when the walk is about as long as the copy. 4M rows: 1/32,
  // 1/32, 1/16, then 1/8 each (measured against eight equal ranges and
  // geometric ranges up to 1/2).
  RowCuts rc;
  rc.nr = 0;
  rc.cut[0] = 0;
  const long long first = std::max<long long>(rows / 32, kMinRangeRows);
  const long long cap = std::max<long long>(rows / 8, first);
  while (rc.cut[rc.nr] < rows) {
    const long long len =
        rc.nr == 0 ? first : std::min(cap, std::max(first, rc.cut[rc.nr]));
    rc.cut[rc.nr + 1] = rc.nr + 1 == kMaxRowRanges ? rows : std::min(rows, rc.cut[rc.nr] + len);
    ++rc.nr;
  }
  for (int r = rc.nr + 1; r <= kMaxRowRanges; ++r) rc.cut[r] = rows;
  // each range's sources in cell order (the walk's locality), found on the device
  const long long nblk = range_partition_blocks(rows);
  const size_t L = size_t(rc.nr) * size_t(nblk);
  LC_TRY(grow(order_, size_t(rows)));
  LC_TRY(grow(part_cnt_, L));
  LC_TRY(grow(part_off_, L + 1));
  LC_TRY(grow(part_tiles_, size_t(scan_tiles((long long)L))));
  if (!copy_stream_) LC_TRY(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
  for (auto &e : range_ev_)
    if (!e) LC_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  LC_TRY(launch_range_partition(b, rc, part_cnt_.p, part_off_.p, part_tiles_.p, tile_counter_.p,
                                order_.p, s));
  if (timed) LC_TRY(cudaEventRecord(ev_[4], s));
  for (int r = 0; r < rc.nr; ++r) {
    const long long r0 = rc.cut[r], r1 = rc.cut[r + 1];
    BatchBuffers br = b;
    br.src_order = order_.p;
    br.src_lo = part_off_.p + size_t(r) * size_t(nblk);
    br.src_hi = part_off_.p + size_t(r + 1) * size_t(nblk);
    LC_TRY(cudaMemsetAsync(work_.p, 0, sizeof(uint32_t), s));
    LC_TRY(cudaMemsetAsync(replay_count_.p, 0, sizeof(uint32_t), s));
    LC_TRY(launch_walk(br, wl, s));
    LC_TRY(launch_replay(br, s, wl.one ? &wl.frame1 : nullptr));
    LC_TRY(cudaEventRecord(range_ev_[r], s));
    LC_TRY(cudaStreamWaitEvent(copy_stream_, range_ev_[r], 0));
    const size_t e0 = elem_at(r0), ne = elem_at(r1) - e0;
    LC_TRY(cudaMemcpyAsync(pipe_.host_nn + e0, b.out_nn + e0, ne * sizeof(int),
                           cudaMemcpyDeviceToHost, copy_stream_));
    if (pipe_.host_d2)
      LC_TRY(cudaMemcpyAsync(pipe_.host_d2 + e0, b.out_d2 + e0, ne * sizeof(double),
                             cudaMemcpyDeviceToHost, copy_stream_));
  }
  if (timed) LC_TRY(cudaEventRecord(ev_[2], s));
  if (timed) LC_TRY(cudaEventRecord(ev_[3], s));
  // the caller's stream finishes only once every range is back
  LC_TRY(cudaEventRecord(range_ev_[rc.nr], copy_stream_));
  LC_TRY(cudaStreamWaitEvent(s, range_ev_[rc.nr], 0));
  pipe_.done = true;
  (void)detail;
  return Code::Ok;
}

}  // namespace lc
