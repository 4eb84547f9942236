// The exported C ABI (include/linkcell.h, include/linkcell_gpu.h) and the
// C++ class linkcell::gpu::Workspace (include/linkcell_gpu.hpp).
//
// Validation order and messages follow the reference: the CPU ABI
// src/capi.rs:184-259 for lc_knearest*, the device ABI src/gpu/capi.cpp and
// src/gpu/knearest.cpp:705-878 for lc_gpu_*.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/linkcell.h"
#include "../../include/linkcell_gpu.h"
#include "../../include/linkcell_gpu.hpp"
#include "lc_mlp.h"
#include "workspace.h"

namespace {

using lc::Code;
using lc::FrameDesc;
using lc::WorkspaceImpl;

thread_local std::string t_cpu_err;
thread_local bool t_cpu_has_err = false;
thread_local std::string t_gpu_err;

int cpu_fail(Code c, const std::string &detail = std::string()) {
  t_cpu_err = lc::cpu_message(c);
  if (!detail.empty() && (c == Code::Cuda || c == Code::DeviceStatus)) t_cpu_err += ": " + detail;
  t_cpu_has_err = true;
  return 1;
}
void cpu_ok() {
  t_cpu_err.clear();
  t_cpu_has_err = false;
}
int gpu_fail(Code c, const std::string &detail = std::string()) {
  t_gpu_err = lc::gpu_message(c);
  if (!detail.empty() && (c == Code::Cuda || c == Code::DeviceStatus)) t_gpu_err += ": " + detail;
  return 1;
}
int gpu_fail_msg(const std::string &m) {
  t_gpu_err = m;
  return 1;
}
void gpu_ok() { t_gpu_err.clear(); }

bool device_present() {
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the sticky "no device" error
    return false;
  }
  return n > 0;
}

// Per-thread workspace of the host-pointer ABI.
WorkspaceImpl &host_workspace() {
  thread_local std::unique_ptr<WorkspaceImpl> ws;
  if (!ws) ws.reset(new WorkspaceImpl());
  return *ws;
}

void rows_of(const lc_cell &c, double rows[9], double origin[3]) {
  rows[0] = c.ax; rows[1] = c.ay; rows[2] = c.az;
  rows[3] = c.bx; rows[4] = c.by; rows[5] = c.bz;
  rows[6] = c.cx; rows[7] = c.cy; rows[8] = c.cz;
  origin[0] = c.ox; origin[1] = c.oy; origin[2] = c.oz;
}

// Cell-only check of Cell::from_vectors (src/cell.rs:97-124); the mesh is
// checked separately because an all-masked search never reaches it
// (src/knearest.rs:370-375).
Code check_cell(const lc_cell &c) {
  double rows[9], origin[3];
  rows_of(c, rows, origin);
  FrameDesc fd;
  const Code code = lc::plan_frame(rows, origin, 0.0, 1, fd);
  return code == Code::BadCell ? Code::BadCell : Code::Ok;
}

// The frame table of a batch of frames with their own cell, n, k and mask
// offset; also the batch's points, output elements and mask extent.
Code plan_batch(const lc_frame *fr, size_t n_frames, bool has_mask,
                std::vector<FrameDesc> &frames, size_t &points, size_t &out_n, size_t &mask_n) {
  if (n_frames == 0) return Code::NoPoints;
  frames.assign(n_frames, FrameDesc());
  long long out_base = 0;
  points = mask_n = 0;
  for (size_t f = 0; f < n_frames; ++f) {
    const lc_frame &x = fr[f];
    if (x.n == 0) return Code::NoPoints;
    if (x.k == 0) return Code::ZeroK;
    if (x.mask_offset >= 0 && !has_mask) return Code::NullPointer;
    double rows[9], origin[3];
    rows_of(x.cell, rows, origin);
    const Code c = lc::plan_frame(rows, origin, x.cell_hint, int(x.k), frames[f]);
    if (c != Code::Ok) return c;
    frames[f].n = (long long)x.n;
    frames[f].has_mask = x.mask_offset >= 0 ? 1 : 0;
    frames[f].mask_base = x.mask_offset >= 0 ? x.mask_offset : 0;
    frames[f].out_base = out_base;
    out_base += (long long)(x.n * x.k);
    points += x.n;
    if (x.mask_offset >= 0) mask_n = std::max(mask_n, size_t(x.mask_offset) + x.n);
  }
  out_n = size_t(out_base);
  return Code::Ok;
}

// Frames with their own cell, n, k and mask offset, planned and searched as
// one batch (lc_gpu_knearest_batch, Workspace::knearest_into_batch).
Code run_batch(WorkspaceImpl &w, const double *xyz, const lc_frame *fr, size_t n_frames,
               const int *mask, int *out_nn, double *out_d2, bool wait, std::string &detail) {
  std::vector<FrameDesc> frames;
  size_t points = 0, out_n = 0, mask_n = 0;
  const Code c = plan_batch(fr, n_frames, mask != nullptr, frames, points, out_n, mask_n);
  if (c != Code::Ok) return c;
  return w.run(frames, xyz, mask, out_nn, out_d2, wait, detail);
}

// n_frames copies of one planned frame (shared cell, shared length-n mask).
Code shared_frames(const lc_cell &cell, size_t n, size_t n_frames, size_t k, bool has_mask,
                   double hint, std::vector<FrameDesc> &frames) {
  double rows[9], origin[3];
  rows_of(cell, rows, origin);
  FrameDesc fd;
  const Code c = lc::plan_frame(rows, origin, hint, int(k), fd);
  if (c != Code::Ok) return c;
  fd.n = (long long)n;
  fd.has_mask = has_mask ? 1 : 0;
  fd.mask_base = 0;
  frames.assign(n_frames, fd);
  for (size_t f = 0; f < n_frames; ++f) frames[f].out_base = (long long)(f * n * k);
  return Code::Ok;
}

// The host-pointer search shared by lc_knearest / _d2 / _many.
int host_search(const double *xyz, size_t n, size_t n_frames, const lc_cell *simbox, size_t k,
                const int *mask, double cell_hint, int *out_nn, double *out_d2) {
  // src/capi.rs:195-214
  if (n == 0 || n_frames == 0) return cpu_fail(Code::NoPoints);
  if (k == 0) return cpu_fail(Code::ZeroK);
  if (!xyz || !simbox || !out_nn) return cpu_fail(Code::NullPointer);
  const size_t smax = std::numeric_limits<size_t>::max();
  if (n > smax / n_frames) return cpu_fail(Code::Overflow);
  const size_t n_pts = n * n_frames;
  if (n_pts > smax / k) return cpu_fail(Code::Overflow);
  const size_t need = n_pts * k;
  const size_t imax = size_t(std::numeric_limits<int64_t>::max());
  if (n_pts > imax / 3 || need > imax / sizeof(int)) return cpu_fail(Code::Overflow);
  // src/capi.rs:215-227
  if (check_cell(*simbox) != Code::Ok) return cpu_fail(Code::BadCell);
  // write_one fills every slot first (src/knearest.rs:293-296); an
  // all-masked search then returns before the mesh is sized
  // (src/knearest.rs:370-375).
  bool any_active = mask == nullptr;
  if (mask)
    for (size_t i = 0; i < n && !any_active; ++i) any_active = mask[i] != 0;
  if (!any_active) {
    for (size_t t = 0; t < need; ++t) out_nn[t] = -1;
    if (out_d2)
      for (size_t t = 0; t < need; ++t) out_d2[t] = std::numeric_limits<double>::quiet_NaN();
    cpu_ok();
    return 0;
  }
  std::vector<FrameDesc> frames;
  const Code pc = shared_frames(*simbox, n, n_frames, k, mask != nullptr, cell_hint, frames);
  if (pc != Code::Ok) return cpu_fail(pc);
  if (need > size_t(INT32_MAX) * 4 || n_pts >= 0xFFFFFFF0ull) return cpu_fail(Code::TooLarge);
  if (!device_present()) return cpu_fail(Code::NoDevice);
  std::string detail;
  const Code rc = host_workspace().run_host(frames, xyz, n_pts * 3, mask, mask ? n : 0, out_nn,
                                            out_d2, need, detail);
  if (rc != Code::Ok) return cpu_fail(rc, detail);
  cpu_ok();
  return 0;
}

}  // namespace

namespace lc {
// Sets (or, with nullptr, clears) this thread's lc_gpu_last_error slot.
void set_gpu_error_message(const char *msg) {
  if (msg)
    t_gpu_err = msg;
  else
    t_gpu_err.clear();
}
}  // namespace lc

// ======================================================================
// C++ class (include/linkcell_gpu.hpp)
namespace linkcell {
namespace gpu {

struct Workspace::Impl {
  WorkspaceImpl ws;
};

bool available() { return device_present(); }

Workspace::Workspace() : impl_(nullptr) {
  if (!device_present()) throw Error(lc::gpu_message(Code::NoDevice));
  impl_ = new Impl();
}
Workspace::~Workspace() { delete impl_; }
Workspace::Workspace(Workspace &&o) noexcept : impl_(o.impl_) { o.impl_ = nullptr; }
Workspace &Workspace::operator=(Workspace &&o) noexcept {
  if (this != &o) {
    delete impl_;
    impl_ = o.impl_;
    o.impl_ = nullptr;
  }
  return *this;
}

void *Workspace::queue() { return impl_ ? static_cast<void *>(impl_->ws.stream()) : nullptr; }



void Workspace::set_mode(int mode) {
  if (mode < 0 || mode > 3) throw Error("unknown walk mode");
  impl_->ws.opts.mode = mode;
}
int Workspace::mode() const { return impl_->ws.opts.mode; }

void Workspace::knearest_into(const double *xyz, std::size_t n, const Cell &cell, std::size_t k,
                              int *out, std::size_t out_len, const int *mask, double cell_hint,
                              double *out_d2) {
  knearest_into_many(xyz, n, 1, cell, k, out, out_len, mask, cell_hint, true, nullptr, out_d2);
}

namespace {
[[noreturn]] void throw_code(Code c, const std::string &detail) {
  std::string m = lc::gpu_message(c);
  if (!detail.empty() && (c == Code::Cuda || c == Code::DeviceStatus)) m += ": " + detail;
  throw Error(m);
}

}  // namespace

void Workspace::wait() {
  if (!impl_) return;
  std::string detail;
  const Code c = impl_->ws.wait(detail);
  if (c != Code::Ok) throw_code(c, detail);
}

void Workspace::knearest_into_batch(const double *xyz, const Frame *frames, std::size_t nFrames,
                                    int *out, std::size_t out_len, const int *mask, double *out_d2,
                                    bool wait) {
  if (!impl_) throw Error(lc::gpu_message(Code::NoDevice));
  if (xyz == nullptr || frames == nullptr || out == nullptr) throw Error("null pointer");
  std::vector<lc_frame> fr(nFrames);
  std::size_t need = 0;
  for (std::size_t f = 0; f < nFrames; ++f) {
    fr[f].n = frames[f].n;
    fr[f].k = frames[f].k;
    fr[f].cell = frames[f].cell.raw();
    fr[f].cell_hint = frames[f].cell_hint;
    fr[f].mask_offset = frames[f].mask_offset;
    need += frames[f].n * frames[f].k;
  }
  if (out_len != need) throw Error("out buffer length must be the sum of n * k over the frames");
  std::string detail;
  const Code c = run_batch(impl_->ws, xyz, fr.data(), nFrames, mask, out, out_d2, wait, detail);
  if (c != Code::Ok) throw_code(c, detail);
}

void Workspace::knearest_into_many(const double *xyz, std::size_t n, std::size_t nFrames,
                                   const Cell &cell, std::size_t k, int *out, std::size_t out_len,
                                   const int *mask, double cell_hint, bool wait,
                                   const double *frameBox, double *out_d2) {
  // src/gpu/knearest.cpp:711-728
  if (!impl_) throw Error(lc::gpu_message(Code::NoDevice));
  if (n == 0 || nFrames == 0) throw Error("no points");
  if (k == 0) throw Error("k must be at least 1");
  if (out_len != n * k * nFrames) throw Error("out buffer length must be nFrames * n * k");
  if (xyz == nullptr || out == nullptr) throw Error("null pointer");
  const lc_cell raw = cell.raw();
  if (check_cell(raw) != Code::Ok) throw Error("bad cell");
  std::vector<FrameDesc> frames;
  Code pc = shared_frames(raw, n, nFrames, k, mask != nullptr, cell_hint, frames);
  if (pc == Code::TooFine && mask) {
    // all-masked: -1 / NaN rows (src/knearest.rs:370-375), checked on the device
    std::string detail;
    const Code c = impl_->ws.too_fine_masked(mask, (long long)n, out, out_d2, (long long)out_len,
                                             wait, detail);
    if (c != Code::Ok) throw_code(c, detail);
    return;
  }
  if (pc != Code::Ok) throw_code(pc, "");
  if (frameBox) {
    // per-frame orthorhombic lengths (src/gpu/knearest.cpp:733-797)
    if (!frames[0].ortho) throw Error("frame boxes on a sheared cell need a shared H");
    for (std::size_t f = 0; f < nFrames; ++f) {
      const double L[3] = {frameBox[3 * f + 0], frameBox[3 * f + 1], frameBox[3 * f + 2]};
      if (!(L[0] > 0.0 && L[1] > 0.0 && L[2] > 0.0)) throw Error("bad frame box");
      const lc_cell fc = {L[0], 0, 0, 0, L[1], 0, 0, 0, L[2], raw.ox, raw.oy, raw.oz};
      double rows[9], origin[3];
      rows_of(fc, rows, origin);
      FrameDesc fd;
      const Code c = lc::plan_frame(rows, origin, cell_hint, int(k), fd);
      if (c != Code::Ok) throw_code(c, "");
      if (fd.nx != frames[0].nx || fd.ny != frames[0].ny || fd.nz != frames[0].nz)
        throw Error("frame boxes need the same cell grid");
      fd.n = frames[f].n;
      fd.has_mask = frames[f].has_mask;
      fd.mask_base = 0;
      fd.out_base = frames[f].out_base;
      frames[f] = fd;
    }
  }
  std::string detail;
  const Code rc = impl_->ws.run(frames, xyz, mask, out, out_d2, wait, detail);
  if (rc != Code::Ok) throw_code(rc, detail);
}

void Workspace::knearest_into_many_dcell(const double *xyz, std::size_t n, std::size_t nFrames,
                                         const double *cell, int cell_n, std::size_t k, int *out,
                                         std::size_t out_len, const int *mask, double cell_hint,
                                         bool wait, double *out_d2) {
  // src/gpu/knearest.cpp:818-878
  if (!impl_) throw Error(lc::gpu_message(Code::NoDevice));
  if (n == 0 || nFrames == 0) throw Error("no points");
  if (k == 0) throw Error("k must be at least 1");
  if (out_len != n * k * nFrames) throw Error("out buffer length must be nFrames * n * k");
  if (xyz == nullptr || out == nullptr || cell == nullptr) throw Error("null pointer");
  if (cell_n != 3 && cell_n != 9 && cell_n != 12)
    throw Error("device cell must have 3, 9, or 12 doubles");
  if (nFrames <= std::size_t(WorkspaceImpl::kDeviceCellFrames)) {
    // planned on the device: no read of the cell, graph-capturable
    std::string detail;
    const Code c = impl_->ws.run_device_cell(cell, cell_n, (long long)n, int(nFrames), int(k),
                                             cell_hint, xyz, mask, out, out_d2, wait, detail);
    if (c != Code::Ok) throw_code(c, detail);
    return;
  }
  double h[12] = {0};
  const cudaStream_t s = impl_->ws.stream();
  if (cudaMemcpyAsync(h, cell, size_t(cell_n) * sizeof(double), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    throw Error("DtoH cell");
  lc_cell raw;
  if (cell_n == 3) {
    raw = lc_cell{h[0], 0, 0, 0, h[1], 0, 0, 0, h[2], 0, 0, 0};
  } else {
    raw = lc_cell{h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], h[8],
                  cell_n == 12 ? h[9] : 0.0, cell_n == 12 ? h[10] : 0.0,
                  cell_n == 12 ? h[11] : 0.0};
  }
  knearest_into_many(xyz, n, nFrames, Cell(raw), k, out, out_len, mask, cell_hint, wait, nullptr,
                     out_d2);
}

}  // namespace gpu
}  // namespace linkcell

// ======================================================================
// C ABI
struct lc_gpu_workspace {
  WorkspaceImpl ws;
};

extern "C" {

int lc_knearest(const double *xyz, size_t n, const lc_cell *simbox, size_t k, const int *mask,
                double cell_hint, int *out_nn) {
  return host_search(xyz, n, 1, simbox, k, mask, cell_hint, out_nn, nullptr);
}

int lc_knearest_d2(const double *xyz, size_t n, const lc_cell *simbox, size_t k, const int *mask,
                   double cell_hint, int *out_nn, double *out_d2) {
  return host_search(xyz, n, 1, simbox, k, mask, cell_hint, out_nn, out_d2);
}

int lc_knearest_many(const double *xyz, size_t n, size_t n_frames, const lc_cell *simbox, size_t k,
                     const int *mask, double cell_hint, int *out_nn, double *out_d2) {
  return host_search(xyz, n, n_frames, simbox, k, mask, cell_hint, out_nn, out_d2);
}

int lc_knearest_batch(const double *xyz, const lc_frame *frames, size_t n_frames, const int *mask,
                      int *out_nn, double *out_d2) {
  if (!xyz || !frames || !out_nn) return cpu_fail(Code::NullPointer);
  std::vector<FrameDesc> fd;
  size_t points = 0, out_n = 0, mask_n = 0;
  const Code c = plan_batch(frames, n_frames, mask != nullptr, fd, points, out_n, mask_n);
  if (c != Code::Ok) return cpu_fail(c);
  if (points >= 0xFFFFFFF0ull || out_n > size_t(INT32_MAX) * 4) return cpu_fail(Code::TooLarge);
  if (!device_present()) return cpu_fail(Code::NoDevice);
  std::string detail;
  const Code rc = host_workspace().run_host(fd, xyz, points * 3, mask, mask_n, out_nn, out_d2,
                                            out_n, detail);
  if (rc != Code::Ok) return cpu_fail(rc, detail);
  cpu_ok();
  return 0;
}

const char *lc_last_error(void) { return t_cpu_has_err ? t_cpu_err.c_str() : nullptr; }

const char *lc_version(void) { return "0.3.3"; }

int lc_gpu_available(void) { return device_present() ? 1 : 0; }

const char *lc_gpu_last_error(void) { return t_gpu_err.empty() ? nullptr : t_gpu_err.c_str(); }

lc_gpu_workspace *lc_gpu_workspace_new(void) {
  if (!device_present()) {
    gpu_fail(Code::NoDevice);
    return nullptr;
  }
  try {
    lc_gpu_workspace *w = new lc_gpu_workspace();
    gpu_ok();
    return w;
  } catch (const std::exception &e) {
    gpu_fail_msg(e.what());
    return nullptr;
  }
}

void lc_gpu_workspace_free(lc_gpu_workspace *ws) { delete ws; }

int lc_gpu_knearest(lc_gpu_workspace *ws, const double *xyz, size_t n, const lc_cell *simbox,
                    size_t k, const int *mask, double cell_hint, int *out_nn, double *out_d2) {
  return lc_gpu_knearest_many(ws, xyz, n, 1, simbox, k, mask, cell_hint, out_nn, out_d2, 1);
}

int lc_gpu_knearest_many(lc_gpu_workspace *ws, const double *xyz, size_t n, size_t n_frames,
                         const lc_cell *simbox, size_t k, const int *mask, double cell_hint,
                         int *out_nn, double *out_d2, int wait) {
  // src/gpu/capi.cpp:77-81, then src/gpu/knearest.cpp:711-762
  if (!ws || !xyz || !simbox || !out_nn) return gpu_fail(Code::NullPointer);
  if (n == 0 || n_frames == 0) return gpu_fail(Code::NoPoints);
  if (k == 0) return gpu_fail(Code::ZeroK);
  const size_t smax = std::numeric_limits<size_t>::max();
  if (n > smax / n_frames || n * n_frames > smax / k) return gpu_fail(Code::Overflow);
  if (check_cell(*simbox) != Code::Ok) return gpu_fail(Code::BadCell);
  std::vector<FrameDesc> frames;
  const Code pc = shared_frames(*simbox, n, n_frames, k, mask != nullptr, cell_hint, frames);
  const size_t need = n * n_frames * k;
  if (pc == Code::TooFine && mask) {
    // all-masked: -1 / NaN rows (src/knearest.rs:370-375), checked on the device
    std::string detail;
    const Code c = ws->ws.too_fine_masked(mask, (long long)n, out_nn, out_d2, (long long)need,
                                          wait != 0, detail);
    if (c != Code::Ok) return gpu_fail(c, detail);
    gpu_ok();
    return 0;
  }
  if (pc != Code::Ok) return gpu_fail(pc);
  std::string detail;
  const Code rc = ws->ws.run(frames, xyz, mask, out_nn, out_d2, wait != 0, detail);
  if (rc != Code::Ok) return gpu_fail(rc, detail);
  gpu_ok();
  return 0;
}

int lc_gpu_knearest_shard(lc_gpu_workspace *ws, const double *xyz, size_t n, size_t n_frames,
                          const lc_cell *simbox, size_t k, const int *mask, double cell_hint,
                          int rank, int world, int *out_nn, double *out_d2, int *out_owned,
                          int wait) {
  if (!ws || !xyz || !simbox || !out_nn || !out_owned) return gpu_fail(Code::NullPointer);
  if (n == 0 || n_frames == 0) return gpu_fail(Code::NoPoints);
  if (k == 0) return gpu_fail(Code::ZeroK);
  if (world < 1 || rank < 0 || rank >= world) return gpu_fail_msg("rank must lie in [0, world)");
  const size_t smax = std::numeric_limits<size_t>::max();
  if (n > smax / n_frames || n * n_frames > smax / k) return gpu_fail(Code::Overflow);
  if (check_cell(*simbox) != Code::Ok) return gpu_fail(Code::BadCell);
  std::vector<FrameDesc> frames;
  const Code pc = shared_frames(*simbox, n, n_frames, k, mask != nullptr, cell_hint, frames);
  const size_t need = n * n_frames * k;
  std::string detail;
  if (pc == Code::TooFine && mask) {
    // all-masked: -1 / NaN rows on every rank, owned by rank 0
    const Code c = ws->ws.too_fine_masked(mask, (long long)n, out_nn, out_d2, (long long)need,
                                          false, detail);
    if (c != Code::Ok) return gpu_fail(c, detail);
    const cudaError_t e = cudaMemsetAsync(out_owned, rank == 0 ? 1 : 0,
                                          n * n_frames * sizeof(int), ws->ws.stream());
    if (e != cudaSuccess) return gpu_fail(Code::Cuda, cudaGetErrorString(e));
    if (wait) {
      const Code w = ws->ws.wait(detail);
      if (w != Code::Ok) return gpu_fail(w, detail);
    }
    gpu_ok();
    return 0;
  }
  if (pc != Code::Ok) return gpu_fail(pc);
  const Code rc = ws->ws.run_shard(frames, xyz, mask, out_nn, out_d2, out_owned, rank, world,
                                   wait != 0, detail);
  if (rc != Code::Ok) return gpu_fail(rc, detail);
  gpu_ok();
  return 0;
}

int lc_gpu_knearest_many_dcell(lc_gpu_workspace *ws, const double *xyz, size_t n, size_t n_frames,
                               const double *cell, int cell_n, size_t k, const int *mask,
                               double cell_hint, int *out_nn, double *out_d2, int wait) {
  // src/gpu/capi.cpp:116-120, src/gpu/knearest.cpp:825-842
  if (!ws || !xyz || !cell || !out_nn) return gpu_fail(Code::NullPointer);
  if (n == 0 || n_frames == 0) return gpu_fail(Code::NoPoints);
  if (k == 0) return gpu_fail(Code::ZeroK);
  if (cell_n != 3 && cell_n != 9 && cell_n != 12) return gpu_fail(Code::BadCellN);
  const size_t smax = std::numeric_limits<size_t>::max();
  if (n > smax / n_frames || n * n_frames > smax / k) return gpu_fail(Code::Overflow);
  if (n_frames <= size_t(WorkspaceImpl::kDeviceCellFrames)) {
    // planned on the device: no read of the cell, graph-capturable
    std::string detail;
    const Code c = ws->ws.run_device_cell(cell, cell_n, (long long)n, int(n_frames), int(k),
                                          cell_hint, xyz, mask, out_nn, out_d2, wait != 0, detail);
    if (c != Code::Ok) return gpu_fail(c, detail);
    gpu_ok();
    return 0;
  }
  // more frames than the device-planned cell arrays cover: read the cell
  double h[12] = {0};
  const cudaStream_t s = ws->ws.stream();
  cudaError_t e = cudaMemcpyAsync(h, cell, size_t(cell_n) * sizeof(double),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return gpu_fail(Code::Cuda, cudaGetErrorString(e));
  lc_cell raw;
  if (cell_n == 3)
    raw = lc_cell{h[0], 0, 0, 0, h[1], 0, 0, 0, h[2], 0, 0, 0};
  else
    raw = lc_cell{h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], h[8],
                  cell_n == 12 ? h[9] : 0.0, cell_n == 12 ? h[10] : 0.0,
                  cell_n == 12 ? h[11] : 0.0};
  return lc_gpu_knearest_many(ws, xyz, n, n_frames, &raw, k, mask, cell_hint, out_nn, out_d2,
                              wait);
}

void *lc_gpu_queue(lc_gpu_workspace *ws) { return ws ? static_cast<void *>(ws->ws.stream()) : nullptr; }

void lc_gpu_wait(lc_gpu_workspace *ws) {
  if (!ws) return;
  std::string detail;
  const Code c = ws->ws.wait(detail);
  if (c != Code::Ok) gpu_fail(c, detail);
}

int lc_gpu_alloc(void **ptr, size_t bytes) {
  if (!ptr) return gpu_fail(Code::NullPointer);
  if (!device_present()) return gpu_fail(Code::NoDevice);
  const cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) return gpu_fail_msg(cudaGetErrorString(e));
  gpu_ok();
  return 0;
}

void lc_gpu_free(void *ptr) {
  if (ptr) cudaFree(ptr);
}

int lc_gpu_memcpy(void *dst, const void *src, size_t bytes, int kind) {
  if (bytes == 0) {
    gpu_ok();
    return 0;
  }
  if (!dst || !src) return gpu_fail(Code::NullPointer);
  if (!device_present()) return gpu_fail(Code::NoDevice);
  const cudaError_t e = cudaMemcpy(dst, src, bytes, static_cast<cudaMemcpyKind>(kind));
  if (e != cudaSuccess) return gpu_fail_msg(cudaGetErrorString(e));
  gpu_ok();
  return 0;
}

int lc_gpu_fill_i32(void *ptr, int value, size_t n) {
  if (!ptr && n != 0) return gpu_fail(Code::NullPointer);
  if (!device_present()) return gpu_fail(Code::NoDevice);
  if (value != 0 && value != -1) return gpu_fail_msg("lc_gpu_fill_i32 only supports 0 and -1");
  const cudaError_t e = cudaMemset(ptr, value == 0 ? 0 : 0xFF, n * sizeof(int));
  if (e != cudaSuccess) return gpu_fail_msg(cudaGetErrorString(e));
  gpu_ok();
  return 0;
}

// The extension setters below leave the error slot alone on success, so a
// caller can still read the message of the search that failed before them.
int lc_gpu_set_mode(lc_gpu_workspace *ws, int mode) {
  if (!ws) return gpu_fail(Code::NullPointer);
  if (mode < 0 || mode > 3) return gpu_fail_msg("unknown walk mode");
  ws->ws.opts.mode = mode;
  return 0;
}

int lc_gpu_get_mode(lc_gpu_workspace *ws) { return ws ? ws->ws.opts.mode : -1; }

int lc_gpu_set_tpp(lc_gpu_workspace *ws, int tpp) {
  if (!ws) return gpu_fail(Code::NullPointer);
  if (tpp != 0 && tpp != 1 && tpp != 32)
    return gpu_fail_msg("threads per source must be 1 or 32 (0: autotune)");
  if (tpp == 0) {
    ws->ws.opts.tpp_forced = false;
  } else {
    ws->ws.opts.tpp = tpp;
    ws->ws.opts.tpp_forced = true;
  }
  return 0;
}

int lc_gpu_get_tpp(lc_gpu_workspace *ws) { return ws ? ws->ws.last_tpp : -1; }

int lc_gpu_set_walk_shape(lc_gpu_workspace *ws, int warps, int grab) {
  if (!ws) return gpu_fail(Code::NullPointer);
  if (!(warps == 0 || warps == 2 || warps == 4 || warps == 8))
    return gpu_fail_msg("warps per block must be 2, 4 or 8 (0: autotune)");
  if (!(grab == 0 || grab == 8 || grab == 16 || grab == 32))
    return gpu_fail_msg("sources per grab must be 8, 16 or 32 (0: autotune)");
  ws->ws.opts.sel_warps = warps;
  ws->ws.opts.sel_grab = grab;
  return 0;
}

int lc_gpu_walk_shape(lc_gpu_workspace *ws, int *shape3, int *trials, int max_trials) {
  if (!ws) return gpu_fail(Code::NullPointer);
  const lc::WalkShape &l = ws->ws.last_shape;
  if (shape3) {
    shape3[0] = l.tpp;
    shape3[1] = l.warps;
    shape3[2] = l.grab;
  }
  const auto &t = ws->ws.trial_shapes_;
  if (trials)
    for (int i = 0; i < max_trials && size_t(i) < t.size(); ++i) {
      trials[3 * i] = t[size_t(i)].tpp;
      trials[3 * i + 1] = t[size_t(i)].warps;
      trials[3 * i + 2] = t[size_t(i)].grab;
    }
  return int(t.size());
}

int lc_gpu_set_graph(lc_gpu_workspace *ws, int on) {
  if (!ws) return gpu_fail(Code::NullPointer);
  ws->ws.opts.graph = on != 0;
  return 0;
}

int lc_gpu_graph_captures(lc_gpu_workspace *ws) { return ws ? ws->ws.graph_captures : -1; }

int lc_gpu_set_stats(lc_gpu_workspace *ws, int on) {
  if (!ws) return gpu_fail(Code::NullPointer);
  ws->ws.opts.stats = on != 0;
  return 0;
}

int lc_gpu_set_scan_limit(lc_gpu_workspace *ws, int spins, long long silent_tile) {
  if (!ws) return gpu_fail(Code::NullPointer);
  ws->ws.opts.scan_spin_limit = spins > 0 ? spins : 0;
  ws->ws.opts.scan_silent_tile = silent_tile >= 0 ? silent_tile : -1;
  return 0;
}

int lc_gpu_set_model(lc_gpu_workspace *ws, const float *params, size_t n_params, float tau) {
  if (!ws || !params) return gpu_fail(Code::NullPointer);
  if (!(tau > 0.f && tau <= 1.f)) return gpu_fail_msg("tau must lie in (0, 1]");
  std::string detail;
  const Code c = ws->ws.set_model(params, n_params, tau, detail);
  if (c != Code::Ok) return gpu_fail_msg(detail.empty() ? lc::gpu_message(c) : detail);
  return 0;
}

int lc_gpu_log_shells(lc_gpu_workspace *ws, int on) {
  if (!ws) return gpu_fail(Code::NullPointer);
  ws->ws.opts.log_shells = on ? 1 : 0;
  return 0;
}

long long lc_gpu_training_rows(lc_gpu_workspace *ws, float *X, int *y, long long cap,
                               long long stride, long long first) {
  if (!ws || !X || !y) return -gpu_fail(Code::NullPointer);
  long long rows = 0;
  std::string detail;
  const Code c = ws->ws.training_rows(X, y, cap, stride, first, rows, detail);
  if (c != Code::Ok) return -gpu_fail_msg(detail.empty() ? lc::gpu_message(c) : detail);
  return rows;
}

long long lc_gpu_proposals(lc_gpu_workspace *ws, signed char *out, long long cap, long long stride,
                           long long first) {
  if (!ws || !out) return -gpu_fail(Code::NullPointer);
  long long rows = 0;
  std::string detail;
  const Code c =
      ws->ws.proposals(reinterpret_cast<int8_t *>(out), cap, stride, first, rows, detail);
  if (c != Code::Ok) return -gpu_fail_msg(detail.empty() ? lc::gpu_message(c) : detail);
  return rows;
}

int lc_gpu_mlp_params(void) { return lc::kMlpParams; }

size_t lc_gpu_mlp_scratch_floats(int batch) { return lc::MlpScratch::floats(batch); }

int lc_gpu_mlp_forward(const float *params, const float *X, int batch, float *probs,
                       float *scratch, void *stream) {
  if (!params || !X || !probs || !scratch) return gpu_fail(Code::NullPointer);
  lc::MlpScratch t = lc::MlpScratch::carve(scratch, batch);
  const cudaError_t e =
      lc::mlp_forward(params, X, batch, t, probs, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return gpu_fail(Code::Cuda, cudaGetErrorString(e));
  return 0;
}

int lc_gpu_mlp_grad(const float *params, const float *X, const int *y, int batch, float *grad,
                    float *loss, float *scratch, void *stream) {
  if (!params || !X || !y || !grad || !scratch) return gpu_fail(Code::NullPointer);
  lc::MlpScratch t = lc::MlpScratch::carve(scratch, batch);
  const cudaError_t e =
      lc::mlp_grad(params, X, y, batch, t, grad, loss, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return gpu_fail(Code::Cuda, cudaGetErrorString(e));
  return 0;
}

int lc_gpu_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr,
                    void *stream) {
  if (!params || !grad || !m || !v) return gpu_fail(Code::NullPointer);
  if (step < 1) return gpu_fail_msg("adam step starts at 1");
  const cudaError_t e =
      lc::mlp_adam(params, grad, m, v, step, lr, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return gpu_fail(Code::Cuda, cudaGetErrorString(e));
  return 0;
}

int lc_gpu_set_proposal(lc_gpu_workspace *ws, int shell) {
  if (!ws) return gpu_fail(Code::NullPointer);
  if (shell < 0 || shell > 127) return gpu_fail_msg("proposal shell must be 0..127");
  ws->ws.opts.fixed_proposal = shell;
  return 0;
}

int lc_gpu_set_stream(lc_gpu_workspace *ws, void *stream) {
  if (!ws) return gpu_fail(Code::NullPointer);
  ws->ws.set_stream(static_cast<cudaStream_t>(stream));
  return 0;
}

int lc_gpu_stats(lc_gpu_workspace *ws, long long *counters, int n_counters, double *device_ms) {
  if (!ws) return gpu_fail(Code::NullPointer);
  lc::Stats st;
  std::string detail;
  const Code c = ws->ws.fetch_stats(st, detail);
  if (c != Code::Ok) return -gpu_fail(c, detail);
  const int m = n_counters < lc::kNumCounters ? n_counters : lc::kNumCounters;
  for (int i = 0; i < m && counters; ++i) counters[i] = st.counters[i];
  if (device_ms) *device_ms = st.ms_total;
  gpu_ok();
  return m;
}

int lc_gpu_phase_times(lc_gpu_workspace *ws, double *prep_ms, double *walk_ms, double *replay_ms) {
  if (!ws) return gpu_fail(Code::NullPointer);
  lc::Stats st;
  std::string detail;
  const Code c = ws->ws.fetch_stats(st, detail);
  if (c != Code::Ok) return gpu_fail(c, detail);
  if (prep_ms) *prep_ms = st.ms_prep;
  if (walk_ms) *walk_ms = st.ms_walk;
  if (replay_ms) *replay_ms = st.ms_replay;
  gpu_ok();
  return 0;
}

int lc_gpu_neighbors_within(lc_gpu_workspace *ws, const int *out_nn, const double *out_d2,
                            size_t rows, size_t k, double cutoff, int *row_ptr, int *col,
                            double *dist2, size_t cap, size_t *nnz) {
  if (!ws || !out_nn || !out_d2 || !row_ptr || !nnz || (cap > 0 && !col))
    return gpu_fail(Code::NullPointer);
  if (k == 0) return gpu_fail(Code::ZeroK);
  if (!(cutoff >= 0.0)) return gpu_fail_msg("cutoff must be a non-negative number");
  std::string detail;
  const Code c = ws->ws.neighbors_within(out_nn, out_d2, rows, k, cutoff, row_ptr, col, dist2, cap,
                                         *nnz, detail);
  if (c != Code::Ok) return gpu_fail(c, detail);
  if (*nnz > cap) return gpu_fail_msg("neighbour list longer than its buffer");
  gpu_ok();
  return 0;
}

int lc_gpu_phase_times4(lc_gpu_workspace *ws, double *prep_ms, double *propose_ms, double *walk_ms,
                        double *replay_ms) {
  if (!ws) return gpu_fail(Code::NullPointer);
  lc::Stats st;
  std::string detail;
  const Code c = ws->ws.fetch_stats(st, detail);
  if (c != Code::Ok) return gpu_fail(c, detail);
  if (prep_ms) *prep_ms = st.ms_prep;
  if (propose_ms) *propose_ms = st.ms_propose;
  if (walk_ms) *walk_ms = st.ms_walk - st.ms_propose;
  if (replay_ms) *replay_ms = st.ms_replay;
  gpu_ok();
  return 0;
}

int lc_gpu_knearest_batch(lc_gpu_workspace *ws, const double *xyz, const lc_frame *fr,
                          size_t n_frames, const int *mask, int *out_nn, double *out_d2,
                          int wait) {
  if (!ws || !xyz || !fr || !out_nn) return gpu_fail(Code::NullPointer);
  std::string detail;
  const Code rc = run_batch(ws->ws, xyz, fr, n_frames, mask, out_nn, out_d2, wait != 0, detail);
  if (rc != Code::Ok) return gpu_fail(rc, detail);
  gpu_ok();
  return 0;
}

}  // extern "C"
