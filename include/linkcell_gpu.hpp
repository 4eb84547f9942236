// Device-resident periodic k-nearest search: the C++ class of the
// reference (HaoZeke/linkcell v0.3.3, include/linkcell_gpu.hpp:29-78) over
// the B200 implementation. xyz, mask and outputs are CUDA device pointers.
// Results equal the host walk's (linkcell::knearest_into) exactly, for any
// k >= 1 (the reference class documents k <= 16).
#ifndef LINKCELL_GPU_HPP
#define LINKCELL_GPU_HPP

#include <cstddef>

#include "linkcell.hpp"

namespace linkcell {
namespace gpu {

/// True when a CUDA device is usable (reference src/gpu/knearest.cpp:542-544).
bool available();

class Workspace {
 public:
  Workspace();
  ~Workspace();
  Workspace(Workspace &&) noexcept;
  Workspace &operator=(Workspace &&) noexcept;
  Workspace(const Workspace &) = delete;
  Workspace &operator=(const Workspace &) = delete;

  /// Device xyz is n * 3 doubles, device out n * k ints, out_d2 n * k
  /// doubles or nullptr. Waits for completion.
  void knearest_into(const double *xyz, std::size_t n, const Cell &cell, std::size_t k, int *out,
                     std::size_t out_len, const int *mask = nullptr, double cell_hint = 0.0,
                     double *out_d2 = nullptr);

  /// nFrames frames sharing one cell, frame-major. frameBox (host, 3 per
  /// frame) gives each frame its own orthorhombic lengths on an
  /// orthorhombic cell; all frames must then share the cell grid
  /// (reference src/gpu/knearest.cpp:733-797).
  void knearest_into_many(const double *xyz, std::size_t n, std::size_t nFrames, const Cell &cell,
                          std::size_t k, int *out, std::size_t out_len, const int *mask = nullptr,
                          double cell_hint = 0.0, bool wait = true,
                          const double *frameBox = nullptr, double *out_d2 = nullptr);

  /// Device-packed cell: 3 ortho lengths, 9 lattice rows, or 12 rows plus
  /// origin. Up to 16 frames the cell is planned on the device (no blocking
  /// read of the mesh; errors surface at wait).
  void knearest_into_many_dcell(const double *xyz, std::size_t n, std::size_t nFrames,
                                const double *cell, int cell_n, std::size_t k, int *out,
                                std::size_t out_len, const int *mask = nullptr,
                                double cell_hint = 0.0, bool wait = true,
                                double *out_d2 = nullptr);

  /// Extension (no counterpart in the reference, whose batch shares one
  /// cell): frames with their own cell, point count, k and mask in one call.
  /// Frame f's points follow frame f - 1's in xyz; its rows start at the sum
  /// of n * k over the frames before it; mask_offset indexes the device mask
  /// (-1: no mask). out_len must be that sum (lc_gpu_knearest_batch).
  struct Frame {
    std::size_t n = 0, k = 0;
    Cell cell;
    double cell_hint = 0.0;
    long long mask_offset = -1;
  };
  void knearest_into_batch(const double *xyz, const Frame *frames, std::size_t nFrames, int *out,
                           std::size_t out_len, const int *mask = nullptr,
                           double *out_d2 = nullptr, bool wait = true);

  /// The workspace's CUDA stream; all work is enqueued there.
  void *queue();
  void wait();

  /// Extension: walk mode (LC_GPU_MODE_* in linkcell_gpu.h).
  void set_mode(int mode);
  int mode() const;

  struct Impl;

 private:
  Impl *impl_;
};

}  // namespace gpu
}  // namespace linkcell

#endif
