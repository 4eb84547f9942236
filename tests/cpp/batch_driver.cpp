// C++ driver for linkcell::gpu::Workspace::knearest_into_batch.
//
// Reads a batch from a binary file, searches it through the C++ class on the
// GPU and writes the rows and squared distances to a second file; the
// calling test compares them with the oracle. Input layout (little endian):
//   int64 n_frames, int64 mask_len
//   per frame: int64 n, int64 k, int64 mask_offset, double cell[12] (a, b, c
//   rows, origin), double cell_hint
//   double xyz[3 * sum n], int32 mask[mask_len]
// Output: int32 rows[sum n k], double dist2[sum n k], then for frame 0 alone
// three more (rows, dist2) pairs of n0 k0 entries each: through
// Workspace::knearest_into, Workspace::knearest_into_many_dcell (the cell
// as 12 device doubles) and the host API linkcell::knearest.
// It also checks that a wrong out_len throws linkcell::Error before any work.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "linkcell_gpu.hpp"

namespace {

bool check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
  return false;
}

template <class T>
bool read_n(std::FILE *f, T *v, std::size_t n) {
  return std::fread(v, sizeof(T), n, f) == n;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: batch_driver IN OUT\n");
    return 2;
  }
  std::FILE *in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  std::int64_t nf = 0, mask_len = 0;
  if (!read_n(in, &nf, 1) || !read_n(in, &mask_len, 1) || nf <= 0) return 2;
  std::vector<linkcell::gpu::Workspace::Frame> frames(static_cast<std::size_t>(nf));
  std::size_t points = 0, rows = 0;
  for (auto &fr : frames) {
    std::int64_t nk[3];
    double c[13];
    if (!read_n(in, nk, 3) || !read_n(in, c, 13)) return 2;
    fr.n = static_cast<std::size_t>(nk[0]);
    fr.k = static_cast<std::size_t>(nk[1]);
    fr.mask_offset = nk[2];
    fr.cell = linkcell::Cell::from_vectors({c[0], c[1], c[2]}, {c[3], c[4], c[5]},
                                           {c[6], c[7], c[8]}, {c[9], c[10], c[11]});
    fr.cell_hint = c[12];
    points += fr.n;
    rows += fr.n * fr.k;
  }
  std::vector<double> xyz(3 * points);
  std::vector<int> mask(static_cast<std::size_t>(mask_len));
  if (!read_n(in, xyz.data(), xyz.size()) || !read_n(in, mask.data(), mask.size())) return 2;
  std::fclose(in);

  double *d_xyz = nullptr, *d_d2 = nullptr;
  int *d_out = nullptr, *d_mask = nullptr;
  if (!check(cudaMalloc(&d_xyz, xyz.size() * sizeof(double)), "malloc xyz") ||
      !check(cudaMalloc(&d_out, rows * sizeof(int)), "malloc out") ||
      !check(cudaMalloc(&d_d2, rows * sizeof(double)), "malloc d2") ||
      !check(cudaMalloc(&d_mask, (mask.size() + 1) * sizeof(int)), "malloc mask") ||
      !check(cudaMemcpy(d_xyz, xyz.data(), xyz.size() * sizeof(double), cudaMemcpyHostToDevice),
             "copy xyz") ||
      !check(cudaMemcpy(d_mask, mask.data(), mask.size() * sizeof(int), cudaMemcpyHostToDevice),
             "copy mask"))
    return 3;

  int rc = 0;
  try {
    linkcell::gpu::Workspace ws;
    bool threw = false;
    try {
      ws.knearest_into_batch(d_xyz, frames.data(), frames.size(), d_out, rows + 1,
                             mask_len ? d_mask : nullptr, d_d2);
    } catch (const linkcell::Error &) {
      threw = true;
    }
    if (!threw) {
      std::fprintf(stderr, "wrong out_len was accepted\n");
      rc = 4;
    } else {
      ws.knearest_into_batch(d_xyz, frames.data(), frames.size(), d_out, rows,
                             mask_len ? d_mask : nullptr, d_d2);
      std::vector<int> out(rows);
      std::vector<double> d2(rows);
      if (!check(cudaMemcpy(out.data(), d_out, rows * sizeof(int), cudaMemcpyDeviceToHost),
                 "copy out") ||
          !check(cudaMemcpy(d2.data(), d_d2, rows * sizeof(double), cudaMemcpyDeviceToHost),
                 "copy d2")) {
        rc = 3;
      } else {
        std::FILE *o = std::fopen(argv[2], "wb");
        if (!o || std::fwrite(out.data(), sizeof(int), rows, o) != rows ||
            std::fwrite(d2.data(), sizeof(double), rows, o) != rows)
          rc = 2;
        // frame 0 through the single-frame entry points
        const auto &f0 = frames[0];
        const std::size_t r0 = f0.n * f0.k;
        const int *dm0 = f0.mask_offset >= 0 ? d_mask + f0.mask_offset : nullptr;
        const int *hm0 = f0.mask_offset >= 0 ? mask.data() + f0.mask_offset : nullptr;
        const lc_cell raw = f0.cell.raw();
        const double cell12[12] = {raw.ax, raw.ay, raw.az, raw.bx, raw.by, raw.bz,
                                   raw.cx, raw.cy, raw.cz, raw.ox, raw.oy, raw.oz};
        double *d_cell = nullptr;
        std::vector<int> o0(r0);
        std::vector<double> e0(r0);
        auto emit = [&]() {
          if (!o || std::fwrite(o0.data(), sizeof(int), r0, o) != r0 ||
              std::fwrite(e0.data(), sizeof(double), r0, o) != r0)
            rc = 2;
        };
        auto fetch = [&]() {
          return check(cudaMemcpy(o0.data(), d_out, r0 * sizeof(int), cudaMemcpyDeviceToHost),
                       "copy out") &&
                 check(cudaMemcpy(e0.data(), d_d2, r0 * sizeof(double), cudaMemcpyDeviceToHost),
                       "copy d2");
        };
        ws.knearest_into(d_xyz, f0.n, f0.cell, f0.k, d_out, r0, dm0, f0.cell_hint, d_d2);
        if (fetch()) emit(); else rc = 3;
        if (check(cudaMalloc(&d_cell, sizeof(cell12)), "malloc cell") &&
            check(cudaMemcpy(d_cell, cell12, sizeof(cell12), cudaMemcpyHostToDevice), "copy cell")) {
          ws.knearest_into_many_dcell(d_xyz, f0.n, 1, d_cell, 12, f0.k, d_out, r0, dm0,
                                      f0.cell_hint, true, d_d2);
          if (fetch()) emit(); else rc = 3;
        } else {
          rc = 3;
        }
        cudaFree(d_cell);
        const linkcell::Neighbours nb = linkcell::knearest(xyz.data(), f0.n, f0.cell, f0.k, hm0,
                                                           f0.cell_hint);
        std::copy(nb.begin(), nb.end(), o0.begin());
        std::copy(nb.distances(), nb.distances() + r0, e0.begin());
        emit();
        if (o) std::fclose(o);
      }
    }
  } catch (const linkcell::Error &e) {
    std::fprintf(stderr, "linkcell error: %s\n", e.what());
    rc = 5;
  }
  cudaFree(d_xyz);
  cudaFree(d_out);
  cudaFree(d_d2);
  cudaFree(d_mask);
  return rc;
}
