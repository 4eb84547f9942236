// Neighbour lists within a cutoff, as CSR, from the rows of a finished
// search: the downstream consumer of an n x k neighbour list that keeps only
// the pairs closer than a cutoff (a force or interaction stencil), built on
// the device without a host round trip.
//
// Rows are sorted ascending by distance and padded with -1 / NaN, so the
// kept entries of a row are its leading ones: a count per row, an exclusive
// scan of the counts into the row pointers, then a copy of the leading
// entries, in row order.
#include "lc_kernels.h"

namespace lc {

namespace {

__global__ void k_csr_count(const int *__restrict__ nn, const double *__restrict__ d2,
                            long long rows, int k, double cut2, uint32_t *__restrict__ counts) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    const int *rn = nn + r * k;
    const double *rd = d2 + r * k;
    int c = 0;
    while (c < k && rn[c] >= 0 && rd[c] <= cut2) ++c;
    counts[r] = uint32_t(c);
  }
}

__global__ void k_csr_fill(const int *__restrict__ nn, const double *__restrict__ d2,
                           long long rows, int k, const uint32_t *__restrict__ counts,
                           const uint32_t *__restrict__ row_off, int *__restrict__ row_ptr,
                           int *__restrict__ col, double *__restrict__ dist2, long long cap) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    const long long o = row_off[r];
    row_ptr[r] = int(o);
    if (r == rows - 1) row_ptr[rows] = int(o + counts[r]);
    const int c = int(counts[r]);
    for (int j = 0; j < c && o + j < cap; ++j) {
      col[o + j] = nn[r * k + j];
      if (dist2) dist2[o + j] = d2[r * k + j];
    }
  }
}

int grid_rows(long long rows) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (rows + 255) / 256;
  return int(want < 1 ? 1 : (want < sms * 8LL ? want : sms * 8LL));
}

}  // namespace

cudaError_t launch_csr(const int *nn, const double *d2, long long rows, int k, double cutoff,
                       uint32_t *counts, uint32_t *row_off, unsigned long long *tile_state,
                       uint32_t *tile_counter, int *status, int *row_ptr, int *col,
                       double *dist2, long long cap, cudaStream_t s) {
  const double cut2 = cutoff * cutoff;
  k_csr_count<<<grid_rows(rows), 256, 0, s>>>(nn, d2, rows, k, cut2, counts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // the cell-count scan serves row counts as well
  BatchBuffers sb;
  sb.count = counts;
  sb.off = row_off;
  sb.ncells = rows;
  sb.tile_state = tile_state;
  sb.tile_counter = tile_counter;
  sb.status = status;
  const long long tiles = scan_tiles(rows);
  if ((e = cudaMemsetAsync(tile_state, 0, size_t(tiles) * sizeof(unsigned long long), s)) !=
          cudaSuccess ||
      (e = cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), s)) != cudaSuccess)
    return e;
  if ((e = launch_scan(sb, s)) != cudaSuccess) return e;
  k_csr_fill<<<grid_rows(rows), 256, 0, s>>>(nn, d2, rows, k, counts, row_off, row_ptr, col, dist2,
                                             cap);
  return cudaGetLastError();
}

}  // namespace lc
