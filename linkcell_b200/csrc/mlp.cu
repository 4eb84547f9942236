// Learned shell proposal: a 126 -> 64 -> 64 -> 8 MLP (SiLU, softmax) that
// reads the occupancy of the 5x5x5 cells around a source's home cell plus
// k / 64 and proposes the shell at which the walk settles.
//
// Hand-written FP32 kernels:
//   - k_cell_features: log(1 + occupancy) of the 125 neighbours (periodic)
//     and k / 64, for a list of cells;
//   - forward (k_dense: tiled FP32 GEMM with bias and optional SiLU),
//     softmax cross-entropy, backward (GEMMs for input and weight
//     gradients, SiLU derivative), and Adam;
//   - k_cell_proposal_tc: inference per non-empty cell on the tensor cores
//     (mma.sync TF32, FP32 accumulation), writing the proposed shell of
//     every cell (the smallest R with P(settled shell <= R) >= tau); the
//     walk reads it for each source.
//
// Parameter layout (floats): W1[64][126] b1[64] W2[64][64] b2[64]
// W3[8][64] b3[8].
#include <cuda_runtime.h>

#include <cmath>

#include "lc_kernels.h"
#include "lc_mlp.h"

namespace lc {

namespace {

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// 125 occupancy features of cell (cx, cy, cz) in frame fr, then k / 64.
__device__ __forceinline__ void cell_features(const FrameDesc &fr, const uint32_t *off, int cx,
                                              int cy, int cz, float *x) {
  int t = 0;
  for (int dx = -2; dx <= 2; ++dx) {
    const int jx = rem_euclid(cx + dx, fr.nx);
    for (int dy = -2; dy <= 2; ++dy) {
      const int jy = rem_euclid(cy + dy, fr.ny);
      for (int dz = -2; dz <= 2; ++dz) {
        const int jz = rem_euclid(cz + dz, fr.nz);
        const long long c = fr.cell_base + ((long long)jz * fr.ny + jy) * (long long)fr.nx + jx;
        x[t++] = log1pf(float(off[c + 1] - off[c]));
      }
    }
  }
  x[125] = float(fr.k) / 64.0f;
}

// Features of listed cells (local cell ids of frame 0..): one thread per row.
__global__ void k_cell_features(const FrameDesc *__restrict__ frames, const uint32_t *__restrict__ off,
                                const int *__restrict__ frame_of_row,
                                const uint32_t *__restrict__ cell_of_row, long long rows,
                                float *__restrict__ X) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    const FrameDesc &fr = frames[frame_of_row ? frame_of_row[r] : 0];
    const uint32_t lc = cell_of_row[r];
    const int cx = int(lc % uint32_t(fr.nx));
    const int cy = int((lc / uint32_t(fr.nx)) % uint32_t(fr.ny));
    const int cz = int(lc / (uint32_t(fr.nx) * uint32_t(fr.ny)));
    float x[kMlpIn];
    cell_features(fr, off, cx, cy, cz, x);
    for (int t = 0; t < kMlpIn; ++t) X[r * kMlpIn + t] = x[t];
  }
}

// C[M x N] = act(A[M x K] * W[N x K]^T + bias[N]); act = SiLU or identity.
// Zpre (optional) receives the pre-activation.
constexpr int kTile = 16;
__global__ void k_dense(const float *__restrict__ A, const float *__restrict__ W,
                        const float *__restrict__ bias, float *__restrict__ C,
                        float *__restrict__ Zpre, int M, int N, int K, int act) {
  __shared__ float sa[kTile][kTile + 1];
  __shared__ float sw[kTile][kTile + 1];
  const int row = blockIdx.y * kTile + threadIdx.y;
  const int col = blockIdx.x * kTile + threadIdx.x;
  float acc = 0.f;
  for (int k0 = 0; k0 < K; k0 += kTile) {
    const int ka = k0 + threadIdx.x;
    sa[threadIdx.y][threadIdx.x] = (row < M && ka < K) ? A[(long long)row * K + ka] : 0.f;
    const int wr = blockIdx.x * kTile + threadIdx.y;
    sw[threadIdx.y][threadIdx.x] = (wr < N && ka < K) ? W[(long long)wr * K + ka] : 0.f;
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kTile; ++t) acc = fmaf(sa[threadIdx.y][t], sw[threadIdx.x][t], acc);
    __syncthreads();
  }
  if (row < M && col < N) {
    const float z = acc + (bias ? bias[col] : 0.f);
    if (Zpre) Zpre[(long long)row * N + col] = z;
    C[(long long)row * N + col] = act ? silu(z) : z;
  }
}

// dA[M x K] = dZ[M x N] * W[N x K]; optionally times SiLU'(Zprev).
__global__ void k_dense_back_input(const float *__restrict__ dZ, const float *__restrict__ W,
                                   const float *__restrict__ Zprev, float *__restrict__ dA, int M,
                                   int N, int K) {
  __shared__ float sd[kTile][kTile + 1];
  __shared__ float sw[kTile][kTile + 1];
  const int row = blockIdx.y * kTile + threadIdx.y;
  const int col = blockIdx.x * kTile + threadIdx.x;  // in K
  float acc = 0.f;
  for (int n0 = 0; n0 < N; n0 += kTile) {
    const int nd = n0 + threadIdx.x;
    sd[threadIdx.y][threadIdx.x] = (row < M && nd < N) ? dZ[(long long)row * N + nd] : 0.f;
    const int nw = n0 + threadIdx.y;
    sw[threadIdx.y][threadIdx.x] = (nw < N && col < K) ? W[(long long)nw * K + col] : 0.f;
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kTile; ++t) acc = fmaf(sd[threadIdx.y][t], sw[t][threadIdx.x], acc);
    __syncthreads();
  }
  if (row < M && col < K) {
    const long long o = (long long)row * K + col;
    dA[o] = Zprev ? acc * silu_grad(Zprev[o]) : acc;
  }
}

// dW[N x K] = dZ[M x N]^T * A[M x K];  db[N] = sum_m dZ[m][n].
__global__ void k_dense_back_weight(const float *__restrict__ dZ, const float *__restrict__ A,
                                    float *__restrict__ dW, float *__restrict__ db, int M, int N,
                                    int K) {
  __shared__ float sd[kTile][kTile + 1];
  __shared__ float sa[kTile][kTile + 1];
  const int n = blockIdx.y * kTile + threadIdx.y;
  const int kk = blockIdx.x * kTile + threadIdx.x;
  float acc = 0.f, bacc = 0.f;
  for (int m0 = 0; m0 < M; m0 += kTile) {
    const int md = m0 + threadIdx.x;
    sd[threadIdx.y][threadIdx.x] =
        (md < M && (blockIdx.y * kTile + threadIdx.y) < N)
            ? dZ[(long long)md * N + blockIdx.y * kTile + threadIdx.y]
            : 0.f;
    const int ma = m0 + threadIdx.y;
    sa[threadIdx.y][threadIdx.x] = (ma < M && kk < K) ? A[(long long)ma * K + kk] : 0.f;
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kTile; ++t) {
      acc = fmaf(sd[threadIdx.y][t], sa[t][threadIdx.x], acc);
      bacc += sd[threadIdx.y][t];
    }
    __syncthreads();
  }
  if (n < N && kk < K) dW[(long long)n * K + kk] = acc;
  if (db && n < N && blockIdx.x == 0 && threadIdx.x == 0) db[n] = bacc;
}

// Softmax cross-entropy over 8 classes: dZ = (softmax - onehot) / B,
// loss accumulated as the mean negative log-likelihood.
__global__ void k_softmax_ce(const float *__restrict__ Z, const int *__restrict__ y, int B,
                             float *__restrict__ dZ, float *__restrict__ probs,
                             float *__restrict__ loss) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (r < B) {
    float m = Z[r * kMlpOut];
    for (int c = 1; c < kMlpOut; ++c) m = fmaxf(m, Z[r * kMlpOut + c]);
    float e[kMlpOut], s = 0.f;
    for (int c = 0; c < kMlpOut; ++c) {
      e[c] = expf(Z[r * kMlpOut + c] - m);
      s += e[c];
    }
    const int cls = y ? y[r] : -1;
    for (int c = 0; c < kMlpOut; ++c) {
      const float pc = e[c] / s;
      if (probs) probs[r * kMlpOut + c] = pc;
      if (dZ) dZ[r * kMlpOut + c] = (pc - (c == cls ? 1.f : 0.f)) / float(B);
    }
    if (cls >= 0) l = -(Z[r * kMlpOut + cls] - m - logf(s)) / float(B);
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) l += __shfl_xor_sync(0xffffffffu, l, d);
  if (loss && (threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// proposal per sorted source = proposal of its cell
__global__ void k_source_proposal(const FrameDesc *__restrict__ frames, int nframes,
                                  const uint32_t *__restrict__ off, long long ncells,
                                  const uint32_t *__restrict__ scell,
                                  const int8_t *__restrict__ cell_prop, int8_t *__restrict__ prop) {
  const long long total = off[ncells];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < total;
       p += (long long)gridDim.x * blockDim.x) {
    int f = 0;
    if (nframes > 1) {
      int lo = 0, hi = nframes - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)off[frames[mid].cell_base] <= p)
          lo = mid;
        else
          hi = mid - 1;
      }
      f = lo;
    }
    prop[p] = cell_prop[frames[f].cell_base + scell[p]];
  }
}

// Training rows: sorted sources first, first + stride, ... with the
// features of their home cell and the class of their settled shell.
__global__ void k_training_rows(BatchBuffers b, const int8_t *__restrict__ stop_log,
                                long long stride, long long first, float *__restrict__ X,
                                int *__restrict__ y, long long rows) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    const long long p = first + r * stride;
    int f = 0;
    if (b.nframes > 1) {
      int lo = 0, hi = b.nframes - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)b.off[b.frames[mid].cell_base] <= p)
          lo = mid;
        else
          hi = mid - 1;
      }
      f = lo;
    }
    const FrameDesc &fr = b.frames[f];
    const uint32_t lc = b.scell[p];
    const int cx = int(lc % uint32_t(fr.nx));
    const int cy = int((lc / uint32_t(fr.nx)) % uint32_t(fr.ny));
    const int cz = int(lc / (uint32_t(fr.nx) * uint32_t(fr.ny)));
    float x[kMlpIn];
    cell_features(fr, b.off, cx, cy, cz, x);
    for (int t = 0; t < kMlpIn; ++t) X[r * kMlpIn + t] = x[t];
    int R = stop_log[p];
    if (R <= 0 || R > kMlpOut) R = kMlpOut;
    y[r] = R - 1;
  }
}

// ---------------------------------------------------------------------
// Tensor-core inference: mma.sync m16n8k8 TF32 (FP32 accumulate). One warp
// evaluates 16 cells at a time: layer 1 is [16 x 128] x [128 x 64] (126
// features padded with zeros), layer 2 [16 x 64] x [64 x 64], layer 3
// [16 x 64] x [64 x 8]. Features are gathered straight into the A
// fragments; the hidden layer goes through shared memory to change from
// the accumulator layout to the A-operand layout.
constexpr int kW1Stride = 132;  // padded rows: conflict-free B-fragment loads
constexpr int kW2Stride = 68;
constexpr int kTcWarps = 4;

struct TcShared {
  float w1[kMlpHidden * kW1Stride];
  float w2[kMlpHidden * kW2Stride];
  float w3[kMlpOut * kW2Stride];
  float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpOut];
  float h[kTcWarps][16 * kW2Stride];
};

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Non-empty cells into a list (order does not matter).
__global__ void k_list_cells(const uint32_t *__restrict__ off, long long ncells,
                             uint32_t *__restrict__ list, uint32_t *__restrict__ count) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += (long long)gridDim.x * blockDim.x) {
    const bool has = off[c + 1] > off[c];
    const unsigned m = __ballot_sync(0xffffffffu, has);
    if (m == 0) continue;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(count, uint32_t(__popc(m)));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
    if (has) list[base + __popc(m & ((1u << lane) - 1u))] = uint32_t(c);
  }
}

__global__ void __launch_bounds__(kTcWarps * 32) k_cell_proposal_tc(
    const float *__restrict__ params, const FrameDesc *__restrict__ frames, int nframes,
    const uint32_t *__restrict__ off, const uint32_t *__restrict__ list,
    const uint32_t *__restrict__ list_count, float tau, int8_t *__restrict__ cell_prop) {
  extern __shared__ float smem_raw[];
  TcShared &sh = *reinterpret_cast<TcShared *>(smem_raw);
  const float *W1 = params, *B1 = W1 + kMlpHidden * kMlpIn;
  const float *W2 = B1 + kMlpHidden, *B2 = W2 + kMlpHidden * kMlpHidden;
  const float *W3 = B2 + kMlpHidden, *B3 = W3 + kMlpOut * kMlpHidden;
  for (int t = threadIdx.x; t < kMlpHidden * kW1Stride; t += blockDim.x) {
    const int n = t / kW1Stride, kk = t % kW1Stride;
    sh.w1[t] = kk < kMlpIn ? __uint_as_float(to_tf32(W1[n * kMlpIn + kk])) : 0.f;
  }
  for (int t = threadIdx.x; t < kMlpHidden * kW2Stride; t += blockDim.x) {
    const int n = t / kW2Stride, kk = t % kW2Stride;
    sh.w2[t] = kk < kMlpHidden ? __uint_as_float(to_tf32(W2[n * kMlpHidden + kk])) : 0.f;
  }
  for (int t = threadIdx.x; t < kMlpOut * kW2Stride; t += blockDim.x) {
    const int n = t / kW2Stride, kk = t % kW2Stride;
    sh.w3[t] = kk < kMlpHidden ? __uint_as_float(to_tf32(W3[n * kMlpHidden + kk])) : 0.f;
  }
  for (int t = threadIdx.x; t < kMlpHidden; t += blockDim.x) {
    sh.b1[t] = B1[t];
    sh.b2[t] = B2[t];
  }
  if (threadIdx.x < kMlpOut) sh.b3[threadIdx.x] = B3[threadIdx.x];
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tig = lane & 3;
  const uint32_t ncl = *list_count;
  float *hbuf = sh.h[warp];
  const long long tiles = (ncl + 15) / 16;
  for (long long tile = (long long)blockIdx.x * kTcWarps + warp; tile < tiles;
       tile += (long long)gridDim.x * kTcWarps) {
    // the two cells (rows g and g + 8) whose features this lane gathers
    int cxs[2], cys[2], czs[2];
    const FrameDesc *frs[2];
    bool valid[2];
    long long cellid[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long row = tile * 16 + g + 8 * h;
      valid[h] = row < ncl;
      const long long c = valid[h] ? (long long)list[row] : 0;
      cellid[h] = c;
      int f = 0;
      if (nframes > 1) {
        int lo = 0, hi = nframes - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (frames[mid].cell_base <= c)
            lo = mid;
          else
            hi = mid - 1;
        }
        f = lo;
      }
      frs[h] = &frames[f];
      const uint32_t lc = uint32_t(c - frs[h]->cell_base);
      cxs[h] = int(lc % uint32_t(frs[h]->nx));
      cys[h] = int((lc / uint32_t(frs[h]->nx)) % uint32_t(frs[h]->ny));
      czs[h] = int(lc / (uint32_t(frs[h]->nx) * uint32_t(frs[h]->ny)));
    }
    auto feature = [&](int h, int fi) -> float {
      if (!valid[h]) return 0.f;
      const FrameDesc &fr = *frs[h];
      if (fi < 125) {
        const int dx = fi / 25 - 2, dy = (fi / 5) % 5 - 2, dz = fi % 5 - 2;
        const int jx = rem_euclid(cxs[h] + dx, fr.nx);
        const int jy = rem_euclid(cys[h] + dy, fr.ny);
        const int jz = rem_euclid(czs[h] + dz, fr.nz);
        const long long q = fr.cell_base + ((long long)jz * fr.ny + jy) * (long long)fr.nx + jx;
        return log1pf(float(off[q + 1] - off[q]));
      }
      return fi == 125 ? float(fr.k) / 64.0f : 0.f;
    };
    // layer 1
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float b0 = sh.b1[nt * 8 + 2 * tig], b1v = sh.b1[nt * 8 + 2 * tig + 1];
      acc[nt][0] = b0;
      acc[nt][1] = b1v;
      acc[nt][2] = b0;
      acc[nt][3] = b1v;
    }
    for (int k0 = 0; k0 < 128; k0 += 8) {
      const uint32_t a0 = to_tf32(feature(0, k0 + tig));
      const uint32_t a1 = to_tf32(feature(1, k0 + tig));
      const uint32_t a2 = to_tf32(feature(0, k0 + tig + 4));
      const uint32_t a3 = to_tf32(feature(1, k0 + tig + 4));
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int n = nt * 8 + g;
        const uint32_t b0 = __float_as_uint(sh.w1[n * kW1Stride + k0 + tig]);
        const uint32_t b1 = __float_as_uint(sh.w1[n * kW1Stride + k0 + tig + 4]);
        mma_tf32(acc[nt], a0, a1, a2, a3, b0, b1);
      }
    }
    // SiLU, then to shared memory (row-major 16 x 64)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * tig;
      hbuf[g * kW2Stride + col] = silu(acc[nt][0]);
      hbuf[g * kW2Stride + col + 1] = silu(acc[nt][1]);
      hbuf[(g + 8) * kW2Stride + col] = silu(acc[nt][2]);
      hbuf[(g + 8) * kW2Stride + col + 1] = silu(acc[nt][3]);
    }
    __syncwarp();
    // layer 2
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float b0 = sh.b2[nt * 8 + 2 * tig], b1v = sh.b2[nt * 8 + 2 * tig + 1];
      acc[nt][0] = b0;
      acc[nt][1] = b1v;
      acc[nt][2] = b0;
      acc[nt][3] = b1v;
    }
#pragma unroll
    for (int k0 = 0; k0 < 64; k0 += 8) {
      const uint32_t a0 = to_tf32(hbuf[g * kW2Stride + k0 + tig]);
      const uint32_t a1 = to_tf32(hbuf[(g + 8) * kW2Stride + k0 + tig]);
      const uint32_t a2 = to_tf32(hbuf[g * kW2Stride + k0 + tig + 4]);
      const uint32_t a3 = to_tf32(hbuf[(g + 8) * kW2Stride + k0 + tig + 4]);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int n = nt * 8 + g;
        const uint32_t b0 = __float_as_uint(sh.w2[n * kW2Stride + k0 + tig]);
        const uint32_t b1 = __float_as_uint(sh.w2[n * kW2Stride + k0 + tig + 4]);
        mma_tf32(acc[nt], a0, a1, a2, a3, b0, b1);
      }
    }
    __syncwarp();
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * tig;
      hbuf[g * kW2Stride + col] = silu(acc[nt][0]);
      hbuf[g * kW2Stride + col + 1] = silu(acc[nt][1]);
      hbuf[(g + 8) * kW2Stride + col] = silu(acc[nt][2]);
      hbuf[(g + 8) * kW2Stride + col + 1] = silu(acc[nt][3]);
    }
    __syncwarp();
    // layer 3: 8 logits per cell
    float z[4] = {sh.b3[2 * tig], sh.b3[2 * tig + 1], sh.b3[2 * tig], sh.b3[2 * tig + 1]};
#pragma unroll
    for (int k0 = 0; k0 < 64; k0 += 8) {
      const uint32_t a0 = to_tf32(hbuf[g * kW2Stride + k0 + tig]);
      const uint32_t a1 = to_tf32(hbuf[(g + 8) * kW2Stride + k0 + tig]);
      const uint32_t a2 = to_tf32(hbuf[g * kW2Stride + k0 + tig + 4]);
      const uint32_t a3 = to_tf32(hbuf[(g + 8) * kW2Stride + k0 + tig + 4]);
      const uint32_t b0 = __float_as_uint(sh.w3[g * kW2Stride + k0 + tig]);
      const uint32_t b1 = __float_as_uint(sh.w3[g * kW2Stride + k0 + tig + 4]);
      mma_tf32(z, a0, a1, a2, a3, b0, b1);
    }
    __syncwarp();
    // each quad holds the 8 logits of rows g (z[0], z[1]) and g + 8 (z[2], z[3])
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float lg[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        lg[2 * q] = __shfl_sync(0xffffffffu, z[2 * h], (lane & ~3) | q);
        lg[2 * q + 1] = __shfl_sync(0xffffffffu, z[2 * h + 1], (lane & ~3) | q);
      }
      if (tig == 0 && valid[h]) {
        float m = lg[0];
#pragma unroll
        for (int o = 1; o < 8; ++o) m = fmaxf(m, lg[o]);
        float e[8], sum = 0.f;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
          e[o] = __expf(lg[o] - m);
          sum += e[o];
        }
        int prop = kMlpOut;
        float cum = 0.f;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
          cum += e[o] / sum;
          if (cum >= tau && prop == kMlpOut) prop = o + 1;
        }
        cell_prop[cellid[h]] = int8_t(prop >= kMlpOut ? 0 : prop);
      }
    }
    __syncwarp();
  }
}

int grid_of(long long n, int block, int cap_per_sm = 8) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long g = (n + block - 1) / block;
  const long long cap = (long long)sms * cap_per_sm;
  if (g > cap) g = cap;
  return int(g < 1 ? 1 : g);
}

}  // namespace

cudaError_t mlp_cell_features(const FrameDesc *frames, const uint32_t *off,
                              const int *frame_of_row, const uint32_t *cell_of_row, long long rows,
                              float *X, cudaStream_t s) {
  if (rows <= 0) return cudaSuccess;
  k_cell_features<<<grid_of(rows, 128), 128, 0, s>>>(frames, off, frame_of_row, cell_of_row, rows,
                                                      X);
  return cudaGetLastError();
}

cudaError_t mlp_forward(const float *params, const float *X, int B, MlpScratch &t, float *probs,
                        cudaStream_t s) {
  const float *W1 = params, *b1 = W1 + kMlpHidden * kMlpIn;
  const float *W2 = b1 + kMlpHidden, *b2 = W2 + kMlpHidden * kMlpHidden;
  const float *W3 = b2 + kMlpHidden, *b3 = W3 + kMlpOut * kMlpHidden;
  const dim3 blk(kTile, kTile);
  const unsigned gy = unsigned((B + kTile - 1) / kTile);
  k_dense<<<dim3((kMlpHidden + kTile - 1) / kTile, gy), blk, 0, s>>>(X, W1, b1, t.h1, t.z1, B,
                                                                     kMlpHidden, kMlpIn, 1);
  k_dense<<<dim3((kMlpHidden + kTile - 1) / kTile, gy), blk, 0, s>>>(t.h1, W2, b2, t.h2, t.z2, B,
                                                                     kMlpHidden, kMlpHidden, 1);
  k_dense<<<dim3(1, gy), blk, 0, s>>>(t.h2, W3, b3, t.z3, nullptr, B, kMlpOut, kMlpHidden, 0);
  if (probs)
    k_softmax_ce<<<(B + 127) / 128, 128, 0, s>>>(t.z3, nullptr, B, nullptr, probs, nullptr);
  return cudaGetLastError();
}

cudaError_t mlp_grad(const float *params, const float *X, const int *y, int B, MlpScratch &t,
                     float *grad, float *loss, cudaStream_t s) {
  cudaError_t e = mlp_forward(params, X, B, t, nullptr, s);
  if (e != cudaSuccess) return e;
  const float *W2 = params + kMlpHidden * kMlpIn + kMlpHidden;
  const float *W3 = W2 + kMlpHidden * kMlpHidden + kMlpHidden;
  float *gW1 = grad, *gb1 = gW1 + kMlpHidden * kMlpIn;
  float *gW2 = gb1 + kMlpHidden, *gb2 = gW2 + kMlpHidden * kMlpHidden;
  float *gW3 = gb2 + kMlpHidden, *gb3 = gW3 + kMlpOut * kMlpHidden;
  if (loss) cudaMemsetAsync(loss, 0, sizeof(float), s);
  k_softmax_ce<<<(B + 127) / 128, 128, 0, s>>>(t.z3, y, B, t.dz3, nullptr, loss);
  const dim3 blk(kTile, kTile);
  const unsigned gy = unsigned((B + kTile - 1) / kTile);
  // layer 3
  k_dense_back_weight<<<dim3((kMlpHidden + kTile - 1) / kTile, 1), blk, 0, s>>>(
      t.dz3, t.h2, gW3, gb3, B, kMlpOut, kMlpHidden);
  k_dense_back_input<<<dim3((kMlpHidden + kTile - 1) / kTile, gy), blk, 0, s>>>(
      t.dz3, W3, t.z2, t.dz2, B, kMlpOut, kMlpHidden);
  // layer 2
  k_dense_back_weight<<<dim3((kMlpHidden + kTile - 1) / kTile, (kMlpHidden + kTile - 1) / kTile),
                        blk, 0, s>>>(t.dz2, t.h1, gW2, gb2, B, kMlpHidden, kMlpHidden);
  k_dense_back_input<<<dim3((kMlpHidden + kTile - 1) / kTile, gy), blk, 0, s>>>(
      t.dz2, W2, t.z1, t.dz1, B, kMlpHidden, kMlpHidden);
  // layer 1
  k_dense_back_weight<<<dim3((kMlpIn + kTile - 1) / kTile, (kMlpHidden + kTile - 1) / kTile), blk,
                        0, s>>>(t.dz1, X, gW1, gb1, B, kMlpHidden, kMlpIn);
  return cudaGetLastError();
}

cudaError_t mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr,
                     cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - std::pow(b1, float(step));
  const float c2 = 1.f - std::pow(b2, float(step));
  k_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, kMlpParams, lr, b1, b2, eps,
                                                  c1, c2);
  return cudaGetLastError();
}

cudaError_t mlp_training_rows(const BatchBuffers &b, const int8_t *stop_log, long long stride,
                              long long first, float *X, int *y, long long cap, cudaStream_t s) {
  if (cap <= 0) return cudaSuccess;
  k_training_rows<<<grid_of(cap, 128), 128, 0, s>>>(b, stop_log, stride, first, X, y, cap);
  return cudaGetLastError();
}

cudaError_t mlp_propose(const float *params, const BatchBuffers &b, int8_t *cell_prop,
                        int8_t *source_prop, float tau, uint32_t *cell_list, uint32_t *list_count,
                        cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(list_count, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  k_list_cells<<<grid_of(b.ncells, 256), 256, 0, s>>>(b.off, b.ncells, cell_list, list_count);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const size_t sm = sizeof(TcShared);
  e = cudaFuncSetAttribute(k_cell_proposal_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_cell_proposal_tc<<<sms * 3, kTcWarps * 32, sm, s>>>(params, b.frames, b.nframes, b.off,
                                                         cell_list, list_count, tau, cell_prop);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_source_proposal<<<grid_of(b.npts, 256), 256, 0, s>>>(b.frames, b.nframes, b.off, b.ncells,
                                                         b.scell, cell_prop, source_prop);
  return cudaGetLastError();
}

}  // namespace lc
