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
//   - k_cell_proposal_tc: inference over 16-cell row tiles on the tensor
//     cores (mma.sync FP16, FP32 accumulation; layer 1 as a 5x5x5
//     convolution of the staged occupancy halo), writing the proposed shell
//     of every occupied cell (the smallest R with P(settled shell <= R) >=
//     tau); the walk reads it for each source.
//
// Parameter layout (floats): W1[64][126] b1[64] W2[64][64] b2[64]
// W3[8][64] b3[8].
#include <cuda_fp16.h>
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
// Tensor-core inference: mma.sync m16n8k16 FP16 (FP32 accumulate; FP16 keeps
// the 10-bit significand of TF32). One warp evaluates a row tile of 16
// consecutive cells along x: layer 1 is [16 x 128] x [128 x 64] (126
// features padded with zeros), layer 2 [16 x 64] x [64 x 64], layer 3
// [16 x 64] x [64 x 8]. The 125 occupancy features of the tile's cells all
// come from one 20 x 5 x 5 halo of log(1 + occupancy) values staged in
// shared memory, so layer 1 is a 5x5x5 convolution: A[m][f] =
// halo[yz(f)][m + dx(f)], read through a 128-entry offset table. The hidden
// layers go through shared memory to change from the accumulator layout to
// the A-operand layout.
constexpr int kW1Stride = 136;  // halves per W1 row: conflict-free B-fragment loads
constexpr int kW2Stride = 72;   // halves per W2 / W3 / hidden row
constexpr int kTcWarps = 8;
constexpr int kHaloX = 24;      // 20 used
constexpr int kHaloK = 25 * kHaloX;        // the constant feature k / 64
constexpr int kHaloZero = kHaloK + 16;     // zero padding features
constexpr int kHaloSize = kHaloZero + 32;

struct TcShared {
  __half w1[kMlpHidden * kW1Stride];
  __half w2[kMlpHidden * kW2Stride];
  __half w3[kMlpOut * kW2Stride];
  float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpOut];
  float lg1p[64];   // log(1 + c) for occupancies c < 64
  int toff[128];    // halo offset of feature f for cell 0 of the tile
  __half h[kTcWarps][16 * kW2Stride];
  __half halo[kTcWarps][kHaloSize];
};

__device__ __forceinline__ void mma_f16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                        uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_h2(__half lo, __half hi) {
  return uint32_t(__half_as_ushort(lo)) | (uint32_t(__half_as_ushort(hi)) << 16);
}

__device__ __forceinline__ uint32_t ld_h2(const __half *p) {
  return *reinterpret_cast<const uint32_t *>(p);
}

// SiLU with the fast division (inference only).
__device__ __forceinline__ float silu_fast(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// Periodic coordinate c + d for |d| <= 2.
__device__ __forceinline__ int wrap_near(int c, int n) {
  if (n < 3) return rem_euclid(c, n);
  return c < 0 ? c + n : (c >= n ? c - n : c);
}

__global__ void __launch_bounds__(kTcWarps * 32, 1) k_cell_proposal_tc(
    const float *__restrict__ params, const FrameDesc *__restrict__ frames, int nframes,
    const uint32_t *__restrict__ off, const uint32_t *__restrict__ count, float tau,
    int8_t *__restrict__ cell_prop) {
  extern __shared__ float smem_raw[];
  TcShared &sh = *reinterpret_cast<TcShared *>(smem_raw);
  const float *W1 = params, *B1 = W1 + kMlpHidden * kMlpIn;
  const float *W2 = B1 + kMlpHidden, *B2 = W2 + kMlpHidden * kMlpHidden;
  const float *W3 = B2 + kMlpHidden, *B3 = W3 + kMlpOut * kMlpHidden;
  for (int t = threadIdx.x; t < kMlpHidden * kW1Stride; t += blockDim.x) {
    const int n = t / kW1Stride, kk = t % kW1Stride;
    sh.w1[t] = __float2half_rn(kk < kMlpIn ? W1[n * kMlpIn + kk] : 0.f);
  }
  for (int t = threadIdx.x; t < kMlpHidden * kW2Stride; t += blockDim.x) {
    const int n = t / kW2Stride, kk = t % kW2Stride;
    sh.w2[t] = __float2half_rn(kk < kMlpHidden ? W2[n * kMlpHidden + kk] : 0.f);
  }
  for (int t = threadIdx.x; t < kMlpOut * kW2Stride; t += blockDim.x) {
    const int n = t / kW2Stride, kk = t % kW2Stride;
    sh.w3[t] = __float2half_rn(kk < kMlpHidden ? W3[n * kMlpHidden + kk] : 0.f);
  }
  for (int t = threadIdx.x; t < kMlpHidden; t += blockDim.x) {
    sh.b1[t] = B1[t];
    sh.b2[t] = B2[t];
  }
  if (threadIdx.x < kMlpOut) sh.b3[threadIdx.x] = B3[threadIdx.x];
  if (threadIdx.x < 64) sh.lg1p[threadIdx.x] = log1pf(float(threadIdx.x));
  if (threadIdx.x < 128) {
    // feature f = (dx + 2) * 25 + (dy + 2) * 5 + (dz + 2); halo row (dy + 2) * 5 + (dz + 2)
    const int f = threadIdx.x;
    sh.toff[f] = f < 125 ? (f % 25) * kHaloX + f / 25 : (f == 125 ? kHaloK : kHaloZero);
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tig = lane & 3;
  __half *hbuf = sh.h[warp];
  __half *halo = sh.halo[warp];
  const FrameDesc &last = frames[nframes - 1];
  const long long tiles = last.row_tile_base + (long long)((last.nx + 15) / 16) * last.ny * last.nz;
  for (long long tile = (long long)blockIdx.x * kTcWarps + warp; tile < tiles;
       tile += (long long)gridDim.x * kTcWarps) {
    int f = 0;
    if (nframes > 1) {
      int lo = 0, hi = nframes - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (frames[mid].row_tile_base <= tile)
          lo = mid;
        else
          hi = mid - 1;
      }
      f = lo;
    }
    const FrameDesc &fr = frames[f];
    const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
    const int per_row = (nx + 15) / 16;
    const long long lt = tile - fr.row_tile_base;
    const int row = int(lt / per_row);
    const int x0 = int(lt - (long long)row * per_row) * 16;
    const int cy = row % ny, cz = row / ny;
    const int ncl = min(16, nx - x0);
    const long long c0 = fr.cell_base + (long long)row * nx + x0;
    if (off[c0] == off[c0 + ncl]) continue;  // no occupied cell in the tile
    // halo: x0 - 2 .. x0 + 17, cy - 2 .. cy + 2, cz - 2 .. cz + 2 (periodic)
    __syncwarp();
    for (int hidx = lane; hidx < 25 * 20; hidx += 32) {
      const int yz = hidx / 20, xx = hidx - yz * 20;
      const int jy = wrap_near(cy + yz / 5 - 2, ny);
      const int jz = wrap_near(cz + yz % 5 - 2, nz);
      const int jx = (nx >= 20) ? wrap_near(x0 + xx - 2, nx) : rem_euclid(x0 + xx - 2, nx);
      const uint32_t cnt = count[fr.cell_base + ((long long)jz * ny + jy) * (long long)nx + jx];
      halo[yz * kHaloX + xx] = __float2half_rn(cnt < 64u ? sh.lg1p[cnt] : log1pf(float(cnt)));
    }
    if (lane < 16) {
      halo[kHaloK + lane] = __float2half_rn(float(fr.k) / 64.0f);
      halo[kHaloZero + lane] = __float2half_rn(0.f);
      halo[kHaloZero + 16 + lane] = __float2half_rn(0.f);
    }
    __syncwarp();
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
#pragma unroll 2
    for (int k0 = 0; k0 < 128; k0 += 16) {
      const int o0 = sh.toff[k0 + 2 * tig], o1 = sh.toff[k0 + 2 * tig + 1];
      const int o2 = sh.toff[k0 + 2 * tig + 8], o3 = sh.toff[k0 + 2 * tig + 9];
      const uint32_t a0 = pack_h2(halo[o0 + g], halo[o1 + g]);
      const uint32_t a1 = pack_h2(halo[o0 + g + 8], halo[o1 + g + 8]);
      const uint32_t a2 = pack_h2(halo[o2 + g], halo[o3 + g]);
      const uint32_t a3 = pack_h2(halo[o2 + g + 8], halo[o3 + g + 8]);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const __half *wr = sh.w1 + (nt * 8 + g) * kW1Stride + k0 + 2 * tig;
        mma_f16(acc[nt], a0, a1, a2, a3, ld_h2(wr), ld_h2(wr + 8));
      }
    }
    // SiLU, then to shared memory (row-major 16 x 64 halves)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * tig;
      *reinterpret_cast<__half2 *>(hbuf + g * kW2Stride + col) =
          __floats2half2_rn(silu_fast(acc[nt][0]), silu_fast(acc[nt][1]));
      *reinterpret_cast<__half2 *>(hbuf + (g + 8) * kW2Stride + col) =
          __floats2half2_rn(silu_fast(acc[nt][2]), silu_fast(acc[nt][3]));
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
    for (int k0 = 0; k0 < 64; k0 += 16) {
      const uint32_t a0 = ld_h2(hbuf + g * kW2Stride + k0 + 2 * tig);
      const uint32_t a1 = ld_h2(hbuf + (g + 8) * kW2Stride + k0 + 2 * tig);
      const uint32_t a2 = ld_h2(hbuf + g * kW2Stride + k0 + 2 * tig + 8);
      const uint32_t a3 = ld_h2(hbuf + (g + 8) * kW2Stride + k0 + 2 * tig + 8);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const __half *wr = sh.w2 + (nt * 8 + g) * kW2Stride + k0 + 2 * tig;
        mma_f16(acc[nt], a0, a1, a2, a3, ld_h2(wr), ld_h2(wr + 8));
      }
    }
    __syncwarp();
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * tig;
      *reinterpret_cast<__half2 *>(hbuf + g * kW2Stride + col) =
          __floats2half2_rn(silu_fast(acc[nt][0]), silu_fast(acc[nt][1]));
      *reinterpret_cast<__half2 *>(hbuf + (g + 8) * kW2Stride + col) =
          __floats2half2_rn(silu_fast(acc[nt][2]), silu_fast(acc[nt][3]));
    }
    __syncwarp();
    // layer 3: 8 logits per cell
    float z[4] = {sh.b3[2 * tig], sh.b3[2 * tig + 1], sh.b3[2 * tig], sh.b3[2 * tig + 1]};
#pragma unroll
    for (int k0 = 0; k0 < 64; k0 += 16) {
      const uint32_t a0 = ld_h2(hbuf + g * kW2Stride + k0 + 2 * tig);
      const uint32_t a1 = ld_h2(hbuf + (g + 8) * kW2Stride + k0 + 2 * tig);
      const uint32_t a2 = ld_h2(hbuf + g * kW2Stride + k0 + 2 * tig + 8);
      const uint32_t a3 = ld_h2(hbuf + (g + 8) * kW2Stride + k0 + 2 * tig + 8);
      const __half *wr = sh.w3 + g * kW2Stride + k0 + 2 * tig;
      mma_f16(z, a0, a1, a2, a3, ld_h2(wr), ld_h2(wr + 8));
    }
    // each quad holds the 8 logits of rows g (z[0], z[1]) and g + 8 (z[2], z[3])
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float lg[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        lg[2 * q] = __shfl_sync(0xffffffffu, z[2 * h], (lane & ~3) | q);
        lg[2 * q + 1] = __shfl_sync(0xffffffffu, z[2 * h + 1], (lane & ~3) | q);
      }
      const int m = g + 8 * h;
      if (tig == 0 && m < ncl) {
        float mx = lg[0];
#pragma unroll
        for (int o = 1; o < 8; ++o) mx = fmaxf(mx, lg[o]);
        float e[8], sum = 0.f;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
          e[o] = __expf(lg[o] - mx);
          sum += e[o];
        }
        int prop = kMlpOut;
        float cum = 0.f;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
          cum += e[o] / sum;
          if (cum >= tau && prop == kMlpOut) prop = o + 1;
        }
        cell_prop[c0 + m] = int8_t(prop >= kMlpOut ? 0 : prop);
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
                        int8_t *source_prop, float tau, cudaStream_t s) {
  if (b.nframes <= 0 || b.ncells <= 0) return cudaSuccess;
  const size_t sm = sizeof(TcShared);
  cudaError_t e =
      cudaFuncSetAttribute(k_cell_proposal_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cell_proposal_tc, kTcWarps * 32, sm);
  if (per_sm < 1) per_sm = 1;
  k_cell_proposal_tc<<<sms * per_sm, kTcWarps * 32, sm, s>>>(params, b.frames, b.nframes, b.off,
                                                              b.count, tau, cell_prop);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_source_proposal<<<grid_of(b.npts, 256), 256, 0, s>>>(b.frames, b.nframes, b.off, b.ncells,
                                                         b.scell, cell_prop, source_prop);
  return cudaGetLastError();
}

}  // namespace lc
