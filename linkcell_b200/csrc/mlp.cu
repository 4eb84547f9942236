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
//   - k_cell_proposal_tc: inference over 128-cell tiles on the tcgen05
//     tensor cores (FP16 operands in shared memory, FP32 accumulators in
//     tensor memory; layer 1 as a 5x5x5 convolution of the staged occupancy
//     halo), writing the proposed shell of every cell (the smallest R with
//     P(settled shell <= R) >= tau); the walk reads it for each source.
//
// Parameter layout (floats): W1[64][126] b1[64] W2[64][64] b2[64]
// W3[8][64] b3[8].
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
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
// Tensor-core inference on the 5th-generation tensor cores (tcgen05). A
// group of four warps evaluates 128 cells at a time -- a 16 x 8-cell tile,
// two 16-cell rows per warp and lane quarter of tensor memory -- as
// the M = 128 rows of the three layers:
//   D1 = A1 W1^T  (A1: [128 x 128] occupancy features, 126 used),
//   D2 = SiLU(D1 + b1) W2^T,  D3 = SiLU(D2 + b2) W3^T  (N = 64, 64, 16 with 8 used).
// The group's first thread issues tcgen05.mma (kind::f16: FP16 operands that
// the tensor cores read from shared memory through matrix descriptors, FP32
// accumulators in tensor memory) and tcgen05.commit, which arrives on the
// group's mbarrier once the products are done; every warp then reads its 32
// accumulator lanes with tcgen05.ld, adds the bias, applies SiLU and writes
// the next layer's A operand. Layer 1 is a 5x5x5 convolution of the
// occupancy grid: the group stages the tile's 20 x 12 x 5 halo of
// log(1 + count), and each lane writes its cell's 128 features (16-byte
// chunks) from it, in two K halves.
//
// Operand layout (K-major, no swizzle): 8-row x 16-byte core matrices; the 8
// rows of a core matrix are 16 B apart, 8-row groups SBO = 128 B apart, and
// the 16-byte K chunks LBO apart (LBO = rows x 16 B).
constexpr int kUmmaThreads = 256;   // two groups of four warps
// halves per halo row: x0 - 2 .. x0 + 17. Lanes 16-31 read the halo five rows
// (200 bytes) after lanes 0-15, which puts their 32-byte spans on other banks.
constexpr int kHaloW = kPropTileX + 4;
constexpr int kHaloRows = (kPropTileY + 4) * 5;  // halo rows of a tile: 12 y x 5 z
constexpr int kMbarSpin = 1 << 22;  // bounded wait for the tensor cores
// A CTA runs kGroups groups of four warps (one per lane quarter of tensor
// memory), each on its own tile with its own operand buffer, halo, 64
// accumulator columns (D1, D2 and D3 share them), barrier and mbarrier, so
// that one group's waits for the tensor cores overlap the other's work.
constexpr int kGroups = 2;
constexpr int kGroupThreads = kUmmaThreads / kGroups;
constexpr int kGroupWarps = kGroupThreads / 32;
constexpr uint32_t kTmemCols = 64 * kGroups;
// Layer 1's A operand (128 x 128) built and multiplied in two K halves in
// one 16 KB buffer per group: shared memory for more tiles in flight, for
// one more round trip to the tensor cores per tile.
constexpr bool kA1Split = true;
constexpr int kAChunks = kA1Split ? 8 : 16;  // 16-byte K chunks the A buffer holds

// The network as the kernel holds it in shared memory, packed once per
// model (mlp_pack) and copied whole by every CTA: FP16 K-major B operands,
// the hidden layers' weights and biases halved (exact), so that their
// accumulators hold z / 2 for the SiLU.
struct UmmaWeights {
  __half w1[64 * 128];  // chunk c at c * 1024 B, row n at n * 16 B
  __half w2[64 * 64];   // chunk c at c * 1024 B
  __half w3[16 * 64];   // rows 8..15 zero; chunk c at c * 256 B
  float b1[64], b2[64], b3[16];
  float lg1p[64];       // log(1 + c) for occupancies c < 64
};
static_assert(sizeof(UmmaWeights) % 16 == 0, "copied in 16-byte pieces");

struct __align__(16) UmmaGroup {
  __half a[128 * 8 * kAChunks];  // A1 (or its halves), then A2 and A3: chunk c at c * 2048 B, row m at m * 16 B
  __half halo[kHaloRows * kHaloW];
  unsigned long long mbar;
};

struct UmmaShared {
  UmmaWeights wt;
  UmmaGroup grp[kGroups];
  uint32_t tmem_base;
};

// Resident CTAs per SM: shared memory (1 KB of it reserved per CTA) and
// tensor-memory columns.
constexpr int kUmmaCtas = (228 * 1024) / (int(sizeof(UmmaShared)) + 1024) < int(512 / kTmemCols)
                              ? (228 * 1024) / (int(sizeof(UmmaShared)) + 1024)
                              : int(512 / kTmemCols);

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm_100 format, version 1, no swizzle).
__device__ __forceinline__ uint64_t umma_desc(const void *p, uint32_t lbo, uint32_t sbo) {
  uint64_t d = uint64_t((smem_u32(p) >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// Instruction descriptor of kind::f16: FP16 A and B, both K-major, FP32 D.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
        "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int i = 0; i < kMbarSpin; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void async_proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Barrier of warp group g (named barrier g + 1; 0 is __syncthreads), and
// the same with an AND of every thread's predicate.
// (Immediate barrier numbers: the kernel reserves three of the CTA's 16.)
template <int ID>
__device__ __forceinline__ void bar_sync_n() {
  asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(kGroupThreads) : "memory");
}
template <int ID>
__device__ __forceinline__ bool bar_and_n(bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred a, b;\n\tsetp.ne.u32 a, %1, 0;\n\t"
      "bar.red.and.pred b, %2, %3, a;\n\tselp.u32 %0, 1, 0, b;\n\t}\n"
      : "=r"(r)
      : "r"(uint32_t(p)), "n"(ID), "n"(kGroupThreads)
      : "memory");
  return r != 0u;
}
__device__ __forceinline__ void group_sync(int g) {
  static_assert(kGroups <= 2, "one named barrier per group");
  if (g == 0)
    bar_sync_n<1>();
  else
    bar_sync_n<2>();
}
__device__ __forceinline__ bool group_sync_and(int g, bool p) {
  return g == 0 ? bar_and_n<1>(p) : bar_and_n<2>(p);
}

// SiLU of two values from their halves u = z / 2 (the hidden layers' weights
// and biases are stored halved): z sigmoid(z) = u (1 + tanh(u)), with the
// hardware tanh approximation on half2.
__device__ __forceinline__ uint32_t silu_h2(float ulo, float uhi) {
  const __half2 u = __floats2half2_rn(ulo, uhi);
  uint32_t t;
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t *>(&u)));
  const __half2 y = __hfma2(u, *reinterpret_cast<const __half2 *>(&t), u);
  return *reinterpret_cast<const uint32_t *>(&y);
}

// Hidden layer epilogue: row m's 64 accumulators + bias, SiLU, as FP16 into
// the next A operand.
__device__ __forceinline__ void hidden_to_a(uint32_t taddr, const float *bias, __half *a, int m) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float v[16];
    tmem_ld16(taddr + 16 * q, v);
    tmem_wait_ld();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float *bq = bias + 16 * q + 8 * h;
      const float *vq = v + 8 * h;
      uint4 w;
      w.x = silu_h2(vq[0] + bq[0], vq[1] + bq[1]);
      w.y = silu_h2(vq[2] + bq[2], vq[3] + bq[3]);
      w.z = silu_h2(vq[4] + bq[4], vq[5] + bq[5]);
      w.w = silu_h2(vq[6] + bq[6], vq[7] + bq[7]);
      *reinterpret_cast<uint4 *>(a + (2 * q + h) * 1024 + m * 8) = w;
    }
  }
}

// A tile of the shell-proposal network: 16 cells along x (x0 .. x0 + 15)
// in each of 8 rows y0 .. y0 + 7 of one z plane of one frame. Matrix row
// m = 32 q + lane is cell (x0 + lane % 16, y0 + 2 q + lane / 16). Tiles are
// numbered frame by frame (FrameDesc::tile_base), x fastest, then y in
// steps of 8, then z. 16 x 8 pads a mesh less than 32 x 4 does along x,
// where most meshes are not a multiple of 32 (138 x 135 x 140 cells: 5 %
// padding against 17 %).
struct TileInfo {
  const FrameDesc *fr;
  int ncl, x0, y0, z0;  // ncl: cells of each row inside the frame (0 past the last tile)
};

__device__ __forceinline__ TileInfo tile_info(const FrameDesc *__restrict__ frames, int nframes,
                                              long long tile, long long tiles) {
  TileInfo g;
  g.fr = frames;
  g.ncl = 0;
  g.x0 = g.y0 = g.z0 = 0;
  if (tile >= tiles) return g;
  int f = 0;
  if (nframes > 1) {
    int lo = 0, hi = nframes - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (frames[mid].tile_base <= tile)
        lo = mid;
      else
        hi = mid - 1;
    }
    f = lo;
  }
  g.fr = &frames[f];
  const FrameDesc &fr = *g.fr;
  // a frame has fewer than 2^31 cells, so its tile numbers fit 32 bits
  const uint32_t per_x = uint32_t(fr.nx + kPropTileX - 1) / uint32_t(kPropTileX);
  const uint32_t per_y = uint32_t(fr.ny + kPropTileY - 1) / uint32_t(kPropTileY);
  const uint32_t lt = uint32_t(tile - fr.tile_base);
  const uint32_t row = lt / per_x;  // (z, y / kPropTileY)
  const uint32_t zq = row / per_y;
  g.x0 = int(lt - row * per_x) * kPropTileX;
  g.y0 = int(row - zq * per_y) * kPropTileY;
  g.z0 = int(zq);
  g.ncl = min(kPropTileX, fr.nx - g.x0);
  return g;
}

// Periodic coordinate: one add or subtract for |c - [0, n)| < n, the
// general remainder otherwise (tiny boxes).
__device__ __forceinline__ int wrap_cell(int c, int n) {
  c = c < 0 ? c + n : (c >= n ? c - n : c);
  return unsigned(c) < unsigned(n) ? c : rem_euclid(c, n);
}

// The tile's halo of log(1 + count): the 20 columns x0 - 2 .. x0 + 17 of
// the 12 x 5 rows (y0 - 2 .. y0 + 9, z0 - 2 .. z0 + 2), row (yi, zi) at halo
// row yi * 5 + zi. Warp w of the group stages the 300 cells of yi = 3 w ..
// 3 w + 2, about ten per lane, all ten loads in flight before the first store.
__device__ __forceinline__ void stage_halo(const TileInfo &g, const uint32_t *__restrict__ count,
                                           const float *lg1p, __half *halo, int w) {
  static_assert(kPropTileY + 4 == 3 * kGroupWarps, "three halo y rows per warp");
  constexpr int kPerWarp = 3 * 5 * kHaloW;  // 300 cells
  constexpr int kLoads = (kPerWarp + 31) / 32;
  const int lane = threadIdx.x & 31;
  auto feat = [&](uint32_t v) { return __float2half_rn(v < 64u ? lg1p[v] : log1pf(float(v))); };
  uint32_t c[kLoads];
#pragma unroll
  for (int i = 0; i < kLoads; ++i) {
    c[i] = 0u;
    const int t = 32 * i + lane;
    if (g.ncl > 0 && t < kPerWarp) {
      const FrameDesc &fr = *g.fr;
      const int nx = fr.nx, ny = fr.ny, nz = fr.nz;
      const int yi = 3 * w + t / (5 * kHaloW), r = t % (5 * kHaloW);
      const int zi = r / kHaloW, col = r % kHaloW;
      const int jy = wrap_cell(g.y0 + yi - 2, ny);
      const int jz = wrap_cell(g.z0 + zi - 2, nz);
      const int jx = wrap_cell(g.x0 + col - 2, nx);
      c[i] = count[fr.cell_base + ((long long)jz * ny + jy) * (long long)nx + jx];
    }
  }
  __half *h = halo + 3 * w * 5 * kHaloW;  // the warp's 15 halo rows, contiguous
#pragma unroll
  for (int i = 0; i < kLoads; ++i) {
    const int t = 32 * i + lane;
    if (t < kPerWarp) h[t] = feat(c[i]);
  }
}

// Feature chunks [c0, c1) (8 features each) of row m = the lane's cell:
// f = (dx + 2) * 25 + (dy + 2) * 5 + (dz + 2) is halo row f % 25 after the
// lane's y row, column lane % 16 + f / 25; then k / 64 and two zeros. halo
// points at the lane's y row.
template <int C0, int C1>
__device__ __forceinline__ void build_a1(const __half *halo, __half *a, int m, int lane,
                                         unsigned short kfeat) {
  const unsigned short *hs = reinterpret_cast<const unsigned short *>(halo) + (lane & 15);
#pragma unroll
  for (int c = C0; c < C1; ++c) {
    uint32_t v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int f = 8 * c + i;
      v[i] = f < 125 ? uint32_t(hs[(f % 25) * kHaloW + f / 25]) : (f == 125 ? kfeat : 0u);
    }
    uint4 w;
    w.x = v[0] | (v[1] << 16);
    w.y = v[2] | (v[3] << 16);
    w.z = v[4] | (v[5] << 16);
    w.w = v[6] | (v[7] << 16);
    *reinterpret_cast<uint4 *>(a + (c % kAChunks) * 1024 + m * 8) = w;
  }
}

// Layer L (0, 1, 2) of one tile: products of A (128 x K) and the layer's
// weights into tensor-memory columns [tcol, tcol + N), then a commit to mbar.
// Layer 0 in two halves (kA1Split): layer 3 = its second K half, whose A
// chunks sit where the first half's did. Called by one thread.
__device__ __forceinline__ void issue_layer(int layer, const UmmaShared &sh, const __half *a,
                                            uint32_t tcol, uint32_t mbar) {
  tmem_fence_after();
  if (layer == 0 || layer == 3) {
    const int s_lo = layer == 3 ? 4 : 0, s_hi = kA1Split && layer == 0 ? 4 : 8;
#pragma unroll
    for (int s2 = 0; s2 < 8; ++s2)
      if (s2 >= s_lo && s2 < s_hi)
        umma_f16(tcol, umma_desc(a + (s2 % (kAChunks / 2)) * 2 * 1024, 2048, 128),
                 umma_desc(sh.wt.w1 + s2 * 2 * 512, 1024, 128), umma_idesc(128, 64), s2 > 0);
  } else if (layer == 1) {
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2)
      umma_f16(tcol, umma_desc(a + s2 * 2 * 1024, 2048, 128),
               umma_desc(sh.wt.w2 + s2 * 2 * 512, 1024, 128), umma_idesc(128, 64), s2 > 0);
  } else {
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2)
      umma_f16(tcol, umma_desc(a + s2 * 2 * 1024, 2048, 128),
               umma_desc(sh.wt.w3 + s2 * 2 * 128, 256, 128), umma_idesc(128, 16), s2 > 0);
  }
  umma_commit(mbar);
}

// Softmax of row m's 8 logits and the proposal (smallest R with P >= tau).
__device__ __forceinline__ void write_proposal(uint32_t taddr, const float *b3, float tau,
                                               int8_t *cell_prop, long long cell, bool valid) {
  float z[16];
  tmem_ld16(taddr, z);
  tmem_wait_ld();
  if (!valid) return;
  float lg[8], mx = -3.0e38f;
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    lg[o] = z[o] + b3[o];
    mx = fmaxf(mx, lg[o]);
  }
  float e[8], sum = 0.f;
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    e[o] = __expf(lg[o] - mx);
    sum += e[o];
  }
  // the first o with P(1..o) >= tau, compared unnormalised
  const float lim = tau * sum;
  int prop = kMlpOut;
  float cum = 0.f;
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    cum += e[o];
    if (cum >= lim && prop == kMlpOut) prop = o + 1;
  }
  cell_prop[cell] = int8_t(prop >= kMlpOut ? 0 : prop);
}

// The network's shared-memory image (UmmaWeights) from its FP32 parameters.
__global__ void k_pack_weights(const float *__restrict__ params, UmmaWeights *__restrict__ out) {
  const float *W1 = params, *B1 = W1 + kMlpHidden * kMlpIn;
  const float *W2 = B1 + kMlpHidden, *B2 = W2 + kMlpHidden * kMlpHidden;
  const float *W3 = B2 + kMlpHidden, *B3 = W3 + kMlpOut * kMlpHidden;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, step = gridDim.x * blockDim.x;
  for (int t = t0; t < 64 * 128; t += step) {
    const int n = t >> 7, k = t & 127;
    out->w1[(k >> 3) * 512 + n * 8 + (k & 7)] =
        __float2half_rn(k < kMlpIn ? 0.5f * W1[n * kMlpIn + k] : 0.f);
  }
  for (int t = t0; t < 64 * 64; t += step) {
    const int n = t >> 6, k = t & 63;
    out->w2[(k >> 3) * 512 + n * 8 + (k & 7)] = __float2half_rn(0.5f * W2[n * kMlpHidden + k]);
  }
  for (int t = t0; t < 16 * 64; t += step) {
    const int n = t >> 6, k = t & 63;
    out->w3[(k >> 3) * 128 + n * 8 + (k & 7)] =
        __float2half_rn(n < kMlpOut ? W3[n * kMlpHidden + k] : 0.f);
  }
  for (int t = t0; t < 64; t += step) {
    out->b1[t] = 0.5f * B1[t];
    out->b2[t] = 0.5f * B2[t];
    out->lg1p[t] = log1pf(float(t));
    if (t < 16) out->b3[t] = t < kMlpOut ? B3[t] : 0.f;
  }
}

// kGroups groups of four warps per CTA. Warp q of a group owns lane
// quarter q of tensor memory (rows 32 q .. 32 q + 31: the tile's y rows
// 2 q and 2 q + 1): it stages three y rows of the group's halo, builds the
// features of its rows, and runs the epilogues of all 64 accumulator
// columns of its rows. The group's first thread issues its products.
__global__ void __launch_bounds__(kUmmaThreads, kUmmaCtas) k_cell_proposal_tc(
    const UmmaWeights *__restrict__ image, const FrameDesc *__restrict__ frames, int nframes,
    const uint32_t *__restrict__ count, float tau, int8_t *__restrict__ cell_prop,
    int *__restrict__ status) {
  extern __shared__ __align__(1024) unsigned char umma_smem[];
  UmmaShared &sh = *reinterpret_cast<UmmaShared *>(umma_smem);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gi = warp / kGroupWarps, quarter = warp % kGroupWarps;
  UmmaGroup &G = sh.grp[gi];
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(image);
    uint4 *dst = reinterpret_cast<uint4 *>(&sh.wt);
    for (int i = threadIdx.x; i < int(sizeof(UmmaWeights) / 16); i += kUmmaThreads) dst[i] = src[i];
  }
  const uint32_t mbar = smem_u32(&G.mbar);
  if (threadIdx.x % kGroupThreads == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sh.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  async_proxy_fence();
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tmem = sh.tmem_base + uint32_t(64 * gi);        // the group's columns
  const uint32_t tlane = tmem + (uint32_t(quarter * 32) << 16);  // this warp's lane quarter
  const int m = quarter * 32 + lane;                              // A row = accumulator lane
  // the lane's row y0 + yl reads halo rows (yl + dy + 2) 5 + dz + 2
  const int yl = 2 * quarter + (lane >> 4), xl = lane & 15;
  const __half *halo = G.halo + yl * 5 * kHaloW;
  const bool issuer = threadIdx.x % kGroupThreads == 0;
  uint32_t phase = 0;
  bool ok = true;
  auto sync_issue = [&](int layer) {
    async_proxy_fence();
    tmem_fence_before();
    group_sync(gi);
    if (issuer) issue_layer(layer, sh, G.a, tmem, mbar);
  };
  // one thread polls the mbarrier; the others wait at the group barrier
  auto wait_products = [&]() -> bool {
    bool w = true;
    if (issuer) w = mbar_wait(mbar, phase);
    phase ^= 1u;
    const bool all = group_sync_and(gi, w);
    tmem_fence_after();
    return all;
  };

  const FrameDesc &last = frames[nframes - 1];
  const long long tiles = last.tile_base + proposal_tiles(last.nx, last.ny, last.nz);
  for (long long ct = (long long)blockIdx.x * kGroups + gi; ct < tiles;
       ct += (long long)gridDim.x * kGroups) {
    const TileInfo g = tile_info(frames, nframes, ct, tiles);
    stage_halo(g, count, sh.wt.lg1p, G.halo, quarter);
    group_sync(gi);  // the halo is in place
    const unsigned short kfeat = __half_as_ushort(__float2half_rn(float(g.fr->k) / 64.0f));
    if (kA1Split) {
      build_a1<0, 8>(halo, G.a, m, lane, kfeat);
      sync_issue(0);
      if (!(ok = wait_products())) break;
      build_a1<8, 16>(halo, G.a, m, lane, kfeat);
      sync_issue(3);
    } else {
      build_a1<0, 16>(halo, G.a, m, lane, kfeat);
      sync_issue(0);
    }
    if (!(ok = wait_products())) break;
    hidden_to_a(tlane, sh.wt.b1, G.a, m);
    sync_issue(1);
    if (!(ok = wait_products())) break;
    hidden_to_a(tlane, sh.wt.b2, G.a, m);
    sync_issue(2);
    if (!(ok = wait_products())) break;
    {
      const int y = g.y0 + yl;
      const FrameDesc &tf = *g.fr;
      const bool valid = xl < g.ncl && y < tf.ny;
      const long long cell =
          tf.cell_base + ((long long)g.z0 * tf.ny + (valid ? y : 0)) * tf.nx + g.x0 + xl;
      write_proposal(tlane, sh.wt.b3, tau, cell_prop, cell, valid);
    }
    // the group's next tile rewrites its halo, A and accumulators
    tmem_fence_before();
    group_sync(gi);
    tmem_fence_after();
  }
  if (!ok && issuer) {
    atomicOr(status, kStatusMmaTimeout);
    mbar_wait(mbar, phase ^ 1u);  // give the products in flight a last bounded wait
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sh.tmem_base),
                 "r"(kTmemCols)
                 : "memory");
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

size_t mlp_image_bytes() { return sizeof(UmmaWeights); }

cudaError_t mlp_pack(const float *params, void *image, cudaStream_t s) {
  k_pack_weights<<<32, 256, 0, s>>>(params, static_cast<UmmaWeights *>(image));
  return cudaGetLastError();
}

cudaError_t mlp_propose(const void *image, const BatchBuffers &b, int8_t *cell_prop,
                        int8_t *source_prop, float tau, cudaStream_t s) {
  if (b.nframes <= 0 || b.ncells <= 0) return cudaSuccess;
  const size_t sm = sizeof(UmmaShared);  // operands without swizzle need 16-byte alignment only
  cudaError_t e =
      cudaFuncSetAttribute(k_cell_proposal_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, smem_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  // resident CTAs: shared memory (1 KB of it reserved per CTA) and the
  // kTmemCols each CTA holds of the SM's 512 tensor-memory columns
  const int per_sm = std::max(1, std::min(smem_sm / int(sm + 1024), int(512 / kTmemCols)));
  k_cell_proposal_tc<<<sms * per_sm, kUmmaThreads, sm, s>>>(
      static_cast<const UmmaWeights *>(image), b.frames, b.nframes, b.count, tau, cell_prop,
      b.status);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_source_proposal<<<grid_of(b.npts, 256), 256, 0, s>>>(b.frames, b.nframes, b.off, b.ncells,
                                                         b.scell, cell_prop, source_prop);
  return cudaGetLastError();
}

}  // namespace lc
