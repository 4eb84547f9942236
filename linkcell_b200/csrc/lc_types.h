// Shared host/device types and the exact FP64 cell arithmetic of the
// periodic linked-cell search.
//
// Every FP64 expression here rounds exactly as the reference Rust code
// (HaoZeke/linkcell v0.3.3, src/cell.rs): one IEEE operation at a time, in
// the Rust association, never fused. Device code uses the __d*_rn
// intrinsics, which nvcc never contracts into an FMA; host code is built
// with -ffp-contract=off.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define LC_HD __host__ __device__ __forceinline__
#else
#define LC_HD inline
#endif

namespace lc {

// Most cells of one frame's mesh (MAX_CELLS, src/knearest.rs:20,386-397).
constexpr long long kMaxCellsPerFrame = 16777216LL;

// Marks a masked point in the cell-of array.
constexpr uint32_t kInactive = 0xFFFFFFFFu;

// Status bits a launch leaves in the device status word.
enum StatusBits : int {
  kStatusScanTimeout = 1,    // decoupled look-back wait ran out of iterations
  kStatusBadIndex = 2,       // a kernel saw an offset outside its buffers
  kStatusReplayOverflow = 4, // replay queue longer than its buffer
  kStatusMmaTimeout = 8,     // a tensor-core product did not complete in bounded time
  kStatusPlanBadCell = 16,   // the device-cell planner rejected the cell (singular)
  kStatusPlanTooFine = 32,   // the device-cell planner's mesh exceeds the bin caps
};

// Per-frame flags (frame_flags[f]).
enum FrameFlags : int {
  kFrameNaN = 1,  // a folded coordinate is NaN: every source takes the exact replay
};

// One frame of a search: the reference Cell (src/cell.rs:36-46) plus the
// linked-cell mesh of search() (src/knearest.rs:377-397,430) and where the
// frame's points, cells and output rows sit in the batch.
struct FrameDesc {
  double h[9];       // lattice vectors as columns: h[col*3 + row]
  double hinv[9];    // inverse, same storage (src/cell.rs:355-388)
  double origin[3];
  double widths[3];  // perpendicular widths |det| / |b x c| ...
  double cell_min;   // min(w_a / n_a)
  double lam_min;    // smallest eigenvalue of the bin-unit metric (pruning)
  double eps64;      // bound on the FP64 rounding of the reference distance terms
  float ev[9];       // FP32 cell edge vectors: ev[axis*3 + comp] = h[axis][comp] / n_axis
  float nhinv[9];    // FP32 (H / n)^-1 rows: bin-unit coordinates of a Cartesian offset
  float ell;         // max over components of sum over axes |ev[axis][comp]|
  int nx, ny, nz;
  int ortho;         // Cell::is_ortho (src/cell.rs:322-331)
  int max_reach;     // max(nx, ny, nz) / 2 + 1
  int k;             // neighbours per source
  int has_mask;
  int mode;          // per-frame walk mode (batched launches)
  int dead;          // the planner rejected the frame's cell: every point inactive
  long long n;          // points in the frame
  long long pt_base;    // first point of the frame in the batch
  long long cell_base;  // first cell of the frame in the batch
  long long out_base;   // first output element (row 0, slot 0)
  long long mask_base;  // offset of the frame's mask (shared masks repeat 0)
  long long tile_base;  // first 16 x 8-cell tile of the frame (shell proposals)
  // Cube select walk, per reach R = 1..8 (index R): the FP32 filter at
  // B(R) = (R cell_min)^2, the row-trimming limit thr / (0.99 lam_min), the
  // FP32 error offset beta (rounded up), B(R) + 2 band(B(R)) rounded up,
  // and the error band of sqrt(d32) / cell_min near an integer.
  float sel_thr[9];
  float sel_qlim[9];       // thr / lam_s, lam_s = 0.99 x the smallest eigenvalue of the (b, c) Schur form
  float sel_r01, sel_r02;  // M_ab / M_aa, M_ac / M_aa of the bin-unit metric M = E^T E
  float sel_ls00;          // lam_s / M_aa
  float sel_beta[9];
  float sel_bhi[9];
  float sel_epsr[9];
  // Partial gather at proposal R: rho2 = max(B(R-1), q B(R)) (exact FP64),
  // the FP32 filter and row-trimming limit at rho2, the FP32 values below /
  // above which the exact distance is surely <= / > rho2, and rho2 + 2 band
  // rounded up (histogram range).
  double sel_rho2[9];
  float sel_rho_thr[9], sel_rho_qlim[9], sel_rho_lo[9], sel_rho_hi[9], sel_rho_bhi[9];
  double inv_nx, inv_nxy;  // 1 / nx, 1 / (nx ny) for exact quotient estimates
  // Cell::lattice_shift of the 27 wrap triples (na, nb, nc) in {-1, 0, 1}^3
  // at index (na + 1) 9 + (nb + 1) 3 + (nc + 1), in the reference expression
  double shift27[27][3];
};

// Shell-proposal tiles: kPropTileX x kPropTileY cells of one z plane of one
// frame, numbered x fastest, then y, then z (the network's M = 128 rows).
constexpr int kPropTileX = 16, kPropTileY = 8;
LC_HD long long proposal_tiles(int nx, int ny, int nz) {
  return (long long)((nx + kPropTileX - 1) / kPropTileX) * ((ny + kPropTileY - 1) / kPropTileY) *
         nz;
}

// ------------------------------------------------------------ exact FP64
LC_HD double xadd(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
LC_HD double xsub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
LC_HD double xmul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
LC_HD double xdiv(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}

// mul(h, v) = H v with H stored by columns (src/cell.rs:333-341):
// row r = h[0][r] v0 + h[1][r] v1 + h[2][r] v2, summed left to right.
LC_HD void mat_vec(const double *m, double v0, double v1, double v2, double &o0, double &o1,
                   double &o2) {
  o0 = xadd(xadd(xmul(m[0], v0), xmul(m[3], v1)), xmul(m[6], v2));
  o1 = xadd(xadd(xmul(m[1], v0), xmul(m[4], v1)), xmul(m[7], v2));
  o2 = xadd(xadd(xmul(m[2], v0), xmul(m[5], v1)), xmul(m[8], v2));
}

LC_HD double floor_d(double s) {
#ifdef __CUDA_ARCH__
  return floor(s);
#else
  return __builtin_floor(s);
#endif
}

// wrap01 (src/cell.rs:290-298).
LC_HD double wrap01(double s) {
  s = xsub(s, floor_d(s));
  return s >= 1.0 ? 0.0 : s;
}

// Cell::fractional (src/cell.rs:175-194): ortho divides by the widths,
// otherwise Hinv (r - origin); then wrap01.
LC_HD void fractional(const FrameDesc &f, double r0, double r1, double r2, double &s0, double &s1,
                      double &s2) {
  const double d0 = xsub(r0, f.origin[0]);
  const double d1 = xsub(r1, f.origin[1]);
  const double d2 = xsub(r2, f.origin[2]);
  if (f.ortho) {
    s0 = wrap01(xdiv(d0, f.widths[0]));
    s1 = wrap01(xdiv(d1, f.widths[1]));
    s2 = wrap01(xdiv(d2, f.widths[2]));
    return;
  }
  mat_vec(f.hinv, d0, d1, d2, s0, s1, s2);
  s0 = wrap01(s0);
  s1 = wrap01(s1);
  s2 = wrap01(s2);
}

// Cell::cartesian (src/cell.rs:199-207): H s + origin (always H, also for
// orthorhombic cells).
LC_HD void cartesian(const FrameDesc &f, double s0, double s1, double s2, double &r0, double &r1,
                     double &r2) {
  double t0, t1, t2;
  mat_vec(f.h, s0, s1, s2, t0, t1, t2);
  r0 = xadd(t0, f.origin[0]);
  r1 = xadd(t1, f.origin[1]);
  r2 = xadd(t2, f.origin[2]);
}

// The bin of one fractional coordinate (src/knearest.rs:408-412):
// ((s * n) as i32).clamp(0, n - 1). Rust maps NaN to 0; s lies in [0, 1).
LC_HD int bin_of(double s, int n) {
  const double v = xmul(s, double(n));
  int b = (v == v) ? int(v) : 0;
  b = b < 0 ? 0 : b;
  return b > n - 1 ? n - 1 : b;
}

// Cell::lattice_shift (src/cell.rs:226-247).
LC_HD void lattice_shift(const FrameDesc &f, int na, int nb, int nc, double &x, double &y,
                         double &z) {
  const double fa = double(na), fb = double(nb), fc = double(nc);
  if (f.ortho) {
    x = xmul(fa, f.widths[0]);
    y = xmul(fb, f.widths[1]);
    z = xmul(fc, f.widths[2]);
    return;
  }
  x = xadd(xadd(xmul(fa, f.h[0]), xmul(fb, f.h[3])), xmul(fc, f.h[6]));
  y = xadd(xadd(xmul(fa, f.h[1]), xmul(fb, f.h[4])), xmul(fc, f.h[7]));
  z = xadd(xadd(xmul(fa, f.h[2]), xmul(fb, f.h[5])), xmul(fc, f.h[8]));
}

// Cell::dist2_shifted (src/cell.rs:268-274): dx = q + shift - p.
LC_HD double dist2_shifted(double px, double py, double pz, double qx, double qy, double qz,
                           double sx, double sy, double sz) {
  const double dx = xsub(xadd(qx, sx), px);
  const double dy = xsub(xadd(qy, sy), py);
  const double dz = xsub(xadd(qz, sz), pz);
  return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
}

// i32::rem_euclid / div_euclid for n > 0.
LC_HD int rem_euclid(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}
LC_HD int div_euclid(int a, int n) {
  const int q = a / n;
  return (a % n < 0) ? q - 1 : q;
}

// The stop bound (reach * cell_min)^2 (src/knearest.rs:466-471).
LC_HD double stop_bound(int reach, double cell_min) {
  const double b = xmul(double(reach), cell_min);
  return xmul(b, b);
}

// f64::total_cmp order key (IEEE totalOrder) for the final row sort.
LC_HD long long total_key(double v) {
#ifdef __CUDA_ARCH__
  long long b = __double_as_longlong(v);
#else
  long long b;
  __builtin_memcpy(&b, &v, 8);
#endif
  b ^= (long long)((unsigned long long)(b >> 63) >> 1);
  return b;
}

}  // namespace lc
