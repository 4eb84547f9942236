// Cell planning: the reference's FP64 cell set-up and mesh
// (src/cell.rs:97-124,322-388 and src/knearest.rs:42-48,377-397,430) into
// a FrameDesc, plus the per-reach constants of the cube select walk.
//
// One implementation serves the host (plan_frame) and the device
// (k_plan_device_cell, the sync-free device-cell search). This file is
// compiled with -ffp-contract=off on the host and -fmad=false on the device,
// so every FP64 operation rounds once, as in the reference Rust code, on
// both sides: the host and device plans of a cell are equal bit for bit.
// The one exception is lam_min (acos / cos of the closed-form eigenvalue),
// a pruning bound with a 1e-6 margin that no result depends on.
#include <math.h>

#include <cstdlib>

#include "workspace.h"

namespace lc {

namespace {

constexpr int kPlanOk = 0, kPlanBadCell = 1, kPlanTooFine = 2;

__host__ __device__ inline bool finite_d(double x) { return x - x == 0.0; }
__host__ __device__ inline double dmax(double a, double b) { return a < b ? b : a; }
__host__ __device__ inline double dmin(double a, double b) { return b < a ? b : a; }
__host__ __device__ inline int imax(int a, int b) { return a < b ? b : a; }

// src/cell.rs:343-353
__host__ __device__ inline void cross3(const double u[3], const double v[3], double o[3]) {
  o[0] = u[1] * v[2] - u[2] * v[1];
  o[1] = u[2] * v[0] - u[0] * v[2];
  o[2] = u[0] * v[1] - u[1] * v[0];
}
__host__ __device__ inline double norm3(const double v[3]) {
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

// Smallest eigenvalue of a symmetric 3x3 matrix (closed form), used only
// for the conservative cell-pruning bound of the walk.
__host__ __device__ inline double min_eig_sym3(const double m[3][3]) {
  const double p1 = m[0][1] * m[0][1] + m[0][2] * m[0][2] + m[1][2] * m[1][2];
  const double q = (m[0][0] + m[1][1] + m[2][2]) / 3.0;
  if (p1 == 0.0) return dmin(m[0][0], dmin(m[1][1], m[2][2]));
  const double p2 = (m[0][0] - q) * (m[0][0] - q) + (m[1][1] - q) * (m[1][1] - q) +
                    (m[2][2] - q) * (m[2][2] - q) + 2.0 * p1;
  const double p = sqrt(p2 / 6.0);
  double bm[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) bm[i][j] = (m[i][j] - (i == j ? q : 0.0)) / p;
  const double detb = bm[0][0] * (bm[1][1] * bm[2][2] - bm[1][2] * bm[2][1]) -
                      bm[0][1] * (bm[1][0] * bm[2][2] - bm[1][2] * bm[2][0]) +
                      bm[0][2] * (bm[1][0] * bm[2][1] - bm[1][1] * bm[2][0]);
  double r = detb / 2.0;
  r = dmax(-1.0, dmin(1.0, r));
  const double phi = acos(r) / 3.0;
  const double e1 = q + 2.0 * p * cos(phi);
  const double e3 = q + 2.0 * p * cos(phi + 2.0943951023931953);
  const double e2 = 3.0 * q - e1 - e3;
  return dmin(e1, dmin(e2, e3));
}

// Smallest float >= v.
__host__ __device__ inline float float_up(double v) {
  float f = float(v);
  if (double(f) < v) f = nextafterf(f, INFINITY);
  return f;
}
// Largest float <= v.
__host__ __device__ inline float float_down(double v) {
  float f = float(v);
  if (double(f) > v) f = nextafterf(f, -INFINITY);
  return f;
}

// Per-reach constants of the cube select walk. The FP32 distance of a
// candidate whose cell offset is at most R per axis differs from the
// reference's FP64 value by at most band(d) = 8u d + beta(R), with
// e = u (6R + 8) ell + eps64 (R + 2) the per-component error of the FP32
// offset and beta(R) = 4 e^2 / u + 4 e^2 (the cross terms 2 |D| e are
// bounded by u D^2 + e^2 / u); 1e-6 of margin on top. rho_q is the
// fraction of B(R) the first gather covers (select_rho_q).
__host__ __device__ void fill_select(FrameDesc &fd, double rho_q) {
  const double u = 5.9604644775390625e-08;  // 2^-24
  // Row trimming: in bin units the squared distance of an offset D is
  // D^T M D with M = E^T E. For fixed (D_b, D_c) the D_a giving at most thr
  // lie within h of c = -(M_ab D_b + M_ac D_c) / M_aa, h^2 = (thr - S) / M_aa,
  // S the Schur form of (D_b, D_c), bounded below by lam_s |(D_b, D_c)|^2.
  double E[3][3];
  for (int a = 0; a < 3; ++a)
    for (int r = 0; r < 3; ++r)
      E[a][r] = fd.h[a * 3 + r] / double(a == 0 ? fd.nx : (a == 1 ? fd.ny : fd.nz));
  double M[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i][j] = E[i][0] * E[j][0] + E[i][1] * E[j][1] + E[i][2] * E[j][2];
  const double s11 = M[1][1] - M[0][1] * M[0][1] / M[0][0];
  const double s12 = M[1][2] - M[0][1] * M[0][2] / M[0][0];
  const double s22 = M[2][2] - M[0][2] * M[0][2] / M[0][0];
  const double tr = 0.5 * (s11 + s22), df = 0.5 * (s11 - s22);
  double lam_s = dmax(0.0, tr - sqrt(df * df + s12 * s12)) * 0.99;
  fd.sel_r01 = float(M[0][1] / M[0][0]);
  fd.sel_r02 = float(M[0][2] / M[0][0]);
  fd.sel_ls00 = float(lam_s / M[0][0]);
  if (!(lam_s > 1e-9 * M[0][0])) {
    // near-degenerate metric: the isotropic bound lam_min |D|^2 <= thr instead
    lam_s = double(float(fd.lam_min) * 0.99f);
    fd.sel_r01 = fd.sel_r02 = 0.f;
    fd.sel_ls00 = 1.f;
  }
  for (int R = 0; R <= 8; ++R) {
    const int Ru = R < 1 ? 1 : R;
    const double e = u * (6.0 * Ru + 8.0) * double(fd.ell) + fd.eps64 * (Ru + 2.0);
    const double beta = (4.0 * e * e / u + 4.0 * e * e) * (1.0 + 1e-6);
    const double b = double(Ru) * fd.cell_min;
    const double B = b * b;
    const double band = B * 8.0 * u + beta;
    fd.sel_beta[R] = float_up(beta);
    fd.sel_thr[R] = float_up(B * (1.0 + 8.0 * u) + beta);
    fd.sel_bhi[R] = float_up(B + 2.0 * band);
    fd.sel_qlim[R] = lam_s > 0.0 ? float_up(double(fd.sel_thr[R]) / lam_s * 1.0001) : 3.0e38f;
    fd.sel_epsr[R] = float_up(band / (2.0 * fd.cell_min * fd.cell_min) + 16.0 * u * (Ru + 2.0));
    const double bm = double(Ru - 1) * fd.cell_min;
    const double rho2 = dmax(bm * bm * (1.0 + 1e-4), rho_q * B);
    const double rband = rho2 * 8.0 * u + beta;
    fd.sel_rho2[R] = rho2;
    fd.sel_rho_thr[R] = float_up(rho2 * (1.0 + 8.0 * u) + beta);
    fd.sel_rho_qlim[R] =
        lam_s > 0.0 ? float_up(double(fd.sel_rho_thr[R]) / lam_s * 1.0001) : 3.0e38f;
    fd.sel_rho_lo[R] = float_down(rho2 - rband);
    fd.sel_rho_hi[R] = float_up(rho2 + rband);
    fd.sel_rho_bhi[R] = float_up(rho2 + 2.0 * rband);
  }
  fd.inv_nx = 1.0 / double(fd.nx);
  fd.inv_nxy = 1.0 / (double(fd.nx) * double(fd.ny));
}

// Cell::from_vectors and the search mesh into fd (zeroed first). rows =
// a, b, c (9 doubles), origin 3 doubles; hint <= 0 or NaN selects the
// default edge 3.0. Returns kPlanOk, kPlanBadCell or kPlanTooFine.
__host__ __device__ int plan_cell(const double *rows, const double *origin, double cell_hint,
                                  int k, double rho_q, FrameDesc &fd) {
  {
    char *p = reinterpret_cast<char *>(&fd);
    for (unsigned i = 0; i < sizeof(FrameDesc); ++i) p[i] = 0;
  }
  const double a[3] = {rows[0], rows[1], rows[2]};
  const double b[3] = {rows[3], rows[4], rows[5]};
  const double c[3] = {rows[6], rows[7], rows[8]};
  // H by columns (src/cell.rs:103)
  for (int r = 0; r < 3; ++r) {
    fd.h[0 * 3 + r] = a[r];
    fd.h[1 * 3 + r] = b[r];
    fd.h[2 * 3 + r] = c[r];
  }
  // invert_columns (src/cell.rs:355-388)
  const double det = a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
                     a[2] * (b[0] * c[1] - b[1] * c[0]);
  if (!finite_d(det) || fabs(det) < 1e-18) return kPlanBadCell;
  const double invdet = 1.0 / det;
  fd.hinv[0] = (b[1] * c[2] - b[2] * c[1]) * invdet;
  fd.hinv[1] = (a[2] * c[1] - a[1] * c[2]) * invdet;
  fd.hinv[2] = (a[1] * b[2] - a[2] * b[1]) * invdet;
  fd.hinv[3] = (b[2] * c[0] - b[0] * c[2]) * invdet;
  fd.hinv[4] = (a[0] * c[2] - a[2] * c[0]) * invdet;
  fd.hinv[5] = (a[2] * b[0] - a[0] * b[2]) * invdet;
  fd.hinv[6] = (b[0] * c[1] - b[1] * c[0]) * invdet;
  fd.hinv[7] = (a[1] * c[0] - a[0] * c[1]) * invdet;
  fd.hinv[8] = (a[0] * b[1] - a[1] * b[0]) * invdet;
  // perpendicular widths (src/cell.rs:108-116)
  double bc[3], ca[3], ab[3];
  cross3(b, c, bc);
  cross3(c, a, ca);
  cross3(a, b, ab);
  const double wa = fabs(det) / norm3(bc);
  const double wb = fabs(det) / norm3(ca);
  const double wc = fabs(det) / norm3(ab);
  if (!(wa > 0.0 && wb > 0.0 && wc > 0.0)) return kPlanBadCell;
  fd.widths[0] = wa;
  fd.widths[1] = wb;
  fd.widths[2] = wc;
  fd.origin[0] = origin[0];
  fd.origin[1] = origin[1];
  fd.origin[2] = origin[2];
  // is_axis_aligned (src/cell.rs:322-331)
  {
    const double scale = fmax(norm3(a) + norm3(b) + norm3(c), 1.0);
    const double tol = 1e-12 * scale;
    fd.ortho = fabs(a[1]) <= tol && fabs(a[2]) <= tol && fabs(b[0]) <= tol && fabs(b[2]) <= tol &&
               fabs(c[0]) <= tol && fabs(c[1]) <= tol;
  }
  // edge and bins (src/knearest.rs:42-48,377-397). The C ABI passes
  // Some(hint) only for hint > 0 (src/capi.rs:235-239).
  double edge = cell_hint > 0.0 ? cell_hint : 3.0;
  if (!finite_d(edge) || edge <= 0.0) edge = 3.0;
  edge = fmin(fmin(fmin(edge, wa), wb), wc);
  int nb[3];
  const double w[3] = {wa, wb, wc};
  for (int d = 0; d < 3; ++d) {
    const double nn = fmax(floor(w[d] / edge), 1.0);
    if (!finite_d(nn) || nn > 1000000.0) return kPlanTooFine;
    nb[d] = int(nn);
  }
  const long long ncell = (long long)nb[0] * nb[1] * nb[2];
  if (!(ncell > 0 && ncell <= kMaxCellsPerFrame)) return kPlanTooFine;
  fd.nx = nb[0];
  fd.ny = nb[1];
  fd.nz = nb[2];
  fd.cell_min = fmin(fmin(wa / double(nb[0]), wb / double(nb[1])), wc / double(nb[2]));
  fd.max_reach = imax(nb[0], imax(nb[1], nb[2])) / 2 + 1;
  fd.k = k;
  // FP32 cell edge vectors and the bin-unit metric (pruning only)
  double ev[3][3];
  for (int ax = 0; ax < 3; ++ax)
    for (int r = 0; r < 3; ++r) {
      ev[ax][r] = fd.h[ax * 3 + r] / double(nb[ax]);
      fd.ev[ax * 3 + r] = float(ev[ax][r]);
    }
  double g[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      g[i][j] = ev[i][0] * ev[j][0] + ev[i][1] * ev[j][1] + ev[i][2] * ev[j][2];
  fd.lam_min = dmax(0.0, min_eig_sym3(g)) * (1.0 - 1e-6);
  // (H / n)^-1 = diag(n) Hinv: row a of Hinv times n_a
  for (int ax = 0; ax < 3; ++ax)
    for (int r = 0; r < 3; ++r) fd.nhinv[ax * 3 + r] = float(double(nb[ax]) * fd.hinv[r * 3 + ax]);
  double ell = 0.0;
  for (int r = 0; r < 3; ++r)
    ell = dmax(ell, fabs(ev[0][r]) + fabs(ev[1][r]) + fabs(ev[2][r]));
  fd.ell = float(ell * (1.0 + 1e-6));
  double mag = fabs(origin[0]) + fabs(origin[1]) + fabs(origin[2]);
  for (int t = 0; t < 9; ++t) mag += fabs(fd.h[t]);
  // generous: 2^-36 of the largest coordinate / shift magnitude per unit wrap
  fd.eps64 = ldexp(mag, -36);
  fill_select(fd, rho_q);
  for (int t = 0; t < 27; ++t)
    lattice_shift(fd, t / 9 - 1, (t / 3) % 3 - 1, t % 3 - 1, fd.shift27[t][0], fd.shift27[t][1],
                  fd.shift27[t][2]);
  return kPlanOk;
}

// The device cell of lc_gpu_knearest_many_dcell (3 orthorhombic lengths,
// 9 lattice rows, or 12: rows then origin) as rows and origin.
__host__ __device__ inline void device_cell_rows(const double *cell, int cell_n, double rows[9],
                                                 double origin[3]) {
  for (int t = 0; t < 9; ++t) rows[t] = 0.0;
  origin[0] = origin[1] = origin[2] = 0.0;
  if (cell_n == 3) {
    rows[0] = cell[0];
    rows[4] = cell[1];
    rows[8] = cell[2];
  } else {
    for (int t = 0; t < 9; ++t) rows[t] = cell[t];
    if (cell_n == 12) {
      origin[0] = cell[9];
      origin[1] = cell[10];
      origin[2] = cell[11];
    }
  }
}

// Plans the shared cell of a device-cell batch on the device and writes the
// frame table: nframes frames of n points each, frame-major. A cell the
// planner rejects leaves a status bit (kStatusPlanBadCell /
// kStatusPlanTooFine) and a table of dead one-cell frames, whose points the
// fold marks inactive (rows -1 / NaN). As in the host path, a too fine mesh
// under an all-zero mask is no error (src/knearest.rs:370-375). One block.
__global__ void __launch_bounds__(256)
    k_plan_device_cell(const double *__restrict__ cell, int cell_n, long long n, int nframes,
                       int k, double hint, double rho_q, const int *__restrict__ mask,
                       FrameDesc *__restrict__ frames, long long *__restrict__ live_cells,
                       int *__restrict__ status) {
  __shared__ FrameDesc s_fd;
  __shared__ int s_code, s_any;
  if (threadIdx.x == 0) {
    double rows[9], origin[3];
    device_cell_rows(cell, cell_n, rows, origin);
    FrameDesc fd;
    int code = plan_cell(rows, origin, hint, k, rho_q, fd);
    if (code != kPlanOk) {
      // a valid one-cell plan with every point inactive
      const double unit[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, zero[3] = {0, 0, 0};
      plan_cell(unit, zero, 2.0, k, rho_q, fd);
      fd.dead = 1;
    }
    fd.n = n;
    fd.has_mask = mask ? 1 : 0;
    fd.mask_base = 0;
    s_fd = fd;
    s_code = code;
    s_any = 0;
  }
  __syncthreads();
  if (s_code == kPlanTooFine && mask) {
    int any = 0;
    for (long long i = threadIdx.x; i < n && !any; i += blockDim.x) any = mask[i] != 0;
    if (__syncthreads_or(any) && threadIdx.x == 0) s_any = 1;
  }
  __syncthreads();
  const long long ncell = (long long)s_fd.nx * s_fd.ny * s_fd.nz;
  const long long tiles = proposal_tiles(s_fd.nx, s_fd.ny, s_fd.nz);
  for (int f = threadIdx.x; f < nframes; f += blockDim.x) {
    FrameDesc fd = s_fd;
    fd.pt_base = (long long)f * n;
    fd.cell_base = (long long)f * ncell;
    fd.tile_base = (long long)f * tiles;
    fd.out_base = (long long)f * n * k;
    frames[f] = fd;
  }
  if (threadIdx.x == 0) {
    *live_cells = (long long)nframes * ncell;
    if (s_code == kPlanBadCell) atomicOr(status, kStatusPlanBadCell);
    if (s_code == kPlanTooFine && (!mask || s_any)) atomicOr(status, kStatusPlanTooFine);
  }
}

Code code_of(int plan) {
  return plan == kPlanOk ? Code::Ok : (plan == kPlanBadCell ? Code::BadCell : Code::TooFine);
}

}  // namespace

// Fraction q of B(R_p) the select walk's first gather covers. The k-th
// distance squared grows like k^(2/3) at a given density, so q follows it
// from q0 at k = 32 (LINKCELL_SELECT_Q sets q0, 0 < q0 <= 1); q = 1 gathers
// the whole proposed ball at once.
double select_rho_q(int k) {
  static const double q0 = [] {
    const char *e = std::getenv("LINKCELL_SELECT_Q");
    const double v = e ? std::atof(e) : 0.65;
    return (v > 0.0 && v <= 1.0) ? v : 0.65;
  }();
  return fmin(1.0, q0 * cbrt(double(k) * double(k) / 1024.0));
}

Code plan_frame(const double *rows, const double *origin, double cell_hint, int k, FrameDesc &fd) {
  return code_of(plan_cell(rows, origin, cell_hint, k, select_rho_q(k), fd));
}

cudaError_t launch_plan_device_cell(const double *cell, int cell_n, long long n, int nframes, int k,
                                    double hint, const int *mask, FrameDesc *frames,
                                    long long *live_cells, int *status, cudaStream_t s) {
  k_plan_device_cell<<<1, 256, 0, s>>>(cell, cell_n, n, nframes, k, hint, select_rho_q(k), mask,
                                       frames, live_cells, status);
  return cudaGetLastError();
}

}  // namespace lc
