/*
 * linkcell oracle: TEST INFRASTRUCTURE, not product code.
 *
 * A plain C++ restatement of the reference CPU walk (HaoZeke/linkcell v0.3.3:
 * src/cell.rs, src/knearest.rs, src/capi.rs, src/error.rs) plus the two
 * independent brute-force checkers the reference tests use
 * (src/knearest.rs:24-40,508-541 and tests/agree.rs:161-210).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library. The product (linkcell_b200/liblinkcell_b200.so) never links
 * or calls it.
 *
 * Built with -O2 -ffp-contract=off so every floating-point expression rounds
 * exactly as the Rust source does (no FMA contraction, left-to-right sums).
 */
#ifndef LINKCELL_ORACLE_H
#define LINKCELL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order as the reference lc_cell (src/capi.rs:12-39). */
typedef struct orc_cell {
  double ax, ay, az, bx, by, bz, cx, cy, cz, ox, oy, oz;
} orc_cell;

/* Restates lc_knearest_many (src/capi.rs:184-259): validation order,
 * messages, -1 / NaN padding. threads = 0 uses every hardware thread,
 * 1 runs the serial walk. Returns 0 or 1 (message in orc_last_error). */
int orc_knearest_many(const double *xyz, size_t n, size_t n_frames,
                      const orc_cell *cell, size_t k, const int *mask,
                      double cell_hint, int *out_nn, double *out_d2,
                      int threads);

/* Thread-local message of the last failing orc_* call, NULL after success. */
const char *orc_last_error(void);

/* knearest_brute (src/knearest.rs:508-541): all pairs, pair_dist2 (ortho
 * MIC, else the 27 nearest images). Packed n*k rows, -1 / NaN padding. */
int orc_knearest_brute(const double *xyz, size_t n, const orc_cell *cell,
                       size_t k, const int *mask, int *out_nn,
                       double *out_d2);

/* tests/agree.rs:161-210 oracle_knearest: independent 27-image MIC. */
int orc_knearest_mic27(const double *xyz, size_t n, const orc_cell *cell,
                       size_t k, const int *mask, int *out_nn,
                       double *out_d2);

/* Cell set-up exactly as Cell::from_vectors + search() (src/cell.rs:97-124,
 * src/knearest.rs:377-397,430). info[0..2] widths, info[3] cell_min,
 * info[4] ortho flag, h[9] and hinv[9] as stored by the reference
 * (h[col*3+row]); grid[0..2] nx ny nz, grid[3] max_reach.
 * Returns 0, 1 for a bad cell, 2 for a too-fine mesh. */
int orc_cell_info(const orc_cell *cell, double cell_hint, double *info,
                  double *h, double *hinv, int *grid);

/* The fold/bin of search() (src/knearest.rs:403-413): folded coordinates
 * (n*3) and linear cell id (cz*ny+cy)*nx+cx, or -1 for masked points. */
int orc_fold_bin(const double *xyz, size_t n, const orc_cell *cell,
                 const int *mask, double cell_hint, double *folded,
                 int *cell_id);

/* Per-source walk statistics of the reference search: stop_reach[i] is
 * the reach at which source i stopped, visits[i] the number of heap pushes
 * (candidate-pair evaluations). Masked sources get 0. */
int orc_walk_stats(const double *xyz, size_t n, const orc_cell *cell,
                   size_t k, const int *mask, double cell_hint,
                   int *stop_reach, long long *visits, int threads);

/* CPU baseline timing: fold + bin + linked lists over all n points, then
 * the walk for the sources i = first, first+stride, ... (count of them),
 * on `threads` threads. Writes prep and walk wall seconds and the number
 * of sources walked. Outputs are discarded after a checksum. */
int orc_time_sample(const double *xyz, size_t n, const orc_cell *cell,
                    size_t k, const int *mask, double cell_hint,
                    size_t first, size_t stride, size_t count, int threads,
                    double *prep_seconds, double *walk_seconds,
                    long long *walked, long long *checksum);

/* Rows of the reference search for the listed sources only (fold, bin and
 * linked lists still cover all n points): row t of out_* belongs to
 * sources[t]. visits (NULL allowed) gets each listed source's heap pushes,
 * the candidate pairs the reference walk evaluates for it. Used for
 * full-size parity checks and pair counts on a sample. */
int orc_knearest_subset(const double *xyz, size_t n, const orc_cell *cell,
                        size_t k, const int *mask, double cell_hint,
                        const long long *sources, size_t count, int *out_nn,
                        double *out_d2, int threads, long long *visits);

const char *orc_version(void);

#ifdef __cplusplus
}
#endif

#endif
