/*
 * linkcell C API, served by the B200 implementation (liblinkcell_b200.so).
 *
 * Drop-in for the reference CPU C ABI (HaoZeke/linkcell v0.3.3,
 * include/linkcell.h, generated from src/capi.rs). Same symbols, argument
 * meaning, validation order, error strings and packed n*k output layout.
 * Pointers are HOST pointers, as in the reference; the search itself runs
 * on the GPU (inputs are copied in, results copied back). There is no CPU
 * fallback: without a CUDA device a call fails with "no CUDA device
 * available" after the argument checks.
 *
 * Memory ownership
 *   - lc_knearest writes into caller-owned out_nn (length n * k).
 *   - lc_knearest_d2 also writes out_d2 (length n * k, unused slots NaN).
 *   - lc_knearest_many is the frame-major batch (n_frames * n * k).
 *   - lc_last_error returns a thread-local pointer. Do not free it. It is
 *     invalid after the next lc_knearest* call on the same thread.
 *     lc_version neither reads nor writes the slot.
 *   - lc_version returns a process-static string. Do not free it.
 *
 * Thread safety
 *   - Distinct threads may search concurrently; each thread uses its own
 *     device workspace and its own last-error slot.
 */
#ifndef LINKCELL_H
#define LINKCELL_H

#include <stddef.h>
#include <stdint.h>

/* Periodic parallelepiped: lattice vectors a, b, c (rows, as in vesin) and
 * the origin of the dump cell. Replaces struct lc_cell of the reference
 * (src/capi.rs:12-39, include/linkcell.h:40-89); same field order. */
typedef struct lc_cell {
  double ax, ay, az;
  double bx, by, bz;
  double cx, cy, cz;
  double ox, oy, oz;
} lc_cell;

#ifdef __cplusplus
extern "C" {
#endif

/* k nearest neighbours of n points (reference: src/capi.rs:123-148,
 * include/linkcell.h:126-132).
 * xyz: n packed (x, y, z) triples. simbox: the periodic cell. k >= 1.
 * mask: NULL, or n ints; nonzero keeps a point as source and candidate.
 * cell_hint: target cell edge; values <= 0 (and NaN) select 3.0.
 * out_nn: n * k ints; row i holds source i's neighbours, nearest first
 * (ties by index), unused slots -1.
 * Returns 0, or 1 with the message in lc_last_error(). Messages, in check
 * order: "no points", "k must be at least 1", "null pointer",
 * "n * k overflows", "singular or non-positive cell",
 * "linked-cell mesh is too fine". */
int lc_knearest(const double *xyz, size_t n, const struct lc_cell *simbox, size_t k,
                const int *mask, double cell_hint, int *out_nn);

/* Like lc_knearest, plus squared distances in out_d2 (n * k doubles, NaN
 * in unused slots; NULL skips them). Reference: src/capi.rs:159-171,
 * include/linkcell.h:145-152. */
int lc_knearest_d2(const double *xyz, size_t n, const struct lc_cell *simbox, size_t k,
                   const int *mask, double cell_hint, int *out_nn, double *out_d2);

/* Frame-major batch of n_frames frames of n points that share one cell and
 * one length-n mask; outputs are n_frames * n * k. Reference:
 * src/capi.rs:183-259, include/linkcell.h:166-174. */
int lc_knearest_many(const double *xyz, size_t n, size_t n_frames, const struct lc_cell *simbox,
                     size_t k, const int *mask, double cell_hint, int *out_nn, double *out_d2);

/* Message of this thread's last failing lc_knearest* call, or NULL after a
 * success (reference: src/capi.rs:70-86). */
const char *lc_last_error(void);

/* "0.3.3": the reference version this library is a drop-in for
 * (src/capi.rs:88-92). */
const char *lc_version(void);

#ifdef __cplusplus
}
#endif

/* Orthorhombic cell with origin at zero (reference include/linkcell.h:206-224). */
static inline lc_cell lc_cell_ortho(double lx, double ly, double lz) {
  lc_cell c;
  c.ax = lx;  c.ay = 0.0; c.az = 0.0;
  c.bx = 0.0; c.by = ly;  c.bz = 0.0;
  c.cx = 0.0; c.cy = 0.0; c.cz = lz;
  c.ox = 0.0; c.oy = 0.0; c.oz = 0.0;
  return c;
}

#endif /* LINKCELL_H */
