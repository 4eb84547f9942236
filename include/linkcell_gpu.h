/*
 * linkcell device C API, served by the B200 implementation
 * (liblinkcell_b200.so, sm_100a kernels built ahead of time with nvcc).
 *
 * Drop-in for the reference device C ABI (HaoZeke/linkcell v0.3.3,
 * include/linkcell_gpu.h, src/gpu/capi.cpp): same 13 symbols, same
 * arguments. xyz, mask, out_nn and out_d2 are CUDA device pointers; the
 * cell is a host lc_cell (or, for _dcell, device doubles).
 *
 * Differences from the reference gpulite path, all toward the reference CPU
 * walk (src/knearest.rs), whose results this library reproduces exactly:
 *   - any k >= 1 (the reference device path stops at k <= 16);
 *   - meshes up to 16,777,216 cells (the reference device path stops at
 *     262,144);
 *   - exact duplicates (dist2 == 0) are kept, as on the CPU;
 *   - a mask has n entries shared by all frames, as on the CPU;
 *   - cell_hint = +inf selects the default edge 3.0, as on the CPU;
 *   - tie order follows the CPU heap exactly.
 *
 * Distinct workspaces may run concurrently. A workspace enqueues all work
 * on one CUDA stream (lc_gpu_queue); call lc_gpu_wait before reading
 * results of a search issued with wait == 0.
 */
#ifndef LINKCELL_GPU_H
#define LINKCELL_GPU_H

#include <stddef.h>

#include "linkcell.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lc_gpu_workspace lc_gpu_workspace;

/* 1 when a CUDA device is usable, else 0 (src/gpu/capi.cpp:21-27). */
int lc_gpu_available(void);
/* This thread's last lc_gpu_* error, NULL after success (src/gpu/capi.cpp:29-31). */
const char *lc_gpu_last_error(void);

/* Workspace: grow-only device buffers and one CUDA stream
 * (src/gpu/capi.cpp:39-57). */
lc_gpu_workspace *lc_gpu_workspace_new(void);
void lc_gpu_workspace_free(lc_gpu_workspace *ws);

/* One frame, waits for completion (src/gpu/capi.cpp:65-70). */
int lc_gpu_knearest(lc_gpu_workspace *ws, const double *xyz, size_t n,
                    const struct lc_cell *simbox, size_t k, const int *mask, double cell_hint,
                    int *out_nn, double *out_d2);

/* n_frames frames sharing one cell; wait == 0 returns after enqueueing
 * (src/gpu/capi.cpp:72-108). */
int lc_gpu_knearest_many(lc_gpu_workspace *ws, const double *xyz, size_t n, size_t n_frames,
                         const struct lc_cell *simbox, size_t k, const int *mask,
                         double cell_hint, int *out_nn, double *out_d2, int wait);

/* Cell given as device doubles: 3 (ortho lengths), 9 (rows a, b, c) or 12
 * (rows plus origin) (src/gpu/capi.cpp:110-148). Up to 16 frames the cell
 * is planned on the device, without the reference's blocking read of the
 * mesh (src/gpu/knearest.cpp:860-864): the call never synchronizes when
 * wait == 0, and a workspace with graphs on replays it with whatever cell
 * the pointer holds at launch. A cell rejected there ("bad cell", "too many
 * cells") is reported when the batch is waited for (wait != 0, or
 * lc_gpu_wait through lc_gpu_last_error). More frames read the cell first. */
int lc_gpu_knearest_many_dcell(lc_gpu_workspace *ws, const double *xyz, size_t n,
                               size_t n_frames, const double *cell, int cell_n, size_t k,
                               const int *mask, double cell_hint, int *out_nn, double *out_d2,
                               int wait);

/* The workspace's cudaStream_t (src/gpu/capi.cpp:150-157). */
void *lc_gpu_queue(lc_gpu_workspace *ws);
/* Stream barrier (src/gpu/capi.cpp:159-167). Errors a kernel of the
 * batch reported are left in lc_gpu_last_error. */
void lc_gpu_wait(lc_gpu_workspace *ws);

/* Helpers used by language bindings (src/gpu/capi.cpp:169-282). kind is a
 * cudaMemcpyKind; fill supports the values 0 and -1 only. */
int lc_gpu_alloc(void **ptr, size_t bytes);
void lc_gpu_free(void *ptr);
int lc_gpu_fill_i32(void *ptr, int value, size_t n);
int lc_gpu_memcpy(void *dst, const void *src, size_t bytes, int kind);

/* ------------------------------------------------------------------
 * Extensions (no counterpart in the reference). Defaults keep the
 * reference's exact results; every mode returns identical indices.
 */

/* Walk selection. Every mode gives the same rows; the default is
 * LC_GPU_MODE_LEARNED (LINKCELL_MODE overrides it for new workspaces). */
#define LC_GPU_MODE_PLAIN_F64 0 /* shell-by-shell FP64 walk */
#define LC_GPU_MODE_FAST_F32 1  /* FP32 candidates, FP64 rerank of the boundary band */
#define LC_GPU_MODE_LEARNED 2   /* FP32 walk that opens a learned shell proposal at once */
#define LC_GPU_MODE_REPLAY 3    /* every source through the literal sequential heap */
int lc_gpu_set_mode(lc_gpu_workspace *ws, int mode);
int lc_gpu_get_mode(lc_gpu_workspace *ws);

/* Learned walk: propose this shell for every source instead of the
 * network's proposal (0 restores the network). Results stay exact for any
 * proposal; only the work changes. */
int lc_gpu_set_proposal(lc_gpu_workspace *ws, int shell);

/* Learned walk: the shell-proposal network. params holds lc_gpu_mlp_params()
 * host floats in the layout W1[64][126] b1[64] W2[64][64] b2[64] W3[8][64]
 * b3[8] (inputs: log(1 + occupancy) of the 5x5x5 cells around the source's
 * cell, then k / 64; outputs: logits of the settled shell 1..7 and "8 or
 * more"). A cell's proposal is the smallest shell whose cumulative
 * probability reaches tau. */
int lc_gpu_set_model(lc_gpu_workspace *ws, const float *params, size_t n_params, float tau);

/* Training data. With logging on, a search records the settled shell of
 * every source; lc_gpu_training_rows then writes, for the sorted sources
 * first, first + stride, ..., up to cap rows of 126 features into device
 * X and the class (settled shell - 1, capped at 7) into device y. Returns
 * the number of rows, or a negative value on error. */
int lc_gpu_log_shells(lc_gpu_workspace *ws, int on);
/* Proposed shells (0: none) the last learned search used for the sorted
 * sources first, first + stride, ..., into host out (up to cap); returns
 * the count, or a negative value on error. Rows line up with
 * lc_gpu_training_rows of the same search. */
long long lc_gpu_proposals(lc_gpu_workspace *ws, signed char *out, long long cap, long long stride,
                           long long first);
long long lc_gpu_training_rows(lc_gpu_workspace *ws, float *X, int *y, long long cap,
                               long long stride, long long first);

/* The network's kernels on device buffers, for training: forward
 * (softmax probabilities, batch x 8), gradient of the mean cross-entropy
 * (and the loss), and one Adam step (step counts from 1). scratch holds
 * lc_gpu_mlp_scratch_floats(batch) floats. */
int lc_gpu_mlp_params(void);
size_t lc_gpu_mlp_scratch_floats(int batch);
int lc_gpu_mlp_forward(const float *params, const float *X, int batch, float *probs,
                       float *scratch, void *stream);
int lc_gpu_mlp_grad(const float *params, const float *X, const int *y, int batch, float *grad,
                    float *loss, float *scratch, void *stream);
int lc_gpu_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr,
                    void *stream);

/* Threads per source of the walk: 32 (a warp per source) or 1 (a thread
 * per source, its heap in shared memory); 0 restores the autotuner, which
 * times both designs on the first batch of each kind (walk mode, k class,
 * single or many frames) and keeps the faster. The environment variables
 * LINKCELL_TPP and LINKCELL_BLOCK override the autotuner for new
 * workspaces. lc_gpu_get_tpp reports the design of the last batch. */
int lc_gpu_set_tpp(lc_gpu_workspace *ws, int tpp);
int lc_gpu_get_tpp(lc_gpu_workspace *ws);

/* Extension: the learned mode's cube select walk in a fixed block shape:
 * warps per block (8 or 4 for k <= 32, 4 or 2 for k <= 64) and sources per
 * work-queue grab (8, 16 or 32). 0, 0 hands both back to the autotuner,
 * which times every such shape (and the thread-per-source walk) once on the
 * first batch of each kind; LINKCELL_GRAB overrides the grab like
 * LINKCELL_BLOCK the block. Results are the same in every shape. */
int lc_gpu_set_walk_shape(lc_gpu_workspace *ws, int warps, int grab);

/* Extension: the walk of the last search: shape3 = threads per source,
 * warps per block, sources per grab (0 where they do not apply). trials
 * (NULL allowed) gets up to max_trials triples of the candidates the last
 * autotuning timed. Returns the number of candidates it timed (0: none). */
int lc_gpu_walk_shape(lc_gpu_workspace *ws, int *shape3, int *trials, int max_trials);

/* CUDA graphs: with on != 0 a search captures its whole launch sequence
 * (frame-table copy, memsets, kernels) in a CUDA graph and replays it while
 * the batch keeps its sizes, pointers and configuration; the frame table
 * (cells may change) is re-read from pinned memory at every replay.
 * lc_gpu_graph_captures counts the captures. */
int lc_gpu_set_graph(lc_gpu_workspace *ws, int on);
int lc_gpu_graph_captures(lc_gpu_workspace *ws);

/* Enqueue on the caller's stream instead of the workspace's own one
 * (NULL restores the workspace stream). */
int lc_gpu_set_stream(lc_gpu_workspace *ws, void *stream);

/* Walk counters of the last search issued with wait != 0: pairs evaluated,
 * heap insertions, exact replays, shells, pruned cells, FP64 reranks,
 * proposal under / over / exact, revisited shells. device_ms is the device
 * time of the whole search. Returns the number of counters written. The
 * learned mode's warp walk counts only with lc_gpu_set_stats on. */
int lc_gpu_stats(lc_gpu_workspace *ws, long long *counters, int n_counters, double *device_ms);

/* Extension: counting in the learned mode's warp-per-source walk (off by
 * default: the counters cost about 3 % of that walk). */
int lc_gpu_set_stats(lc_gpu_workspace *ws, int on);

/* Extension (several GPUs, one process each): one rank's share of a search
 * whose inputs every rank holds. No counterpart in the reference; its split
 * point is the per-source loop of src/knearest.rs:477-485 (sources are
 * independent once the points are binned). Arguments as for
 * lc_gpu_knearest_many (device pointers, shared cell and mask), plus rank in
 * [0, world). Every rank bins the whole input; the cell-sorted sources are cut
 * into world contiguous ranges of equal expected work (cell occupancy times
 * the proposed cube) and this call walks rank's range. out_owned (n * n_frames
 * device ints) gets nonzero exactly for the rows this call wrote (its
 * sources, and on rank 0 the -1 / NaN rows of masked points); the other rows
 * of out_nn / out_d2 are left as they were. Zeroing the rows a rank does not
 * own and summing over the ranks (one all-reduce) gives the full rows. */
int lc_gpu_knearest_shard(lc_gpu_workspace *ws, const double *xyz, size_t n, size_t n_frames,
                          const struct lc_cell *simbox, size_t k, const int *mask,
                          double cell_hint, int rank, int world, int *out_nn, double *out_d2,
                          int *out_owned, int wait);

/* Extension, for failure-detection tests: the cell-count scan's look-back
 * waits at most spins loads (spins <= 0: the default bound), and the scan
 * tile silent_tile (-1: none) never publishes its state, so that the next
 * tile's wait runs out. A wait that runs out still yields exact offsets (the
 * tile sums its prefix from the counts) and the search then fails with
 * "device search failed" when it is waited for. No counterpart in the
 * reference, whose prefix scan does not wait across blocks. */
int lc_gpu_set_scan_limit(lc_gpu_workspace *ws, int spins, long long silent_tile);

/* Device time of the last search's phases, from CUDA events on the
 * workspace stream: fold + bin + scan + placement, the walk kernel, and the
 * exact replay of tied sources. Waits for the search to finish. */
int lc_gpu_phase_times(lc_gpu_workspace *ws, double *prep_ms, double *walk_ms, double *replay_ms);
/* Neighbour lists within a cutoff, as CSR, from the rows of a finished
 * search (no counterpart in the reference; its downstream consumers filter
 * the n * k list by a cutoff themselves). out_nn / out_d2: the search's
 * device output, rows x k, each row sorted ascending with -1 / NaN padding.
 * Entry j of row i is kept when out_nn[i*k + j] >= 0 and
 * out_d2[i*k + j] <= cutoff^2, in row order. row_ptr: rows + 1 device ints;
 * col and dist2 (dist2 may be NULL): device arrays of capacity cap. Waits,
 * stores the number of kept entries in *nnz, and fails (with row_ptr and
 * *nnz complete, the first cap entries written) when *nnz > cap. */
int lc_gpu_neighbors_within(lc_gpu_workspace *ws, const int *out_nn, const double *out_d2,
                            size_t rows, size_t k, double cutoff, int *row_ptr, int *col,
                            double *dist2, size_t cap, size_t *nnz);

/* The same split with the learned mode's shell proposals apart: walk_ms is
 * then the walk kernel alone. */
int lc_gpu_phase_times4(lc_gpu_workspace *ws, double *prep_ms, double *propose_ms, double *walk_ms,
                        double *replay_ms);

/* One frame of a heterogeneous batch: its own point count, cell, k and
 * hint. Frames are packed back to back in xyz (3 doubles per point) and in
 * the outputs (frame f starts at sum over g < f of n_g * k_g). mask_offset
 * is the frame's first entry in mask, or -1 for an unmasked frame. */
typedef struct lc_frame {
  size_t n;
  size_t k;
  struct lc_cell cell;
  double cell_hint;
  long long mask_offset;
} lc_frame;

int lc_gpu_knearest_batch(lc_gpu_workspace *ws, const double *xyz, const lc_frame *frames,
                          size_t n_frames, const int *mask, int *out_nn, double *out_d2,
                          int wait);

/* Extension: the same heterogeneous batch with HOST pointers (xyz, mask and
 * outputs), served like lc_knearest_d2 by the calling thread's workspace:
 * with page-locked output buffers the rows come back in ranges while the
 * rest is searched. mask spans max(mask_offset + n) ints. Errors go to
 * lc_last_error. Returns 0 or 1. */
int lc_knearest_batch(const double *xyz, const lc_frame *frames, size_t n_frames, const int *mask,
                      int *out_nn, double *out_d2);

/* One search that allocates no device memory (no counterpart in the
 * reference). For callers that cannot call cudaMalloc: hosts whose own pool
 * allocator owns all device memory, real-time loops that must not allocate,
 * plug-ins inside frameworks that own the allocator. Every scratch buffer
 * lives in one fixed static device array (about 6.7 MB on each GPU that
 * loads the library, held until exit); the caller passes device xyz, mask
 * (n ints or NULL), out_nn and out_d2 (n * k each, out_d2 may be NULL) and
 * a host lc_cell. Limits: n <= 65536 points, at most 65536 linked cells,
 * k <= 64; larger searches fail with an error. Work is enqueued on stream
 * (a cudaStream_t, NULL for the legacy default stream); wait != 0 also
 * waits and checks the device status. Every call looks up the array's
 * device address on the current device; the first call on a device also
 * loads the library's kernels there, so it should come before any stream
 * capture. With a mask, a mesh past the limits is an error only when some
 * point is active; an all-masked search returns -1 / NaN rows, as the
 * reference does, and the call then waits for its check of the mask. All
 * calls share the array and leave their contents in it: calls that overlap
 * on the GPU race and must not be issued. Results equal lc_gpu_knearest's. */
int lc_gpu_knearest_noalloc(const double *xyz, size_t n, const struct lc_cell *simbox, size_t k,
                            const int *mask, double cell_hint, int *out_nn, double *out_d2,
                            void *stream, int wait);

#ifdef __cplusplus
}
#endif

#endif /* LINKCELL_GPU_H */
