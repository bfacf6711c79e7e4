/* cbspmv.h -- C ABI of the B200-native CB-SpMV (cache-friendly block SpMV).
 *
 * The reference (xing-cong/CB-Sparse-DCU, cb-spmv-dcu/src/) is a header-only
 * C++/HIP library whose operator surface is two calls:
 *
 *   void coo2block_gather(const int *row, const int *col, const ValType *val,
 *                         GLOBAL_BLOCK &gb);                 coo2block.h:628
 *   PROGRAM_METRICS cb_spmv(const GLOBAL_BLOCK &gb, const ValType *x,
 *                           ValType *y);                      cb-spmv-dcu.hpp:1088
 *
 * This header keeps that surface (cbspmv_coo2block_gather, cbspmv_cb_spmv) and
 * splits the second call into upload / execute / free so the packed matrix
 * stays resident in HBM across solves.  Conventions:
 *   - every function returns a cbspmv_status; 0 is success.  No call exits
 *     the process (the reference's CHECK_HIP does, macros.h:17-31);
 *   - cbspmv_last_error() gives the message of the calling thread's last
 *     failure;
 *   - pointers are plain host or device addresses; streams are cudaStream_t
 *     passed as void* (0 = the legacy default stream);
 *   - a plan is immutable after upload; one plan may be executed on one
 *     stream at a time (its split-row scratch is shared by its launches).
 */
#ifndef CBSPMV_H
#define CBSPMV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int cbspmv_status;
enum {
    CBSPMV_OK = 0,
    CBSPMV_ERR_INVALID = 1,     /* bad argument, size or option           */
    CBSPMV_ERR_UNSORTED = 2,    /* COO rows not in non-decreasing order   */
    CBSPMV_ERR_BOUNDS = 3,      /* COO index outside [0,m) x [0,n)        */
    CBSPMV_ERR_ALLOC = 4,       /* host or device allocation failed       */
    CBSPMV_ERR_CUDA = 5,        /* a CUDA runtime call failed             */
    CBSPMV_ERR_STATE = 6,       /* plan not uploaded / wrong value type   */
    CBSPMV_ERR_UNSUPPORTED = 7, /* size beyond a documented limit         */
    CBSPMV_ERR_DEVICE = 8       /* a bounded device wait gave up in an
                                   earlier launch (see cbspmv_check)       */
};

enum { CBSPMV_F64 = 0, CBSPMV_F32 = 1 };

/* Build options.  The first five mirror the reference's compile-time macros
 * (macros.h:38-97; its Makefile:4-7 sets the defaults used here). */
typedef struct cbspmv_opts {
    int block_size;       /* CB_BLOCK_SIZE: 16 (default) or 32              */
    int row_owned;        /* CB_ROW_OWNED: 1 (default) row-owned segments;
                             0 builds the reference's balance permutation  */
    int waves_per_block;  /* CB_WAVES_PER_BLOCK: blocks per segment, 4      */
    int dense_sixteenths; /* CB_DENSE_SIXTEENTHS: dense if nnz >= bs*bs*k/16
                             (default 15)                                   */
    int force_coo64;      /* CB_FORCE_COO64: 0                              */
    int value_type;       /* CBSPMV_F64 (default) or CBSPMV_F32 values      */
    int want_transpose;   /* also build the CB layout of A^T for adjoints   */
    int tile_entries;     /* device tile size in stored entries (0 = auto)  */
    int kernel;           /* single-vector SpMV kernel: 0 auto, 1 streaming
                             (TMA-staged tiles, for COO-dominant matrices),
                             2 direct (high occupancy, for CSR/dense-heavy
                             ones), 3 staged (the several-right-hand-side
                             kernel, one vector), 4 pattern reuse (unit-
                             valued plans: one sum per row pattern, the
                             reference's EXEC_PATTERN_REUSE; automatic when
                             patterns are fewer than half the rows, as in
                             cb-spmv-dcu.hpp:1431-1433), 5 row segments (the
                             stored entries sorted by row in chunks of 128,
                             summed per lane and joined by one scan; built
                             at upload, and the automatic choice, when every
                             block is a COO block and values are stored;
                             keeps a second copy of the values on the
                             device), 6 balanced (plans built with row_owned
                             = 0 and stored values: the entries in the
                             plan's block order, grouped as the reference's
                             CTAs, added into y with atomics as its
                             non-row-owned mode does; the automatic choice
                             for one right-hand side on such plans); see
                             cbspmv_autotune */
    int keep_values;      /* 0 (default): when every stored value is 1, store
                             no values and DENSE blocks as bitmasks, as the
                             reference does (UNIT_VALUES,
                             cb-spmv-dcu.hpp:1105-1127); such a plan refuses
                             cbspmv_set_values.  1: always store values    */
} cbspmv_opts;

/* Host COO, 0-based, rows in non-decreasing order (the order the reference's
 * reader produces, io/mmio_highlevel.h:392-398); duplicates are allowed and
 * summed as the reference's builder sums them (coo2block.h:249-255). */
typedef struct cbspmv_coo {
    int32_t m, n;
    int64_t nnz;
    const int32_t *row;
    const int32_t *col;
    const double *val;
} cbspmv_coo;

/* PROGRAM_METRICS (format.h:185-188): mean kernel time and GFLOP/s. */
typedef struct cbspmv_metrics {
    double runtime_ms;
    double gflops;
} cbspmv_metrics;

/* Sizes of the built structure (GLOBAL_BLOCK counters, format.h:62-104) and
 * of the device layout. */
typedef struct cbspmv_info {
    int64_t m, n, nnz, gb_m, gb_n, gb_nnzb;
    int32_t gather_flag, direct_coo_columns, compact_coo_indices;
    int32_t load_balanced, unit_values;
    int64_t super_sparse_blocks, analyzed_blocks;
    double super_sparse_ratio, load_stddev_before, load_stddev_after;
    int64_t coo_blocks, csr_blocks, dense_blocks, uniform_blocks;
    int64_t segments, patterns, stored_values;
    int64_t tiles, split_rows, device_bytes, algorithmic_bytes;
    int64_t scratch_bytes;
    int64_t rowseg_bytes;   /* device bytes of the row-segment stream (kernel
                               5) once uploaded, else 0 */
} cbspmv_info;

typedef struct cbspmv_plan cbspmv_plan;

/* ---- reference surface ------------------------------------------------ */

/* Builds the CB structure on the host.  Replaces coo2block_gather
 * (coo2block.h:628-670) and produces the same GLOBAL_BLOCK content bit for
 * bit (block order, formats, index encodings, gather lists, segments,
 * balance permutation, row patterns).  opts may be NULL for the defaults. */
cbspmv_status cbspmv_coo2block_gather(const cbspmv_coo *coo,
                                      const cbspmv_opts *opts,
                                      cbspmv_plan **out);

/* Replaces cb_spmv (cb-spmv-dcu.hpp:1088-1667): host x (n values) and host y
 * (m values, overwritten), value type double.  Uploads the plan if needed,
 * runs one checked launch, 100 warm-up and 1000 timed launches as the
 * reference does (:1625-1656) and returns their mean time and 2*nnz/t. */
cbspmv_status cbspmv_cb_spmv(cbspmv_plan *plan, const double *x, double *y,
                             cbspmv_metrics *metrics);

/* ---- split surface ---------------------------------------------------- */

void cbspmv_default_opts(cbspmv_opts *opts);

/* Plan files (.cbplan, versioned binary): save writes a built plan's host
 * CB structures and device layouts (and the kernel chosen by
 * cbspmv_autotune); load recreates the plan without the COO input or the CB
 * build -- the reference rebuilds its structure on every run
 * (main.hip.cpp:67-68).  A loaded plan is not uploaded yet.  A file of
 * another format version, another byte order, or one that is truncated or
 * fails its checksum is refused with CBSPMV_ERR_INVALID. */
cbspmv_status cbspmv_plan_save(const cbspmv_plan *plan, const char *path);
cbspmv_status cbspmv_plan_load(const char *path, cbspmv_plan **out);

/* cbspmv_plan_save with flags.  CBSPMV_PLAN_SPMV_ONLY writes what products
 * need -- the options, the host structures' scalars, the block counts and
 * the device layouts' tiles, blocks and payload -- and leaves out the host
 * GLOBAL_BLOCK arrays and the per-value arrays (PL: 0.22 GB instead of 1.5
 * GB).  A plan loaded from such a file uploads, multiplies (cbspmv_spmv,
 * cbspmv_spmv_t, host and batch calls), autotunes and saves SpMV-only; the
 * calls that need per-value data (cbspmv_set_values, cbspmv_grad_vals, the
 * value gradient of cbspmv_adjoint, cbspmv_value_coords,
 * cbspmv_input_slots) return CBSPMV_ERR_STATE, and cbspmv_export returns -1
 * for every name but dev_tiles, dev_blocks, dev_payload and the rs_* names
 * (the row-segment stream is built from the tiles, so it is the same as the
 * saved plan's). */
#define CBSPMV_PLAN_SPMV_ONLY 1
cbspmv_status cbspmv_plan_save_ex(const cbspmv_plan *plan, const char *path,
                                  int flags);

/* The options a plan was built (or loaded) with; `kernel` reflects
 * cbspmv_autotune. */
cbspmv_status cbspmv_plan_opts(const cbspmv_plan *plan, cbspmv_opts *opts);

/* Copies the packed device layout to the current CUDA device. */
cbspmv_status cbspmv_upload(cbspmv_plan *plan, void *stream);

/* y = A x on the device, asynchronously on `stream`.  x and y are device
 * arrays of the plan's value type: x has n rows, y has m rows.  With
 * nrhs > 1 they are row-major n x nrhs / m x nrhs with leading dimensions
 * ldx, ldy >= nrhs (pass 0 for nrhs).  y is overwritten. */
cbspmv_status cbspmv_spmv(cbspmv_plan *plan, const void *x, void *y, int nrhs,
                          int64_t ldx, int64_t ldy, void *stream);

/* cbspmv_spmv for callers that may not allocate device memory while they
 * run -- e.g. a plugin whose execute step is handed only its inputs and
 * outputs by a host framework that owns all device memory, or a serving loop
 * with a fixed memory budget.  No counterpart in the reference (its cb_spmv
 * allocates on every call).  The plan must already be uploaded; the caller
 * passes x and y as for cbspmv_spmv.  The split-row partial sums, arrival
 * counters and scheduler words this call needs live in one fixed device
 * array of 8 MiB compiled into the library (held on every GPU that loads it
 * until the process exits), so this call allocates nothing.  A plan needing
 * more than 8 MiB of scratch (16 B + 4 B per block row + split tiles x nrhs
 * x bs values) is rejected with CBSPMV_ERR_UNSUPPORTED and a message giving
 * both sizes.  The first call on each device looks up the array's device
 * address; make that first call before any stream capture.  All calls share
 * the array and it keeps the last call's contents (the counters are cleared
 * at the start of every call), so calls that overlap on the GPU -- on
 * different streams, or from different plans -- race.  The looked-up address
 * is kept for the process: do not use this call after a device reset
 * (cudaDeviceReset) in the same process.  Plans whose kernel is the
 * row-segment stream need no scratch from the array (their span counters
 * and slots are the plan's own, allocated at upload). */
cbspmv_status cbspmv_spmv_noalloc(cbspmv_plan *plan, const void *x, void *y,
                                  int nrhs, int64_t ldx, int64_t ldy,
                                  void *stream);

/* The same through host buffers: copies x to the device, runs, copies y
 * back, and synchronizes `stream`.  Device buffers are kept in the plan. */
cbspmv_status cbspmv_spmv_host(cbspmv_plan *plan, const void *x_host,
                               void *y_host, int nrhs, void *stream);

/* cbspmv_spmv_host without the wait, for a stream of solves: copies x in,
 * runs and copies y out on three streams the plan keeps (two sets of device
 * buffers), so one call's copy in overlaps the previous call's kernel and the
 * one before's copy out, and returns at once.  x_host must hold the input
 * when the call is made (the copy in does not wait for `stream`).  `stream`
 * waits for this call's copy out; synchronize it before reading y_host, and
 * keep x_host unchanged and both buffers alive until then (pinned host memory
 * lets the copies run asynchronously).  The first call, and a call with more right-hand sides
 * than before, allocates the device buffers.  No counterpart in the
 * reference (its cb_spmv copies, runs and copies back one call at a time). */
cbspmv_status cbspmv_spmv_host_async(cbspmv_plan *plan, const void *x_host,
                                     void *y_host, int nrhs, void *stream);

/* Adjoint: gx = A^T g (g: m rows, gx: n rows, same conventions).  Needs the
 * plan built with want_transpose. */
cbspmv_status cbspmv_spmv_t(cbspmv_plan *plan, const void *g, void *gx,
                            int nrhs, int64_t ldg, int64_t ldgx, void *stream);

/* Gradient of <g, A x> with respect to the plan's stored value slots, in
 * packed order: gvals[k] = sum_j g[row_k, j] * x[col_k, j] (device arrays
 * of the plan's value type; gvals has cbspmv_num_values entries). */
cbspmv_status cbspmv_grad_vals(cbspmv_plan *plan, const void *g,
                               const void *x, void *gvals, int nrhs,
                               int64_t ldg, int64_t ldx, void *stream);

/* The whole backward pass of Y = A X for one upstream gradient g: gx = A^T g
 * (when gx is not NULL; needs want_transpose) and the value gradient gvals
 * (when gvals is not NULL), as cbspmv_spmv_t and cbspmv_grad_vals compute
 * them.  The two are independent, so the value gradient runs on a second
 * stream of the plan's own, forked from and joined back to `stream` by
 * events: work issued to `stream` afterwards sees both results, and the call
 * can be captured in a CUDA graph.  The first call with both outputs creates
 * that stream and its events, so make it before capturing one. */
cbspmv_status cbspmv_adjoint(cbspmv_plan *plan, const void *g, const void *x,
                             void *gx, void *gvals, int nrhs, int64_t ldg,
                             int64_t ldx, int64_t ldgx, void *stream);

/* The backward pass of Y = A X in ONE kernel launch on the transposed
 * layout (plans built with want_transpose and with stored values): gx = A^T g
 * and, from the same gathered rows of g, the value gradient of every stored
 * value of A^T, g[row] . x[col] summed over the right-hand sides.  gvals_t is
 * a device array of cbspmv_grad_size_t values indexed by payload position
 * (A^T's packed payload read as an array of values, so the gradient is
 * written in packed block order, coalesced); positions that hold no value
 * are left unchanged.  cbspmv_grad_positions_t gives, for each input nonzero
 * (caller's order), its position there.  No counterpart in the reference. */
cbspmv_status cbspmv_adjoint_fused(cbspmv_plan *plan, const void *g, const void *x,
                                   void *gx, void *gvals_t, int nrhs, int64_t ldg,
                                   int64_t ldx, int64_t ldgx, void *stream);
int64_t cbspmv_grad_size_t(const cbspmv_plan *plan);
cbspmv_status cbspmv_grad_positions_t(const cbspmv_plan *plan, int64_t *pos);

/* Stored values: the plan's packed value slots, in device (tile) order.
 * Dense blocks store all bs*bs values, so there can be more slots than input
 * nonzeros; COO blocks merge duplicates (coo2block.h:249-255), so there can
 * be fewer.  cbspmv_set_values takes NEW INPUT values (nnz of them, in the
 * caller's COO order, plan value type, device memory) and re-packs every slot
 * of A -- and of A^T when built -- as the sum of its input nonzeros, in the
 * builder's summation order. */
int64_t cbspmv_num_values(const cbspmv_plan *plan);
cbspmv_status cbspmv_set_values(cbspmv_plan *plan, const void *input_values,
                                void *stream);
/* For each stored slot: its row and column (-1 for dense padding outside
 * the matrix) and its first input nonzero (-1 if none).  Host arrays of
 * cbspmv_num_values entries; any pointer may be NULL. */
cbspmv_status cbspmv_value_coords(const cbspmv_plan *plan, int32_t *row,
                                  int32_t *col, int64_t *first_input);
/* For each input nonzero (caller's order): the slot it is summed into. */
cbspmv_status cbspmv_input_slots(const cbspmv_plan *plan, int64_t *slot);

cbspmv_status cbspmv_info_get(const cbspmv_plan *plan, cbspmv_info *info);

/* Copies one named GLOBAL_BLOCK array (the dump names of the oracle:
 * gb_row_idx, nnz_per_blk, type_per_blk, block_cols, segment_*, pattern_*,
 * bidx_*, pay_u32, pay_f64, pay_*_off, ...) into out (may be NULL) and
 * returns its length, or -1 for an unknown name.  The names dev_tiles,
 * dev_blocks (uint32 words), dev_payload (bytes) and dev_values (double, one
 * per stored slot) give the device layout itself; rs_sizes (nch, M, nseg,
 * nord, G, W), rs_chunks (bytes), rs_meta, rs_spans, rs_rowmap, rs_empty,
 * rs_vpos and rs_wbase (int32), each
 * followed by ":W", the row-segment stream as built for W resident warps
 * (-1 when the layout does not take it); bal_rows, bal_cols (uint32), bal_vals
 * (the value type) and bal_gstart (int64), the balanced schedule's stream
 * of a plan built with row_owned = 0 (-1 otherwise). */
int64_t cbspmv_export(const cbspmv_plan *plan, const char *name, void *out);

/* The same for the CB structure of A^T (plans built with want_transpose). */
int64_t cbspmv_export_t(const cbspmv_plan *plan, const char *name, void *out);

/* GLOBAL_BLOCK scalars of A (transpose = 0) or A^T: out12 = m, n, nnz, gb_m,
 * gb_n, gb_nnzb, gather_flag, direct_coo_columns, compact_coo_indices,
 * super_sparse_blocks, analyzed_blocks, load_balanced; out3 =
 * super_sparse_ratio, load_stddev_before, load_stddev_after. */
void cbspmv_export_scalars(const cbspmv_plan *plan, int transpose,
                           int64_t *out12, double *out3);

cbspmv_status cbspmv_destroy(cbspmv_plan *plan);

/* Message of the calling thread's last error ("" if none); returns its full
 * length. */
size_t cbspmv_last_error(char *buf, size_t len);

/* Device-side failure reporting.  The kernels wait on their own bulk copies
 * with bounded waits (no counterpart in the reference, whose row-epoch claim
 * spins without bound, cb-spmv-dcu.hpp:238-282).  A wait that gives up sets
 * an error word of the plan (host-mapped memory) and its warp stops, so the
 * launch's output is incomplete.  cbspmv_check synchronizes `stream` (and the
 * plan's own streams), and returns CBSPMV_ERR_DEVICE if a launch on the plan
 * gave up since the last report, else CBSPMV_OK.  Every launching call also
 * returns CBSPMV_ERR_DEVICE, without launching, when it finds the word set.
 * Either report clears the word and resets the plan's scratch (arrival
 * counters, scheduler words) on `stream`, so later calls run normally. */
cbspmv_status cbspmv_check(cbspmv_plan *plan, void *stream);

/* For tests of that path: the number of polls each device wait makes before
 * it gives up (0: at once, even when the copy has landed); polls < 0 restores
 * the default.  Process-wide; applies to launches made afterwards. */
void cbspmv_debug_wait_polls(int64_t polls);

/* Times the kernels that can run this plan for nrhs right-hand sides (one
 * vector: streaming when the layout allows it, direct, staged, and pattern
 * reuse, row segments and the balanced schedule when the plan has them;
 * several: the staged kernel and row segments) on scratch vectors, keeps
 * the fastest for later calls and returns it in *kernel (1 to 6) with its
 * mean time in *ms (either may be
 * NULL).  The plan must be uploaded; allocates and frees scratch device
 * memory and synchronizes `stream`.  No counterpart in the reference (its
 * kernel choice is compile-time, cb-spmv-dcu.hpp:1428-1450). */
cbspmv_status cbspmv_autotune(cbspmv_plan *plan, int nrhs, void *stream, int *kernel,
                              double *ms);

/* cbspmv_autotune that also tries, for nrhs > 1, the lanes per stored entry
 * of the several-right-hand-side kernel (1, 2 or 4 lanes side by side on one
 * x row, or its automatic choice from nrhs), keeps the fastest and returns it
 * in *rhs_lanes (0 = automatic; may be NULL).  Times on a non-zero x. */
cbspmv_status cbspmv_autotune_ex(cbspmv_plan *plan, int nrhs, void *stream, int *kernel,
                                 int *rhs_lanes, double *ms);

/* Lanes per stored entry of the several-right-hand-side kernel for this plan
 * (0: chosen from nrhs; 1, 2 or 4). */
cbspmv_status cbspmv_set_rhs_lanes(cbspmv_plan *plan, int lanes);

/* The tuner over the build's dimensions: builds the plan from the COO for
 * block size 16 and 32 and tile sizes (stored entries per warp tile) auto and
 * 128, uploads each, autotunes its kernel and lanes per entry
 * (cbspmv_autotune_ex) for nrhs right-hand sides, keeps the fastest plan in
 * *out and destroys the others.  The reference fixes these as compile-time
 * macros (macros.h:38-97, its Makefile:4-7).  rep (may be NULL) receives the
 * choice and its mean time.  Warps per CTA are fixed per kernel; the resident
 * count follows from registers and the L1 reserve. */
typedef struct cbspmv_tune_report {
    int block_size, tile_entries, kernel, rhs_lanes;
    double ms;
    int tried;
} cbspmv_tune_report;

cbspmv_status cbspmv_tune(const cbspmv_coo *coo, const cbspmv_opts *opts, int nrhs,
                          void *stream, cbspmv_plan **out, cbspmv_tune_report *rep);

/* ---- batches (no counterpart in the reference) ------------------------ */

/* Many uploaded plans -- same block size and value type, same device -- run
 * together: Y_k = A_k X_k for k < count, X_k row-major n_k x nrhs[k] and Y_k
 * row-major m_k x nrhs[k] (contiguous rows), nrhs[k] >= 1 per matrix.  One
 * batch launch runs every matrix, whatever its size and right-hand-side
 * count, in ONE persistent kernel: its warps take scheduling units of the
 * matrices' concatenated tiles from a device counter (the units are cut here
 * for the current device).  A plan may belong to several batches but is run
 * by one of them (or by itself) at a time. */
typedef struct cbspmv_batch cbspmv_batch;

cbspmv_status cbspmv_batch_create(cbspmv_plan *const *plans, int count,
                                  const int *nrhs, cbspmv_batch **out);

/* Binds the device arrays X_k (x[k]) and Y_k (y[k]) used by every later run
 * (host arrays of `count` device pointers).  Re-binding is allowed; a
 * per-matrix graph (below) is captured again after it. */
cbspmv_status cbspmv_batch_bind(cbspmv_batch *batch, const void *const *x,
                                void *const *y, void *stream);

/* One kernel launch over all matrices; allocates and copies nothing, so it
 * can be captured in a CUDA graph by the caller. */
cbspmv_status cbspmv_batch_run(cbspmv_batch *batch, void *stream);

/* The same result as one cbspmv_spmv launch per matrix, in order (the
 * unbatched way, kept for comparison). */
cbspmv_status cbspmv_batch_run_each(cbspmv_batch *batch, void *stream);

/* Replays a CUDA graph held by the batch: per_matrix = 0 captures
 * cbspmv_batch_run, per_matrix = 1 captures the per-matrix launches spread
 * over 8 parallel branches.  Captured on first use (and after a re-bind),
 * then launched on `stream`. */
cbspmv_status cbspmv_batch_graph_launch(cbspmv_batch *batch, int per_matrix,
                                        void *stream);

/* cbspmv_check for a batch: synchronizes `stream` and returns
 * CBSPMV_ERR_DEVICE if a batch launch gave up a bounded device wait since the
 * last report (its outputs are then incomplete; the batch's scratch is
 * reset).  cbspmv_batch_run and the graph launch report it too, without
 * launching. */
cbspmv_status cbspmv_batch_check(cbspmv_batch *batch, void *stream);

cbspmv_status cbspmv_batch_destroy(cbspmv_batch *batch);

/* Number of kernels this library launched in the calling process. */
int64_t cbspmv_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* CBSPMV_H */
