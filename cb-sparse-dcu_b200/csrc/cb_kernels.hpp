// Launchers of the sm_100a kernels (cb_kernels.cu), callable from host C++.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace cb {

// The row-segment stream on the device (layout in cb_rowseg.hpp); chunks is
// NULL when the plan has none.
struct RowSegDev {
    const uint8_t *chunks = nullptr;
    int32_t nch = 0, M = 0, nseg = 0, nord = 0;
    const int4 *meta = nullptr;       // per segment: ord0, starts_row, head span, tail span
    const int4 *spans = nullptr;      // per span: first segment, last segment, ordinal, 0
    int32_t *counters = nullptr;      // per span, zero between launches
    void *part = nullptr;             // 2 * nseg partial sums
    const int32_t *rowmap = nullptr;  // ordinal -> row, NULL when every row is non-empty
    const int32_t *empty = nullptr;   // rows without stored entries
    int32_t nempty = 0;
    const int32_t *vpos = nullptr;    // per stored value: its stream entry
    int32_t G = 0, W = 0;             // CTAs of every launch; window length (values)
    const int32_t *wbase = nullptr;   // per CTA: first column of its x window
    int64_t n = 0;                    // columns (length of x)
    int unit = 0;                     // words only: every stored value is 1
    int auto1 = 0;                    // the automatic choice for one right-hand side
};

// The balanced schedule's stream on the device (cb_rowseg.hpp,
// BalancedHost); rows is NULL when the plan has none.
struct BalancedDev {
    const uint4 *rows = nullptr, *cols = nullptr;  // 4 entries per quad
    const void *vals = nullptr;                    // 4 values per quad
    const int64_t *gstart = nullptr;               // ngroups + 1 quad indices
    const int64_t *eoff = nullptr;                 // per entry: payload offset (-1: skip)
    int64_t ngroups = 0, nquads = 0;
};

// Device-resident pieces of one DeviceLayout (cb_layout.hpp).
struct DevLayout {
    const void *tiles = nullptr;      // TileDesc[ntiles]
    const void *blocks = nullptr;     // BlockDesc[nblocks]
    const uint8_t *payload = nullptr;
    const int32_t *block_cols = nullptr;
    int64_t ntiles = 0;
    int bs = 16, f32 = 0, gather = 0;
    int unit = 0;                     // no stored values (all 1), DENSE as bitmasks
    int64_t m = 0, n = 0;
    void *partials = nullptr;         // slots * bs values (scratch)
    int32_t *counters = nullptr;      // gb_m arrival counters (scratch)
    uint32_t *sched = nullptr;        // scheduler words (scratch, zeroed)
    uint32_t *err = nullptr;          // error word: set when a bounded wait gives up
    int has_x = 1;                    // the layout has CSR/DENSE blocks
    int rl = 0;                       // lanes per entry of the several-right-hand-side
                                      // kernel (0: its automatic choice)
    // pattern reuse (unit-valued plans, one right-hand side): the rows that
    // share one column pattern share one sum (kernel 4)
    const int32_t *pat_ptr = nullptr, *pat_col = nullptr;
    const int32_t *pat_out_ptr = nullptr, *pat_out_rows = nullptr;
    int64_t npat = 0, pat_cols = 0;
    int pat_auto = 0;                 // the automatic choice takes it
    // small unit-valued gathered matrices: the automatic choice is the
    // direct kernel, whose block rows then fit one unit each and store y
    // directly (the reference's EXEC_SMALL_DIRECT, cb-spmv-dcu.hpp:1437-1439)
    int small_direct = 0;
    int64_t max_entries = 0;          // largest COO section of a tile
    int kernel = 0;                   // 0 auto, 1 streaming (TMA), 2 direct, 3 several
                                      // right-hand sides, 4 pattern reuse, 5 row segments,
                                      // 6 balanced
    RowSegDev rs;                     // row-segment stream (kernel 5)
    BalancedDev bal;                  // balanced schedule (kernel 6; row_owned = 0)
    double coo_share = 1.0;
    const uint32_t *wpart = nullptr;  // streaming: per-warp tile ranges
    int64_t nwarps = 0;               // streaming: warps of the launch
    uint32_t pay16_end = 0;           // payload size in 16-byte units
    // direct kernel: units of one block row (kDirectUnitTiles tiles at most)
    const uint32_t *dunit = nullptr;  // ndunits + 1 tile indices
    int64_t ndunits = 0;
    // several right-hand sides: tile buffer bytes, scheduling units
    uint32_t mcap = 0;
    const int64_t *ustart = nullptr;  // nunits + 1 tile indices
    int64_t nunits = 0;
};

// One matrix as the multi-right-hand-side and batch kernels see it (plain
// data, copied to the device as a table for batches).
struct MatView {
    const uint4 *tiles = nullptr;
    const uint4 *blocks = nullptr;
    const uint8_t *payload = nullptr;
    const int32_t *block_cols = nullptr;
    const void *x = nullptr;    // n x nrhs, row stride ldx
    void *y = nullptr;          // m x nrhs, row stride ldy
    void *partials = nullptr;   // slots * nrhs * bs values
    int32_t *counters = nullptr;
    int64_t ntiles = 0, m = 0, ldx = 1, ldy = 1;
    int nrhs = 1, gather = 0;
    int xvec = 0;               // x rows allow vector loads of V values
    int unit = 0;               // no stored values (all 1), DENSE as bitmasks
    uint32_t pay16_end = 0;     // payload size in 16-byte units
    // value gradient in the same pass (the transposed layout of an adjoint):
    // gv[p] = sum_j x[col, j] * xo[row, j] for the value at payload position p
    // (the payload read as an array of values); NULL: none
    void *gv = nullptr;
    const void *xo = nullptr;   // row vectors of the layout's rows, stride ldo
    int64_t ldo = 0;
    int rl = 0;                 // lanes per entry (0: chosen from nrhs)
};

// Shared-memory buffer bytes for tiles of at most max_tile_bytes.
uint32_t ms_cap(int64_t max_tile_bytes);
MatView mat_view(const DevLayout &d, const void *x, void *y, int nrhs, int64_t ldx,
                 int64_t ldy);
// Scheduling units of the multi-right-hand-side kernel.  ms_warps: warps one
// launch keeps resident on the current device; ms_tile_cost: relative cost of
// one tile (TileDesc words, the layout's BlockDesc words), for cost-balanced
// static units (one per warp) of a single matrix; ms_unit_starts: dynamic
// units of a batch -- the unit starts of one matrix's tiles (TileDesc words;
// tile indices offset by `base`) appended to ustart, boundaries at block-row
// starts once a unit holds `target` tiles, anywhere at twice that.  The
// caller appends the end (total tiles).
int64_t ms_warps(int bs, int f32, uint32_t cap);
int64_t ms_tile_cost(const uint32_t *tile8, const uint32_t *blocks4);
void ms_unit_starts(const uint32_t *tile8, int64_t ntiles, int64_t target, int64_t base,
                    std::vector<int64_t> &ustart);
// Y = A X through the multi-right-hand-side kernel (d.mcap, d.ustart,
// d.nunits set; scheduler words d.sched[0..1], error word d.err).
// With gv: also the value gradient of every stored value, gv[p] = sum over
// the right-hand sides of x[col] . xo[row] for the value at payload position
// p (the payload read as an array of values; xo row-major, stride ldo).
cudaError_t launch_spmm(const DevLayout &d, const void *x, void *y, int nrhs, int64_t ldx,
                        int64_t ldy, cudaStream_t stream, void *gv = nullptr,
                        const void *xo = nullptr, int64_t ldo = 0);
// The same kernel over a device table of nmats matrices (each with its own
// right-hand-side count) in ONE launch: tile offsets toff[nmats + 1], units
// ustart[nunits + 1] over the concatenated tiles taken in the queue order
// uorder[nunits], shared buffers of cap bytes (>= every matrix's largest
// tile), two scheduler words (zero before the first launch; the kernel leaves
// them zero) and an error word.
cudaError_t launch_batch(int bs, int f32, const MatView *mats, int nmats, const int64_t *toff,
                         const int64_t *ustart, const int32_t *uorder, int64_t nunits,
                         uint32_t cap, uint32_t *sched, uint32_t *err, cudaStream_t stream);
// Relative cost of one tile of a matrix with nrhs right-hand sides (the
// entries and block values it reads, times its passes over V columns).
int64_t ms_tile_cost_rhs(const uint32_t *tile8, const uint32_t *blocks4, int nrhs, int f32);

// The direct kernel's scheduling units: each block row's tiles in pieces of
// at most kDirectUnitTiles, starting at the row's first tile; direct_units
// returns the unit starts followed by the tile count.
constexpr int kDirectUnitTiles = 16;
std::vector<uint32_t> direct_units(const uint32_t *tile8, int64_t ntiles);

// Warps of a streaming-kernel launch for this layout on the current device,
// or 0 when the direct kernel is the one that runs.
int64_t stream_warps(const DevLayout &d);

// The pattern-reuse schedule (unit values, one right-hand side): per column
// pattern, lanes sum x over its columns and write the sum to every row of the
// pattern (the reference's EXEC_PATTERN_REUSE_*, cb-spmv-dcu.hpp:626-674).
cudaError_t launch_pattern(const DevLayout &d, const void *x, void *y, cudaStream_t stream);

// Row-segment stream (cb_rowseg_kernels.cu): warps of one launch on the current
// device (one CTA of kRsWarps warps per SM; 0 when the kernel cannot run);
// y = A x over d.rs; the stream's values refreshed from the tile payload
// (after the payload's values changed).
int64_t rowseg_warps(int f32);
cudaError_t launch_rowseg(const DevLayout &d, const void *x, void *y, cudaStream_t stream);
// Y = A X over d.rs for nrhs right-hand sides (row-major, leading dims ldx,
// ldy; slabs of 16 per launch); partial slots hold 16 values.
constexpr int kRsSlotValues = 16;
cudaError_t launch_rowseg_mrhs(const DevLayout &d, const void *x, void *y, int nrhs,
                               int64_t ldx, int64_t ldy, cudaStream_t stream);
cudaError_t launch_rowseg_values(const DevLayout &d, int64_t nvals, const uint64_t *val_off,
                                 cudaStream_t stream);

// The fused adjoint over a transposed plan's stream d.rs (values stored):
// gx = A^T g (n x nrhs, the stream's rows) and, per stream entry e of row j
// gathering row i of g, gv[e] = sum over the right-hand sides of
// g[i, :] . x[j, :] (gv holds nch * 128 values; padding entries get 0).
cudaError_t launch_rowseg_adjoint(const DevLayout &d, const void *g, void *gx, int nrhs,
                                  int64_t ldg, int64_t ldgx, const void *x, int64_t ldx,
                                  void *gv, cudaStream_t stream);

// y = A x by the balanced schedule over d.bal (zeroes y, then one launch
// adding with atomics); its values refreshed from the tile payload.
cudaError_t launch_balanced(const DevLayout &d, const void *x, void *y, cudaStream_t stream);
cudaError_t launch_balanced_values(const DevLayout &d, cudaStream_t stream);

// Batches over the row-segment streams: one matrix of the device table.
struct RsBatchMat {
    const uint8_t *chunks = nullptr;
    const int32_t *rowmap = nullptr;  // NULL: ordinals are rows
    const void *x = nullptr;
    void *y = nullptr;
    int64_t ldx = 0, ldy = 0;
    int32_t nrhs = 0, nord = 0;
    int32_t xvec = 0, yvec = 0;       // 16-byte x loads / y stores allowed
    int32_t g = 1, unit = 0;          // lanes per entry; words only
};
// Lanes per entry for nrhs right-hand sides (1, 2, 4; 8 for FP64 above 8).
int rs_lanes_per_entry(int f32, int nrhs);
// Warps of one batch launch on the current device (one CTA of kRsBatchWarps
// warps per SM).
int64_t rowseg_batch_warps(int f32);
// One launch: warps take segments segs[0 .. nseg) ({matrix, first chunk,
// end chunk, -}, in queue order) from the scheduler word sched[0] (sched[0..1]
// zero before the first launch; the kernel leaves them zero), with meta[]
// ({ordinal before, starts a row, head span, tail span}); empty rows {matrix,
// row} are zeroed first; spans {first segment, last segment, ordinal, -},
// counters (zero) and partial slots (kRsSlotValues values, two per segment)
// belong to the batch.
cudaError_t launch_rowseg_batch(int f32, const RsBatchMat *mats, const int4 *segs,
                                const int4 *meta, int32_t nseg, uint32_t *sched, int64_t nwarps,
                                const int2 *empty, int64_t nempty, const int4 *spans,
                                int32_t *counters, void *part, cudaStream_t stream);

// y = A x; x: n rows, y: m rows, row-major with leading dims for nrhs > 1.
cudaError_t launch_spmv(const DevLayout &d, const void *x, void *y, int nrhs,
                        int64_t ldx, int64_t ldy, cudaStream_t stream);

// The same SpMV with its scratch (scheduler words, arrival counters, split-row
// partials) placed in a fixed device array of kFixedScratchBytes instead of
// the plan's own allocations; no device memory is allocated.  Fails with
// cudaErrorInvalidValue when the plan needs more scratch than the array holds
// (fixed_scratch_need tells how much).
constexpr size_t kFixedScratchBytes = size_t(8) << 20;
size_t fixed_scratch_need(int64_t gb_m, int64_t slots, int nrhs, int bs, int f32);
cudaError_t launch_spmv_fixed_scratch(const DevLayout &d, int64_t gb_m, int64_t slots,
                                      const void *x, void *y, int nrhs, int64_t ldx,
                                      int64_t ldy, cudaStream_t stream);

// payload value v = sum of in[vsrc[z]] for z in [vsrc_ptr[v], vsrc_ptr[v+1])
cudaError_t launch_set_values(int f32, int64_t nvals, const int64_t *vsrc_ptr,
                              const int32_t *vsrc, const uint64_t *val_off,
                              const void *in, uint8_t *payload,
                              cudaStream_t stream);

// gvals[v] = sum_j g[row_v * ldg + j] * x[col_v * ldx + j] (0 when the slot
// has no row or column)
cudaError_t launch_grad_vals(int f32, int64_t nvals, const int32_t *vrow,
                             const int32_t *vcol, const void *g, int64_t ldg,
                             const void *x, int64_t ldx, int nrhs, void *gvals,
                             cudaStream_t stream);

// Kernel launches made by this library so far (every launcher above);
// note_launch() counts one.
int64_t kernel_launches();
void note_launch();

// Launch facts of the current device, kept per device (a process may drive
// several GPUs, and cudaFuncSetAttribute applies to the current device only):
// its SM count; for a kernel, the dynamic shared memory enabled so far
// (raised when a launch needs more) and its resident blocks per SM at a block
// size and shared-memory size.  Thread-safe.
int dev_sms();
cudaError_t dev_enable_smem(const void *fn, size_t smem);
int dev_resident(const void *fn, int threads, size_t smem);
// Resident blocks per SM for the gather-heavy SpMV kernels: at most as many
// as fit in kL1Keep bytes less than the largest shared-memory carveout, with
// the kernel's carveout set to what they use, so that the SM's unified
// L1/shared memory keeps at least that much more for the L1 (the x gathers'
// misses in flight are held there: with the largest carveout the power-law
// SpMV ran 1.4x slower).
constexpr size_t kL1Keep = size_t(32) << 10;
int dev_resident_l1(const void *fn, int threads, size_t smem);

// Polls a bounded device wait makes before giving up (the kernels' `limit`
// argument): dev::kWaitLimit unless set_wait_polls(p >= 0) set p for tests of
// the give-up path; set_wait_polls(-1) restores the default.
uint32_t wait_polls();
void set_wait_polls(int64_t polls);

// Dynamic shared memory of the SpMV kernel per CTA.
size_t spmv_smem_bytes(int bs, int f32);

}  // namespace cb
