// Launchers of the sm_100a kernels (cb_kernels.cu), callable from host C++.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace cb {

// Device-resident pieces of one DeviceLayout (cb_layout.hpp).
struct DevLayout {
    const void *tiles = nullptr;      // TileDesc[ntiles]
    const void *blocks = nullptr;     // BlockDesc[nblocks]
    const uint8_t *payload = nullptr;
    const int32_t *block_cols = nullptr;
    int64_t ntiles = 0;
    int bs = 16, f32 = 0, gather = 0;
    int64_t m = 0, n = 0;
    void *partials = nullptr;         // slots * bs values (scratch)
    int32_t *counters = nullptr;      // gb_m arrival counters (scratch)
    uint32_t *sched = nullptr;        // scheduler words (scratch, zeroed)
    int64_t max_entries = 0;          // largest COO section of a tile
    int kernel = 0;                   // 0 auto, 1 streaming (TMA), 2 direct
    double coo_share = 1.0;
    const uint32_t *wpart = nullptr;  // streaming: per-warp tile ranges
    int64_t nwarps = 0;               // streaming: warps of the launch
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
    int lanes = 1;              // lanes per entry (spmm_lanes(nrhs))
};

// Lanes per stored entry of the multi-right-hand-side kernel for nrhs
// right-hand sides: the next power of two, at most 32.
int spmm_lanes(int nrhs);
MatView mat_view(const DevLayout &d, const void *x, void *y, int nrhs, int64_t ldx,
                 int64_t ldy);
// Y = A X through the multi-right-hand-side kernel (lanes = 0: spmm_lanes).
cudaError_t launch_spmm(const DevLayout &d, const void *x, void *y, int nrhs, int64_t ldx,
                        int64_t ldy, int lanes, cudaStream_t stream);
// Batch: warps one launch keeps resident on the current device, and the
// launch itself over a device table of nmats matrices (tile offsets
// toff[nmats + 1], warp ranges wpart[nwarps + 1] over the concatenated tiles).
int64_t batch_warps(int bs, int f32);
cudaError_t launch_batch(int bs, int f32, const MatView *mats, int nmats, const int64_t *toff,
                         const int64_t *wpart, int64_t nwarps, cudaStream_t stream);
// Relative cost of one tile (TileDesc words, the layout's BlockDesc words)
// with nrhs right-hand sides, for balancing warps over a batch.
int64_t batch_tile_cost(const uint32_t *tile8, const uint32_t *blocks4, int nrhs);

// Warps of a streaming-kernel launch for this layout on the current device,
// or 0 when the direct kernel is the one that runs.
int64_t stream_warps(const DevLayout &d);

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

// Dynamic shared memory of the SpMV kernel per CTA.
size_t spmv_smem_bytes(int bs, int f32);

}  // namespace cb
