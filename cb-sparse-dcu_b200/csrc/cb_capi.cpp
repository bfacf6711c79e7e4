// C ABI of include/cbspmv.h.  Plans own the host structure (for export and
// parity), the device layout, and the device buffers.  Every entry point
// returns a status and records a message; none exits or throws.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <future>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "cb_builder.hpp"
#include "cb_kernels.hpp"
#include "cb_layout.hpp"
#include "cb_planfile.hpp"
#include "cb_rowseg.hpp"
#include "cbspmv.h"

namespace {

thread_local std::string g_error;

cbspmv_status fail(cbspmv_status code, const std::string &msg) {
    g_error = msg;
    return code;
}

cbspmv_status cuda_fail(cudaError_t e, const char *what) {
    cudaGetLastError();  // clear a sticky-free error so later calls can run
    return fail(CBSPMV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CB_CUDA(call, what)                              \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

template <class T>
cudaError_t upload_vec(const std::vector<T> &v, T **dst, cudaStream_t s) {
    *dst = nullptr;
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc((void **)dst, v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T),
                           cudaMemcpyHostToDevice, s);
}

struct DevSide {
    cb::DeviceLayout lay;
    cb::DevLayout d;
    void *tiles = nullptr, *blocks = nullptr;
    uint8_t *payload = nullptr;
    int32_t *block_cols = nullptr;
    void *partials = nullptr;
    int32_t *counters = nullptr;
    uint32_t *wpart = nullptr;
    uint32_t *dunit = nullptr;
    int64_t *ustart = nullptr;
    int partial_nrhs = 0;
    int64_t *vsrc_ptr = nullptr;
    int32_t *vsrc = nullptr;
    uint64_t *val_off = nullptr;
    int32_t *val_row = nullptr, *val_col = nullptr;
    int32_t *pat[4] = {};  // pattern row_ptr, col_idx, output_ptr, output_rows
    // row-segment stream (kernel 5): chunks, segment meta, spans, counters,
    // partial slots, rowmap, empty rows, value positions, window bases
    void *rs[9] = {};
    int64_t rs_bytes = 0;
    std::vector<int32_t> rs_cinfo;  // per chunk summaries (batches cut their own segments)
    std::vector<int32_t> rs_empty;  // rows without entries
    std::vector<int32_t> rs_vpos;   // per stored value: its stream entry (-1: none)
    // balanced schedule (row_owned = 0 plans): rows, cols, vals, gstart, eoff
    void *bal[5] = {};
    int64_t bal_bytes = 0;

    void release() {
        void *ps[] = {tiles, blocks, payload, block_cols, partials, counters,
                      wpart, dunit, ustart, vsrc_ptr, vsrc, val_off, val_row, val_col,
                      pat[0], pat[1], pat[2], pat[3]};
        for (void *p : ps)
            if (p) cudaFree(p);
        for (void *&q : rs) {
            if (q) cudaFree(q);
            q = nullptr;
        }
        rs_bytes = 0;
        for (void *&q : bal) {
            if (q) cudaFree(q);
            q = nullptr;
        }
        bal_bytes = 0;
        rs_cinfo.clear();
        rs_empty.clear();
        rs_vpos.clear();
        for (int32_t *&q : pat) q = nullptr;
        tiles = blocks = partials = nullptr;
        payload = nullptr;
        block_cols = counters = vsrc = val_row = val_col = nullptr;
        wpart = nullptr;
        dunit = nullptr;
        ustart = nullptr;
        vsrc_ptr = nullptr;
        val_off = nullptr;
        partial_nrhs = 0;
        d = cb::DevLayout();
    }
};

}  // namespace

// Pipelined host-buffer calls (cbspmv_spmv_host_async): copy in, compute and
// copy out on three streams of their own, two sets of device buffers, so call
// i+1's copy in overlaps call i's kernel and call i-1's copy out.
struct HostPipe {
    cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
    void *x[2] = {}, *y[2] = {};
    size_t xb = 0, yb = 0;  // bytes of each buffer
    // x_ready: copy in done; x_free: kernel done reading x; y_ready: kernel
    // done writing y; y_free: copy out done
    cudaEvent_t x_ready[2] = {}, x_free[2] = {}, y_ready[2] = {}, y_free[2] = {};
    bool used[2] = {false, false};
    int64_t calls = 0;
    void release() {
        for (int b = 0; b < 2; ++b) {
            if (x[b]) cudaFree(x[b]);
            if (y[b]) cudaFree(y[b]);
            x[b] = y[b] = nullptr;
            for (cudaEvent_t *e : {&x_ready[b], &x_free[b], &y_ready[b], &y_free[b]})
                if (*e) cudaEventDestroy(*e), *e = nullptr;
            used[b] = false;
        }
        for (cudaStream_t *st : {&in, &comp, &out})
            if (*st) cudaStreamDestroy(*st), *st = nullptr;
        xb = yb = 0;
    }
};

struct cbspmv_plan {
    cbspmv_opts opts;
    cb::HostCB host, host_t;
    DevSide A, AT;
    bool has_t = false;
    bool uploaded = false;
    int device = -1;
    // staging for the host-buffer entry points
    void *hx = nullptr, *hy = nullptr;
    size_t hx_bytes = 0, hy_bytes = 0;
    HostPipe pipe;
    // loaded from an SpMV-only plan file: no per-value arrays, no host block
    // arrays; counts = the block counts the plan's info reports
    bool spmv_only = false;
    int64_t counts[6] = {};
    // cbspmv_adjoint: the value gradient's stream and its fork/join events
    cudaStream_t adj = nullptr;
    cudaEvent_t adj_fork = nullptr, adj_join = nullptr;
    // error words of A's and A^T's launches (host-mapped pinned memory, so the
    // host reads them without a copy): set by a kernel whose bounded wait gave
    // up; herr is the host view, derr the device view
    uint32_t *herr = nullptr, *derr = nullptr;
    ~cbspmv_plan() {
        if (pipe.comp) cudaStreamSynchronize(pipe.out ? pipe.out : pipe.comp);
        pipe.release();
        if (adj) cudaStreamSynchronize(adj), cudaStreamDestroy(adj);
        if (adj_fork) cudaEventDestroy(adj_fork);
        if (adj_join) cudaEventDestroy(adj_join);
        A.release();
        AT.release();
        if (hx) cudaFree(hx);
        if (hy) cudaFree(hy);
        if (herr) cudaFreeHost(herr);
    }
};

namespace {

// A's COO, CSR, DENSE and uniform blocks, segments and row patterns.
void block_counts(const cbspmv_plan *p, int64_t out[6]) {
    if (p->spmv_only) {
        std::memcpy(out, p->counts, sizeof p->counts);
        return;
    }
    const cb::HostCB &g = p->host;
    for (int q = 0; q < 6; ++q) out[q] = 0;
    for (int64_t i = 0; i < g.nnzb; ++i) {
        if (g.nnz_blk[i] <= 0) continue;
        const int t = g.type_blk[i] & cb::kTypeMask;
        out[0] += t == cb::kCOO;
        out[1] += t == cb::kCSR;
        out[2] += t == cb::kDENSE;
        out[3] += (g.type_blk[i] & cb::kUniform) != 0;
    }
    out[4] = (int64_t)g.seg_rows.size();
    out[5] = g.pat_row_ptr.empty() ? 0 : (int64_t)g.pat_row_ptr.size() - 1;
}

// Calls that need the per-value arrays an SpMV-only plan file leaves out.
cbspmv_status refuse_spmv_only(const cbspmv_plan *p) {
    return p->spmv_only
        ? fail(CBSPMV_ERR_STATE, "plan loaded from an SpMV-only plan file holds no "
                                 "per-value data")
        : CBSPMV_OK;
}

size_t vsize(const cbspmv_plan *p) {
    return p->opts.value_type == CBSPMV_F32 ? 4 : 8;
}

cbspmv_status upload_side(DevSide &s, cudaStream_t st) {
    const cb::DeviceLayout &L = s.lay;
    CB_CUDA(upload_vec(L.tiles, (cb::TileDesc **)&s.tiles, st), "upload tiles");
    CB_CUDA(upload_vec(L.blocks, (cb::BlockDesc **)&s.blocks, st), "upload blocks");
    CB_CUDA(upload_vec(L.payload, &s.payload, st), "upload payload");
    CB_CUDA(upload_vec(L.block_cols, &s.block_cols, st), "upload gather list");
    CB_CUDA(upload_vec(L.vsrc_ptr, &s.vsrc_ptr, st), "upload value sources");
    CB_CUDA(upload_vec(L.vsrc, &s.vsrc, st), "upload value sources");
    CB_CUDA(upload_vec(L.val_off, &s.val_off, st), "upload value offsets");
    CB_CUDA(upload_vec(L.val_row, &s.val_row, st), "upload value rows");
    CB_CUDA(upload_vec(L.val_col, &s.val_col, st), "upload value columns");
    // scratch: 4 scheduler words (next tile, warps done, error word, spare),
    // then one arrival counter per block row
    CB_CUDA(cudaMalloc((void **)&s.counters, (L.gb_m + 4) * sizeof(int32_t)),
            "allocate counters");
    CB_CUDA(cudaMemsetAsync(s.counters, 0, (L.gb_m + 4) * sizeof(int32_t), st),
            "clear counters");
    s.d.tiles = s.tiles;
    s.d.blocks = s.blocks;
    s.d.payload = s.payload;
    s.d.block_cols = s.block_cols;
    s.d.ntiles = (int64_t)L.tiles.size();
    s.d.bs = L.bs;
    s.d.f32 = L.f32;
    s.d.gather = L.gather;
    s.d.m = L.m;
    s.d.n = L.n;
    s.d.pay16_end = (uint32_t)(L.payload.size() / 16);
    s.d.unit = L.unit;
    s.d.sched = reinterpret_cast<uint32_t *>(s.counters);
    s.d.counters = s.counters + 4;
    s.d.max_entries = L.max_entries;
    s.d.coo_share = L.coo_share;
    s.d.has_x = 0;
    for (const cb::TileDesc &t : L.tiles)
        if ((t.counts >> 16) & 0xffu) {
            s.d.has_x = 1;
            break;
        }
    return CBSPMV_OK;
}

// The streaming kernel's per-warp tile ranges for this device's grid, and the
// multi-right-hand-side kernel's tile buffer size.
cbspmv_status upload_partition(DevSide &s, int kernel, cudaStream_t st) {
    // the streaming partition whenever the layout allows that kernel, so a
    // later kernel choice (cbspmv_autotune) needs no new upload
    s.d.kernel = kernel == 0 || kernel == 1 ? kernel : 1;
    const int64_t warps = cb::stream_warps(s.d);
    s.d.kernel = kernel;
    if (warps > 0) {  // else the direct kernel runs single vectors
        const std::vector<uint32_t> part = cb::partition_tiles(s.lay, warps);
        CB_CUDA(upload_vec(part, &s.wpart, st), "upload tile partition");
        s.d.wpart = s.wpart;
        s.d.nwarps = warps;
    }
    const int64_t nt = (int64_t)s.lay.tiles.size();
    if (nt > 0) {  // the direct kernel's block-row units
        const std::vector<uint32_t> du =
            cb::direct_units(reinterpret_cast<const uint32_t *>(s.lay.tiles.data()), nt);
        CB_CUDA(upload_vec(du, &s.dunit, st), "upload direct units");
        s.d.dunit = s.dunit;
        s.d.ndunits = (int64_t)du.size() - 1;
    }
    // several right-hand sides: tile buffer size and scheduling units
    s.d.mcap = cb::ms_cap(s.lay.max_tile_bytes);
    if (nt > 0) {  // one cost-balanced range of tiles per resident warp
        const int64_t warps = std::min<int64_t>(nt, cb::ms_warps(s.lay.bs, s.lay.f32, s.d.mcap));
        if (warps <= 0) return fail(CBSPMV_ERR_CUDA, "multi-right-hand-side kernel setup");
        const uint32_t *t8 = reinterpret_cast<const uint32_t *>(s.lay.tiles.data());
        const uint32_t *b4 = reinterpret_cast<const uint32_t *>(s.lay.blocks.data());
        double total = 0, acc = 0;
        std::vector<int64_t> cost(nt);
        for (int64_t t = 0; t < nt; ++t) total += (double)(cost[t] = cb::ms_tile_cost(t8 + 8 * t, b4));
        std::vector<int64_t> us(1, 0);
        for (int64_t t = 0; t < nt && (int64_t)us.size() < warps; ++t) {
            acc += (double)cost[t];
            if (acc >= total * (double)us.size() / (double)warps && t + 1 < nt) us.push_back(t + 1);
        }
        s.d.nunits = (int64_t)us.size();
        us.push_back(nt);
        CB_CUDA(upload_vec(us, &s.ustart, st), "upload scheduling units");
        s.d.ustart = s.ustart;
    }
    return CBSPMV_OK;
}

// The row-segment stream (kernel 5; the automatic choice for several
// right-hand sides, and for one when every block is a COO block), segmented
// for this device's resident warps.
cbspmv_status upload_rowseg(DevSide &s, int kernel, cudaStream_t st) {
    if ((kernel != 0 && kernel != 5) || !cb::rowseg_applies(s.lay)) return CBSPMV_OK;
    const int64_t warps = cb::rowseg_warps(s.lay.f32);
    if (warps <= 0) return CBSPMV_OK;
    cb::RowSegHost R;
    const std::string msg = cb::build_rowseg(s.lay, warps, R);
    if (!msg.empty()) return fail(CBSPMV_ERR_UNSUPPORTED, msg);
    const size_t vsz = s.lay.f32 ? 4 : 8;
    const std::vector<int32_t> zeros(std::max<size_t>(1, R.spans.size() / 4), 0);
    CB_CUDA(upload_vec(R.chunks, (uint8_t **)&s.rs[0], st), "upload row segments");
    CB_CUDA(upload_vec(R.meta, (int32_t **)&s.rs[1], st), "upload row segments");
    if (!R.spans.empty())
        CB_CUDA(upload_vec(R.spans, (int32_t **)&s.rs[2], st), "upload row segments");
    CB_CUDA(upload_vec(zeros, (int32_t **)&s.rs[3], st), "upload row segments");
    CB_CUDA(cudaMalloc(&s.rs[4], 2 * (size_t)R.nseg * cb::kRsSlotValues * vsz),
            "allocate row-segment slots");
    CB_CUDA(upload_vec(R.rowmap, (int32_t **)&s.rs[5], st), "upload row segments");
    CB_CUDA(upload_vec(R.empty, (int32_t **)&s.rs[6], st), "upload row segments");
    CB_CUDA(upload_vec(R.vpos, (int32_t **)&s.rs[7], st), "upload row segments");
    CB_CUDA(upload_vec(R.wbase, (int32_t **)&s.rs[8], st), "upload row segments");
    cb::RowSegDev &d = s.d.rs;
    d.chunks = static_cast<const uint8_t *>(s.rs[0]);
    d.nch = R.nch;
    d.M = R.M;
    d.nseg = R.nseg;
    d.nord = R.nord;
    d.meta = static_cast<const int4 *>(s.rs[1]);
    d.spans = static_cast<const int4 *>(s.rs[2]);
    d.counters = static_cast<int32_t *>(s.rs[3]);
    d.part = s.rs[4];
    d.rowmap = R.rowmap.empty() ? nullptr : static_cast<const int32_t *>(s.rs[5]);
    d.empty = static_cast<const int32_t *>(s.rs[6]);
    d.nempty = (int32_t)R.empty.size();
    d.vpos = static_cast<const int32_t *>(s.rs[7]);
    d.G = R.G;
    d.W = R.W;
    d.wbase = static_cast<const int32_t *>(s.rs[8]);
    d.n = R.n;
    d.unit = R.unit;
    d.auto1 = cb::rowseg_all_coo(s.lay) ? 1 : 0;
    s.rs_bytes = (int64_t)(R.chunks.size() + 4 * (R.meta.size() + R.spans.size() +
                                                  R.rowmap.size() + R.empty.size()));
    s.rs_cinfo = std::move(R.cinfo);
    s.rs_empty = std::move(R.empty);
    s.rs_vpos = std::move(R.vpos);
    return CBSPMV_OK;
}

// The balanced schedule's stream (kernel 6, and the automatic choice for one
// right-hand side) of a plan built with row_owned = 0 and stored values.
cbspmv_status upload_balanced(DevSide &s, const cb::HostCB &g, int kernel, cudaStream_t st) {
    if ((kernel != 0 && kernel != 6) || g.o.row_owned || s.lay.unit || s.lay.nvals <= 0 ||
        g.gb_row.empty())
        return CBSPMV_OK;
    cb::BalancedHost B;
    const std::string msg = cb::build_balanced(s.lay, g, B);
    if (!msg.empty()) return fail(CBSPMV_ERR_UNSUPPORTED, msg);
    CB_CUDA(upload_vec(B.rows, (uint32_t **)&s.bal[0], st), "upload balanced stream");
    CB_CUDA(upload_vec(B.cols, (uint32_t **)&s.bal[1], st), "upload balanced stream");
    CB_CUDA(upload_vec(B.vals, (uint8_t **)&s.bal[2], st), "upload balanced stream");
    CB_CUDA(upload_vec(B.gstart, (int64_t **)&s.bal[3], st), "upload balanced stream");
    CB_CUDA(upload_vec(B.eoff, (int64_t **)&s.bal[4], st), "upload balanced stream");
    cb::BalancedDev &d = s.d.bal;
    d.rows = static_cast<const uint4 *>(s.bal[0]);
    d.cols = static_cast<const uint4 *>(s.bal[1]);
    d.vals = s.bal[2];
    d.gstart = static_cast<const int64_t *>(s.bal[3]);
    d.eoff = static_cast<const int64_t *>(s.bal[4]);
    d.ngroups = (int64_t)B.gstart.size() - 1;
    d.nquads = B.nquads;
    s.bal_bytes = (int64_t)(B.rows.size() * 8 + B.vals.size() + B.gstart.size() * 8);
    return CBSPMV_OK;
}

// The row patterns of a unit-valued plan (the reference's pattern_* arrays,
// coo2block.h:566-602) for the pattern-reuse schedule; its automatic choice
// follows the reference's rule: fewer patterns than half the rows
// (cb-spmv-dcu.hpp:1431-1433).
cbspmv_status upload_patterns(DevSide &s, const cb::HostCB &g, cudaStream_t st) {
    s.d.small_direct = s.lay.unit && g.gather_flag && g.compact && g.nnz < 10000 &&
                       g.o.row_owned;
    if (!s.lay.unit || g.pat_row_ptr.size() < 2) return CBSPMV_OK;
    CB_CUDA(upload_vec(g.pat_row_ptr, &s.pat[0], st), "upload patterns");
    CB_CUDA(upload_vec(g.pat_col, &s.pat[1], st), "upload patterns");
    CB_CUDA(upload_vec(g.pat_out_ptr, &s.pat[2], st), "upload patterns");
    CB_CUDA(upload_vec(g.pat_out_rows, &s.pat[3], st), "upload patterns");
    s.d.pat_ptr = s.pat[0];
    s.d.pat_col = s.pat[1];
    s.d.pat_out_ptr = s.pat[2];
    s.d.pat_out_rows = s.pat[3];
    s.d.npat = (int64_t)g.pat_row_ptr.size() - 1;
    s.d.pat_cols = (int64_t)g.pat_col.size();
    s.d.pat_auto = s.d.npat * 2 < g.m;
    return CBSPMV_OK;
}

// Partial slots sized for nrhs right-hand sides.
cbspmv_status ensure_partials(DevSide &s, int nrhs, size_t vsz) {
    if (s.lay.slots == 0 || s.partial_nrhs >= nrhs) return CBSPMV_OK;
    if (s.partials) cudaFree(s.partials);
    s.partials = nullptr;
    const size_t bytes = (size_t)s.lay.slots * nrhs * s.lay.bs * vsz;
    CB_CUDA(cudaMalloc(&s.partials, bytes), "allocate split-row partials");
    s.partial_nrhs = nrhs;
    s.d.partials = s.partials;
    return CBSPMV_OK;
}

// Reports (once) that a launch on side s (0 = A, 1 = A^T) of the plan gave up
// a bounded device wait, and resets the side's scheduler words and arrival
// counters on `st` so that later launches start clean.
cbspmv_status take_device_error(cbspmv_plan *p, int side, cudaStream_t st) {
    if (!p->herr) return CBSPMV_OK;
    volatile uint32_t *w = p->herr + side;
    if (*w == 0) return CBSPMV_OK;
    *w = 0;
    DevSide &s = side ? p->AT : p->A;
    if (s.counters) {
        const cudaError_t e =
            cudaMemsetAsync(s.counters, 0, (s.lay.gb_m + 4) * sizeof(int32_t), st);
        if (e != cudaSuccess) return cuda_fail(e, "reset scratch after a device error");
    }
    return fail(CBSPMV_ERR_DEVICE,
                std::string("a bounded device wait gave up in an earlier launch on this plan (") +
                    (side ? "A^T" : "A") +
                    "): that launch's output is incomplete; the plan's scratch was reset");
}

cbspmv_status device_errors(cbspmv_plan *p, cudaStream_t st) {
    cbspmv_status rc = take_device_error(p, 0, st);
    const cbspmv_status rt = take_device_error(p, 1, st);
    return rc ? rc : rt;
}

cbspmv_status run_side(cbspmv_plan *p, DevSide &s, const void *x, void *y,
                       int nrhs, int64_t ldx, int64_t ldy, cudaStream_t st) {
    if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "plan not uploaded");
    if (cbspmv_status rc = take_device_error(p, &s == &p->AT ? 1 : 0, st)) return rc;
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    if (ldx == 0) ldx = nrhs;
    if (ldy == 0) ldy = nrhs;
    if (ldx < nrhs || ldy < nrhs)
        return fail(CBSPMV_ERR_INVALID, "leading dimension smaller than nrhs");
    if ((s.lay.m > 0 && !y) || (s.lay.n > 0 && !x && s.lay.nvals > 0))
        return fail(CBSPMV_ERR_INVALID, "null x or y");
    cbspmv_status rc = ensure_partials(s, nrhs, vsize(p));
    if (rc) return rc;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != p->device)
        return fail(CBSPMV_ERR_STATE, "plan was uploaded to another device");
    CB_CUDA(cb::launch_spmv(s.d, x, y, nrhs, ldx, ldy, st), "spmv launch");
    return CBSPMV_OK;
}

cb::BuildOpts to_build(const cbspmv_opts &o) {
    cb::BuildOpts b;
    b.bs = o.block_size;
    b.row_owned = o.row_owned;
    b.waves = o.waves_per_block;
    b.dense_sixteenths = o.dense_sixteenths;
    b.force_coo64 = o.force_coo64;
    return b;
}

}  // namespace

extern "C" {

void cbspmv_default_opts(cbspmv_opts *o) {
    if (!o) return;
    o->block_size = 16;
    o->row_owned = 1;
    o->waves_per_block = 4;
    o->dense_sixteenths = 15;
    o->force_coo64 = 0;
    o->value_type = CBSPMV_F64;
    o->want_transpose = 0;
    o->tile_entries = 0;
    o->kernel = 0;
    o->keep_values = 0;
}

cbspmv_status cbspmv_coo2block_gather(const cbspmv_coo *coo,
                                      const cbspmv_opts *opts,
                                      cbspmv_plan **out) {
    if (!coo || !out) return fail(CBSPMV_ERR_INVALID, "null argument");
    *out = nullptr;
    cbspmv_opts o;
    cbspmv_default_opts(&o);
    if (opts) o = *opts;
    if (o.value_type != CBSPMV_F64 && o.value_type != CBSPMV_F32)
        return fail(CBSPMV_ERR_INVALID, "value_type must be CBSPMV_F64 or CBSPMV_F32");
    if (o.kernel < 0 || o.kernel > 6)
        return fail(CBSPMV_ERR_INVALID, "kernel must be 0 (auto) or 1 to 6");
    cbspmv_plan *p = new (std::nothrow) cbspmv_plan;
    if (!p) return fail(CBSPMV_ERR_ALLOC, "out of host memory");
    p->opts = o;
    try {
        // A^T (when wanted) is built on a second host thread while A is built
        // here: the two builds share nothing but the caller's COO, read-only.
        const int64_t nnz = coo->nnz;
        std::vector<int32_t> tr, tc, perm;
        std::vector<double> tv;
        std::future<std::pair<std::string, int>> side;
        // (a COO that fails these checks is refused by A's build below)
        if (o.want_transpose && coo->m >= 0 && coo->n >= 0 && nnz >= 0 &&
            (nnz == 0 || (coo->row && coo->col && coo->val))) {
            // A^T as a row-sorted COO: a stable counting sort by column keeps
            // each column's entries in row order.  The input is checked here
            // (columns in range) before it indexes anything; build_cb checks
            // the rest of it for A.
            const int64_t n = coo->n;
            for (int64_t i = 0; i < nnz; ++i)
                if (coo->col[i] < 0 || coo->col[i] >= n || coo->row[i] < 0 ||
                    coo->row[i] >= coo->m) {
                    delete p;
                    return fail(CBSPMV_ERR_BOUNDS, "COO index out of range");
                }
            std::vector<int64_t> cnt(n + 1, 0);
            for (int64_t i = 0; i < nnz; ++i) cnt[coo->col[i] + 1]++;
            for (int64_t c = 0; c < n; ++c) cnt[c + 1] += cnt[c];
            tr.resize(nnz);
            tc.resize(nnz);
            perm.resize(nnz);
            tv.resize(nnz);
            for (int64_t i = 0; i < nnz; ++i) {
                const int64_t d = cnt[coo->col[i]]++;
                tr[d] = coo->col[i];
                tc[d] = coo->row[i];
                tv[d] = coo->val[i];
                perm[d] = (int32_t)i;
            }
            side = std::async(std::launch::async, [&]() -> std::pair<std::string, int> {
                int c = 0;
                std::string e = cb::build_cb(to_build(o), coo->n, coo->m, nnz, tr.data(),
                                             tc.data(), tv.data(), p->host_t, &c);
                if (e.empty())
                    e = cb::build_layout(p->host_t, o.value_type == CBSPMV_F32, o.tile_entries,
                                         o.kernel, !o.keep_values, p->AT.lay, &c);
                return {e, c};
            });
        }
        int code = 0;
        std::string err = cb::build_cb(to_build(o), coo->m, coo->n, coo->nnz,
                                       coo->row, coo->col, coo->val, p->host, &code);
        if (err.empty())
            err = cb::build_layout(p->host, o.value_type == CBSPMV_F32, o.tile_entries,
                                   o.kernel, !o.keep_values, p->A.lay, &code);
        std::pair<std::string, int> terr;
        const bool have_t = side.valid();
        if (have_t) terr = side.get();  // joined before any return
        if (!err.empty()) {
            delete p;
            return fail(code, err);
        }
        if (o.want_transpose) {
            if (!have_t) {  // not reached: A's build refuses such input
                delete p;
                return fail(CBSPMV_ERR_INVALID, "transpose: invalid COO");
            }
            if (!terr.first.empty()) {
                delete p;
                return fail(terr.second, "transpose: " + terr.first);
            }
            // value sources of A^T refer to the caller's nonzero order
            for (int32_t &s : p->AT.lay.vsrc) s = perm[s];
            std::vector<int64_t> slot(nnz);
            for (int64_t i = 0; i < nnz; ++i) slot[perm[i]] = p->AT.lay.input_slot[i];
            p->AT.lay.input_slot.swap(slot);
            p->has_t = true;
        }
    } catch (const std::bad_alloc &) {
        delete p;
        return fail(CBSPMV_ERR_ALLOC, "out of host memory while building");
    }
    *out = p;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_plan_save(const cbspmv_plan *p, const char *path) {
    return cbspmv_plan_save_ex(p, path, 0);
}

cbspmv_status cbspmv_plan_save_ex(const cbspmv_plan *p, const char *path, int flags) {
    if (!p || !path) return fail(CBSPMV_ERR_INVALID, "null argument");
    if (flags & ~CBSPMV_PLAN_SPMV_ONLY) return fail(CBSPMV_ERR_INVALID, "unknown flags");
    if (p->spmv_only && !(flags & CBSPMV_PLAN_SPMV_ONLY))
        return fail(CBSPMV_ERR_STATE, "an SpMV-only plan can only be saved SpMV-only");
    cb::PlanImage img;
    img.flags = (flags & CBSPMV_PLAN_SPMV_ONLY) ? cb::kPlanSpmvOnly : 0;
    block_counts(p, img.counts);
    const cbspmv_opts &o = p->opts;
    const int32_t opts[10] = {o.block_size,  o.row_owned,      o.waves_per_block,
                              o.dense_sixteenths, o.force_coo64, o.value_type,
                              o.want_transpose,   o.tile_entries, o.kernel, o.keep_values};
    std::memcpy(img.opts, opts, sizeof opts);
    img.has_t = p->has_t ? 1 : 0;
    auto *q = const_cast<cbspmv_plan *>(p);  // visited, not modified, by the writer
    img.host = &q->host;
    img.host_t = &q->host_t;
    img.A = &q->A.lay;
    img.AT = &q->AT.lay;
    const std::string err = cb::save_plan(img, path);
    if (!err.empty()) return fail(CBSPMV_ERR_INVALID, err);
    return CBSPMV_OK;
}

cbspmv_status cbspmv_plan_opts(const cbspmv_plan *p, cbspmv_opts *opts) {
    if (!p || !opts) return fail(CBSPMV_ERR_INVALID, "null argument");
    *opts = p->opts;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_plan_load(const char *path, cbspmv_plan **out) {
    if (!path || !out) return fail(CBSPMV_ERR_INVALID, "null argument");
    *out = nullptr;
    cbspmv_plan *p = new (std::nothrow) cbspmv_plan;
    if (!p) return fail(CBSPMV_ERR_ALLOC, "out of host memory");
    cb::PlanImage img;
    img.host = &p->host;
    img.host_t = &p->host_t;
    img.A = &p->A.lay;
    img.AT = &p->AT.lay;
    std::string err;
    try {
        err = cb::load_plan(path, img);
    } catch (const std::bad_alloc &) {
        err = "out of host memory while loading";
    }
    if (!err.empty()) {
        delete p;
        return fail(CBSPMV_ERR_INVALID, err);
    }
    p->spmv_only = (img.flags & cb::kPlanSpmvOnly) != 0;
    std::memcpy(p->counts, img.counts, sizeof p->counts);
    cbspmv_opts &o = p->opts;
    o.block_size = img.opts[0];
    o.row_owned = img.opts[1];
    o.waves_per_block = img.opts[2];
    o.dense_sixteenths = img.opts[3];
    o.force_coo64 = img.opts[4];
    o.value_type = img.opts[5];
    o.want_transpose = img.opts[6];
    o.tile_entries = img.opts[7];
    o.kernel = img.opts[8];
    o.keep_values = img.opts[9];
    p->has_t = img.has_t != 0;
    if ((o.block_size != 16 && o.block_size != 32) ||
        (o.value_type != CBSPMV_F64 && o.value_type != CBSPMV_F32) || o.kernel < 0 ||
        o.kernel > 6 || p->A.lay.bs != o.block_size) {
        delete p;
        return fail(CBSPMV_ERR_INVALID, std::string(path) + " holds inconsistent options");
    }
    *out = p;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_upload(cbspmv_plan *p, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (p->uploaded) return CBSPMV_OK;
    cudaStream_t st = (cudaStream_t)stream;
    CB_CUDA(cudaGetDevice(&p->device), "cudaGetDevice");
    if (!p->herr) {
        CB_CUDA(cudaHostAlloc((void **)&p->herr, 16, cudaHostAllocMapped), "allocate error words");
        std::memset(p->herr, 0, 16);
        CB_CUDA(cudaHostGetDevicePointer((void **)&p->derr, p->herr, 0), "map error words");
    }
    cbspmv_status rc = upload_side(p->A, st);
    if (!rc) rc = upload_partition(p->A, p->opts.kernel, st);
    if (!rc) rc = upload_patterns(p->A, p->host, st);
    if (!rc) rc = upload_rowseg(p->A, p->opts.kernel, st);
    if (!rc && !p->spmv_only) rc = upload_balanced(p->A, p->host, p->opts.kernel, st);
    if (!rc && p->has_t) rc = upload_side(p->AT, st);
    if (!rc && p->has_t) rc = upload_partition(p->AT, p->opts.kernel, st);
    if (!rc && p->has_t) rc = upload_rowseg(p->AT, p->opts.kernel, st);
    p->A.d.err = p->derr;
    p->AT.d.err = p->derr + 1;
    if (rc) {
        p->A.release();
        p->AT.release();
        return rc;
    }
    CB_CUDA(cudaStreamSynchronize(st), "upload");
    p->uploaded = true;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_spmv(cbspmv_plan *p, const void *x, void *y, int nrhs,
                          int64_t ldx, int64_t ldy, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    return run_side(p, p->A, x, y, nrhs, ldx, ldy, (cudaStream_t)stream);
}

cbspmv_status cbspmv_spmv_noalloc(cbspmv_plan *p, const void *x, void *y, int nrhs,
                                  int64_t ldx, int64_t ldy, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "plan not uploaded");
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    if (ldx == 0) ldx = nrhs;
    if (ldy == 0) ldy = nrhs;
    if (ldx < nrhs || ldy < nrhs)
        return fail(CBSPMV_ERR_INVALID, "leading dimension smaller than nrhs");
    DevSide &s = p->A;
    if ((s.lay.m > 0 && !y) || (s.lay.n > 0 && !x && s.lay.nvals > 0))
        return fail(CBSPMV_ERR_INVALID, "null x or y");
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != p->device)
        return fail(CBSPMV_ERR_STATE, "plan was uploaded to another device");
    if (cbspmv_status rc = take_device_error(p, 0, (cudaStream_t)stream)) return rc;
    const size_t need = cb::fixed_scratch_need(s.lay.gb_m, s.lay.slots, nrhs, s.lay.bs,
                                               s.lay.f32);
    if (need > cb::kFixedScratchBytes)
        return fail(CBSPMV_ERR_UNSUPPORTED,
                    "cbspmv_spmv_noalloc: this plan needs " + std::to_string(need) +
                        " bytes of scratch for nrhs=" + std::to_string(nrhs) +
                        "; the fixed scratch holds " +
                        std::to_string(cb::kFixedScratchBytes) +
                        " bytes (use cbspmv_spmv, fewer right-hand sides or larger tiles)");
    CB_CUDA(cb::launch_spmv_fixed_scratch(s.d, s.lay.gb_m, s.lay.slots, x, y, nrhs, ldx,
                                          ldy, (cudaStream_t)stream),
            "spmv_noalloc launch");
    return CBSPMV_OK;
}

cbspmv_status cbspmv_check(cbspmv_plan *p, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (!p->uploaded) return CBSPMV_OK;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    CB_CUDA(cudaStreamSynchronize(st), "check: synchronize");
    if (p->pipe.comp) CB_CUDA(cudaStreamSynchronize(p->pipe.comp), "check: synchronize");
    if (p->adj) CB_CUDA(cudaStreamSynchronize(p->adj), "check: synchronize");
    return device_errors(p, st);
}

void cbspmv_debug_wait_polls(int64_t polls) { cb::set_wait_polls(polls); }

cbspmv_status cbspmv_set_rhs_lanes(cbspmv_plan *p, int lanes) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (lanes != 0 && lanes != 1 && lanes != 2 && lanes != 4)
        return fail(CBSPMV_ERR_INVALID, "rhs lanes must be 0 (automatic), 1, 2 or 4");
    p->A.d.rl = lanes;
    p->AT.d.rl = lanes;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_autotune_ex(cbspmv_plan *p, int nrhs, void *stream, int *kernel,
                                 int *rhs_lanes, double *ms) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "plan not uploaded");
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    DevSide &s = p->A;
    // candidates: (kernel, lanes per entry of the several-right-hand-side
    // kernel; 0 = its automatic choice)
    std::vector<std::pair<int, int>> cands;
    if (nrhs == 1) {
        cb::DevLayout probe = s.d;
        probe.kernel = 1;
        if (s.d.wpart && cb::stream_warps(probe) > 0) cands.push_back({1, 0});
        cands.push_back({2, 0});
        cands.push_back({3, 0});
        if (s.d.npat) cands.push_back({4, 0});
        if (s.d.rs.chunks) cands.push_back({5, 0});
        if (s.d.bal.rows) cands.push_back({6, 0});
    } else {
        for (int rl : {0, 1, 2, 4}) cands.push_back({3, rl});
        if (s.d.rs.chunks) cands.push_back({5, 0});
    }
    const size_t vsz = vsize(p);
    void *x = nullptr, *y = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        if (x) cudaFree(x);
        if (y) cudaFree(y);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    const size_t xb = std::max<size_t>(1, (size_t)s.lay.n * nrhs * vsz);
    cudaError_t e = cudaMalloc(&x, xb);
    if (e == cudaSuccess) e = cudaMalloc(&y, std::max<size_t>(1, (size_t)s.lay.m * nrhs * vsz));
    // a non-zero x (every byte 0x3c: small positive finite values), so that
    // no zero shortcut flatters a kernel
    if (e == cudaSuccess) e = cudaMemsetAsync(x, 0x3c, xb, st);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "autotune scratch");
    }
    const int keep = s.d.kernel, keep_rl = s.d.rl;
    int best = -1, best_rl = 0;
    float best_ms = 0.f;
    for (const auto &c : cands) {
        s.d.kernel = c.first;
        s.d.rl = c.second;
        cbspmv_status rc = CBSPMV_OK;
        for (int i = 0; i < 3 && !rc; ++i) rc = run_side(p, s, x, y, nrhs, nrhs, nrhs, st);
        constexpr int reps = 10;
        cudaEventRecord(e0, st);
        for (int i = 0; i < reps && !rc; ++i) rc = run_side(p, s, x, y, nrhs, nrhs, nrhs, st);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (rc || e != cudaSuccess) {
            s.d.kernel = keep;
            s.d.rl = keep_rl;
            cleanup();
            return rc ? rc : cuda_fail(e, "autotune timing");
        }
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        t /= reps;
        if (best < 0 || t < best_ms) {
            best = c.first;
            best_rl = c.second;
            best_ms = t;
        }
    }
    cleanup();
    s.d.kernel = best;
    s.d.rl = best_rl;
    p->opts.kernel = best;
    if (p->has_t) {
        p->AT.d.kernel = best == 1 && !p->AT.d.wpart ? 2 : best;
        p->AT.d.rl = best_rl;
    }
    if (kernel) *kernel = best;
    if (rhs_lanes) *rhs_lanes = best_rl;
    if (ms) *ms = best_ms;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_autotune(cbspmv_plan *p, int nrhs, void *stream, int *kernel, double *ms) {
    return cbspmv_autotune_ex(p, nrhs, stream, kernel, nullptr, ms);
}

cbspmv_status cbspmv_tune(const cbspmv_coo *coo, const cbspmv_opts *opts, int nrhs,
                          void *stream, cbspmv_plan **out, cbspmv_tune_report *rep) {
    if (!coo || !out) return fail(CBSPMV_ERR_INVALID, "null argument");
    *out = nullptr;
    cbspmv_opts base;
    cbspmv_default_opts(&base);
    if (opts) base = *opts;
    cbspmv_plan *best = nullptr;
    cbspmv_tune_report r;
    std::memset(&r, 0, sizeof r);
    r.ms = -1.0;
    for (int bs : {16, 32}) {
        for (int te : {0, 128}) {
            cbspmv_opts o = base;
            o.block_size = bs;
            o.tile_entries = te;
            o.kernel = 0;
            cbspmv_plan *p = nullptr;
            cbspmv_status rc = cbspmv_coo2block_gather(coo, &o, &p);
            if (!rc) rc = cbspmv_upload(p, stream);
            int k = 0, rl = 0;
            double ms = 0;
            if (!rc) rc = cbspmv_autotune_ex(p, nrhs, stream, &k, &rl, &ms);
            if (rc) {
                cbspmv_destroy(p);
                if (best) cbspmv_destroy(best);
                return rc;
            }
            ++r.tried;
            if (r.ms < 0 || ms < r.ms) {
                if (best) cbspmv_destroy(best);
                best = p;
                r.block_size = bs;
                r.tile_entries = te;
                r.kernel = k;
                r.rhs_lanes = rl;
                r.ms = ms;
            } else {
                cbspmv_destroy(p);
            }
        }
    }
    best->opts.tile_entries = r.tile_entries;
    *out = best;
    if (rep) *rep = r;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_spmv_t(cbspmv_plan *p, const void *g, void *gx, int nrhs,
                            int64_t ldg, int64_t ldgx, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (!p->has_t) return fail(CBSPMV_ERR_STATE, "plan built without want_transpose");
    return run_side(p, p->AT, g, gx, nrhs, ldg, ldgx, (cudaStream_t)stream);
}

cbspmv_status cbspmv_spmv_host(cbspmv_plan *p, const void *x_host, void *y_host,
                               int nrhs, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    cbspmv_status rc = cbspmv_upload(p, stream);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t xb = (size_t)p->host.n * nrhs * vsize(p);
    const size_t yb = (size_t)p->host.m * nrhs * vsize(p);
    if (xb > p->hx_bytes) {
        if (p->hx) cudaFree(p->hx);
        p->hx = nullptr;
        p->hx_bytes = 0;
        CB_CUDA(cudaMalloc(&p->hx, xb), "allocate x");
        p->hx_bytes = xb;
    }
    if (yb > p->hy_bytes) {
        if (p->hy) cudaFree(p->hy);
        p->hy = nullptr;
        p->hy_bytes = 0;
        CB_CUDA(cudaMalloc(&p->hy, yb), "allocate y");
        p->hy_bytes = yb;
    }
    if (xb) CB_CUDA(cudaMemcpyAsync(p->hx, x_host, xb, cudaMemcpyHostToDevice, st), "copy x");
    rc = run_side(p, p->A, p->hx, p->hy, nrhs, nrhs, nrhs, st);
    if (rc) return rc;
    if (yb) CB_CUDA(cudaMemcpyAsync(y_host, p->hy, yb, cudaMemcpyDeviceToHost, st), "copy y");
    CB_CUDA(cudaStreamSynchronize(st), "spmv_host");
    return take_device_error(p, 0, st);
}

cbspmv_status cbspmv_spmv_host_async(cbspmv_plan *p, const void *x_host, void *y_host,
                                     int nrhs, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    cbspmv_status rc = cbspmv_upload(p, stream);
    if (rc) return rc;
    HostPipe &q = p->pipe;
    const cudaStream_t user = static_cast<cudaStream_t>(stream);
    const size_t xb = (size_t)p->host.n * nrhs * vsize(p);
    const size_t yb = (size_t)p->host.m * nrhs * vsize(p);
    if (!q.comp || xb > q.xb || yb > q.yb) {  // set up, or grow for more rhs
        if (q.comp) {
            CB_CUDA(cudaStreamSynchronize(q.out), "drain host pipeline");
            CB_CUDA(cudaStreamSynchronize(q.comp), "drain host pipeline");
        }
        q.release();
        for (cudaStream_t *st : {&q.in, &q.comp, &q.out})
            CB_CUDA(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "create stream");
        for (int b = 0; b < 2; ++b) {
            CB_CUDA(cudaMalloc(&q.x[b], std::max<size_t>(16, xb)), "allocate x");
            CB_CUDA(cudaMalloc(&q.y[b], std::max<size_t>(16, yb)), "allocate y");
            for (cudaEvent_t *e : {&q.x_ready[b], &q.x_free[b], &q.y_ready[b], &q.y_free[b]})
                CB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "create event");
        }
        q.xb = std::max<size_t>(16, xb);
        q.yb = std::max<size_t>(16, yb);
    }
    const int b = (int)(q.calls & 1);
    // copy in (x_host holds the input now), after the kernel that last read
    // this buffer; not after the caller's stream, which waits for earlier
    // calls' copies out
    if (q.used[b]) CB_CUDA(cudaStreamWaitEvent(q.in, q.x_free[b], 0), "wait");
    if (xb) CB_CUDA(cudaMemcpyAsync(q.x[b], x_host, xb, cudaMemcpyHostToDevice, q.in), "copy x");
    CB_CUDA(cudaEventRecord(q.x_ready[b], q.in), "record");
    // compute, once x is in and the previous copy out of this y is done
    CB_CUDA(cudaStreamWaitEvent(q.comp, q.x_ready[b], 0), "wait");
    if (q.used[b]) CB_CUDA(cudaStreamWaitEvent(q.comp, q.y_free[b], 0), "wait");
    rc = run_side(p, p->A, q.x[b], q.y[b], nrhs, nrhs, nrhs, q.comp);
    if (rc) return rc;
    CB_CUDA(cudaEventRecord(q.x_free[b], q.comp), "record");
    CB_CUDA(cudaEventRecord(q.y_ready[b], q.comp), "record");
    // copy out; the caller's stream waits for it
    CB_CUDA(cudaStreamWaitEvent(q.out, q.y_ready[b], 0), "wait");
    if (yb) CB_CUDA(cudaMemcpyAsync(y_host, q.y[b], yb, cudaMemcpyDeviceToHost, q.out), "copy y");
    CB_CUDA(cudaEventRecord(q.y_free[b], q.out), "record");
    CB_CUDA(cudaStreamWaitEvent(user, q.y_free[b], 0), "wait");
    q.used[b] = true;
    ++q.calls;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_cb_spmv(cbspmv_plan *p, const double *x, double *y,
                             cbspmv_metrics *metrics) {
    if (!p || !x || !y) return fail(CBSPMV_ERR_INVALID, "null argument");
    if (p->opts.value_type != CBSPMV_F64)
        return fail(CBSPMV_ERR_STATE, "cbspmv_cb_spmv takes double values");
    if (metrics) *metrics = cbspmv_metrics{0.0, 0.0};
    if (p->host.nnz == 0) {  // cb-spmv-dcu.hpp:1091-1098
        for (int64_t i = 0; i < p->host.m; ++i) y[i] = 0.0;
        return CBSPMV_OK;
    }
    cbspmv_status rc = cbspmv_spmv_host(p, x, y, 1, nullptr);
    if (rc) return rc;
    // 100 warm-up and 1000 timed launches (cb-spmv-dcu.hpp:1631-1656)
    for (int i = 0; i < 100; ++i) {
        rc = run_side(p, p->A, p->hx, p->hy, 1, 1, 1, nullptr);
        if (rc) return rc;
    }
    cudaEvent_t a, b;
    CB_CUDA(cudaEventCreate(&a), "event");
    CB_CUDA(cudaEventCreate(&b), "event");
    cudaEventRecord(a, nullptr);
    for (int i = 0; i < 1000 && !rc; ++i) rc = run_side(p, p->A, p->hx, p->hy, 1, 1, 1, nullptr);
    cudaEventRecord(b, nullptr);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "timing");
    if ((rc = take_device_error(p, 0, nullptr))) return rc;
    if (metrics) {
        metrics->runtime_ms = ms / 1000.0;
        if (metrics->runtime_ms > 0)
            metrics->gflops = 2.0 * (double)p->host.nnz * 1.0e-6 / metrics->runtime_ms;
    }
    return CBSPMV_OK;
}

cbspmv_status cbspmv_grad_vals(cbspmv_plan *p, const void *g, const void *x,
                               void *gvals, int nrhs, int64_t ldg, int64_t ldx,
                               void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (cbspmv_status rc = refuse_spmv_only(p)) return rc;
    if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "plan not uploaded");
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    if (ldg == 0) ldg = nrhs;
    if (ldx == 0) ldx = nrhs;
    if (ldg < nrhs || ldx < nrhs)
        return fail(CBSPMV_ERR_INVALID, "leading dimension smaller than nrhs");
    DevSide &s = p->A;
    CB_CUDA(cb::launch_grad_vals(s.lay.f32, s.lay.nvals, s.val_row, s.val_col, g,
                                 ldg, x, ldx, nrhs, gvals, (cudaStream_t)stream),
            "grad_vals launch");
    return CBSPMV_OK;
}

cbspmv_status cbspmv_adjoint(cbspmv_plan *p, const void *g, const void *x, void *gx,
                             void *gvals, int nrhs, int64_t ldg, int64_t ldx, int64_t ldgx,
                             void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (!gx && !gvals) return fail(CBSPMV_ERR_INVALID, "neither gx nor gvals given");
    if (gx && !p->has_t) return fail(CBSPMV_ERR_STATE, "plan built without want_transpose");
    if (!gx) return cbspmv_grad_vals(p, g, x, gvals, nrhs, ldg, ldx, stream);
    if (!gvals) return cbspmv_spmv_t(p, g, gx, nrhs, ldg, ldgx, stream);
    if (cbspmv_status rc = refuse_spmv_only(p)) return rc;
    if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "plan not uploaded");
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    const int64_t lg = ldg ? ldg : nrhs, lx = ldx ? ldx : nrhs;
    if (lg < nrhs || lx < nrhs)
        return fail(CBSPMV_ERR_INVALID, "leading dimension smaller than nrhs");
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != p->device)
        return fail(CBSPMV_ERR_STATE, "plan was uploaded to another device");
    if (!p->adj) {
        CB_CUDA(cudaStreamCreateWithFlags(&p->adj, cudaStreamNonBlocking), "adjoint stream");
        CB_CUDA(cudaEventCreateWithFlags(&p->adj_fork, cudaEventDisableTiming), "adjoint event");
        CB_CUDA(cudaEventCreateWithFlags(&p->adj_join, cudaEventDisableTiming), "adjoint event");
    }
    cudaStream_t st = (cudaStream_t)stream;
    CB_CUDA(cudaEventRecord(p->adj_fork, st), "adjoint fork");
    CB_CUDA(cudaStreamWaitEvent(p->adj, p->adj_fork, 0), "adjoint fork");
    DevSide &s = p->A;
    CB_CUDA(cb::launch_grad_vals(s.lay.f32, s.lay.nvals, s.val_row, s.val_col, g, lg, x, lx,
                                 nrhs, gvals, p->adj),
            "grad_vals launch");
    const cbspmv_status rc = run_side(p, p->AT, g, gx, nrhs, lg, ldgx, st);
    // join even when A^T g failed, so no work is left unordered on `stream`
    CB_CUDA(cudaEventRecord(p->adj_join, p->adj), "adjoint join");
    CB_CUDA(cudaStreamWaitEvent(st, p->adj_join, 0), "adjoint join");
    return rc;
}

namespace {
// The fused adjoint runs on the transposed plan's row-segment stream (its
// value gradient then in stream order) once the plan is uploaded with one
// that holds values and their positions; otherwise on the transposed tiles
// (gradient in payload order).
bool fused_on_stream(const cbspmv_plan *p) {
    const DevSide &s = p->AT;
    return p->uploaded && s.d.rs.chunks && !s.d.rs.unit &&
           (int64_t)s.rs_vpos.size() == s.lay.nvals && s.lay.nvals > 0;
}
}  // namespace

cbspmv_status cbspmv_adjoint_fused(cbspmv_plan *p, const void *g, const void *x, void *gx,
                                   void *gvals_t, int nrhs, int64_t ldg, int64_t ldx,
                                   int64_t ldgx, void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (!p->has_t) return fail(CBSPMV_ERR_STATE, "plan built without want_transpose");
    if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "plan not uploaded");
    if (p->AT.lay.unit)
        return fail(CBSPMV_ERR_UNSUPPORTED,
                    "this plan stores no values (every value was 1); build it with "
                    "keep_values = 1 for a value gradient");
    if (nrhs < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    if (ldg == 0) ldg = nrhs;
    if (ldx == 0) ldx = nrhs;
    if (ldgx == 0) ldgx = nrhs;
    if (ldg < nrhs || ldx < nrhs || ldgx < nrhs)
        return fail(CBSPMV_ERR_INVALID, "leading dimension smaller than nrhs");
    DevSide &s = p->AT;
    if ((s.lay.m > 0 && (!gx || !x)) || (s.lay.n > 0 && !g) || !gvals_t)
        return fail(CBSPMV_ERR_INVALID, "null g, x, gx or gvals_t");
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != p->device) return fail(CBSPMV_ERR_STATE, "plan was uploaded to another device");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cbspmv_status rc = take_device_error(p, 1, st)) return rc;
    if (fused_on_stream(p)) {
        CB_CUDA(cb::launch_rowseg_adjoint(s.d, g, gx, nrhs, ldg, ldgx, x, ldx, gvals_t, st),
                "fused adjoint launch");
        return CBSPMV_OK;
    }
    if (cbspmv_status rc = ensure_partials(s, nrhs, vsize(p))) return rc;
    CB_CUDA(cb::launch_spmm(s.d, g, gx, nrhs, ldg, ldgx, st, gvals_t, x, ldx),
            "fused adjoint launch");
    return CBSPMV_OK;
}

int64_t cbspmv_grad_size_t(const cbspmv_plan *p) {
    if (!p || !p->has_t) return -1;
    if (fused_on_stream(p)) return (int64_t)p->AT.d.rs.nch * cb::rs_chunk_entries();
    return (int64_t)(p->AT.lay.payload.size() / vsize(p));
}

cbspmv_status cbspmv_grad_positions_t(const cbspmv_plan *p, int64_t *pos) {
    if (!p || !pos) return fail(CBSPMV_ERR_INVALID, "null argument");
    if (!p->has_t) return fail(CBSPMV_ERR_STATE, "plan built without want_transpose");
    if (cbspmv_status rc = refuse_spmv_only(p)) return rc;
    const cb::DeviceLayout &L = p->AT.lay;
    if (fused_on_stream(p)) {
        for (int64_t i = 0; i < p->host.nnz; ++i) pos[i] = p->AT.rs_vpos[L.input_slot[i]];
        return CBSPMV_OK;
    }
    const int64_t vsz = (int64_t)vsize(p);
    for (int64_t i = 0; i < p->host.nnz; ++i) pos[i] = (int64_t)L.val_off[L.input_slot[i]] / vsz;
    return CBSPMV_OK;
}

int64_t cbspmv_num_values(const cbspmv_plan *p) { return p ? p->A.lay.nvals : -1; }

cbspmv_status cbspmv_set_values(cbspmv_plan *p, const void *input_values,
                                void *stream) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (cbspmv_status rc = refuse_spmv_only(p)) return rc;
    if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "plan not uploaded");
    if (p->A.lay.unit)
        return fail(CBSPMV_ERR_UNSUPPORTED,
                    "this plan stores no values (every value was 1); build it with "
                    "keep_values = 1 to change them");
    cudaStream_t st = (cudaStream_t)stream;
    DevSide *sides[2] = {&p->A, p->has_t ? &p->AT : nullptr};
    for (DevSide *s : sides) {
        if (!s) continue;
        CB_CUDA(cb::launch_set_values(s->lay.f32, s->lay.nvals, s->vsrc_ptr, s->vsrc,
                                      s->val_off, input_values, s->payload, st),
                "set_values launch");
        CB_CUDA(cb::launch_rowseg_values(s->d, s->lay.nvals, s->val_off, st),
                "set_values launch");
        CB_CUDA(cb::launch_balanced_values(s->d, st), "set_values launch");
    }
    return CBSPMV_OK;
}

cbspmv_status cbspmv_value_coords(const cbspmv_plan *p, int32_t *row, int32_t *col,
                                  int64_t *first_input) {
    if (!p) return fail(CBSPMV_ERR_INVALID, "null plan");
    if (cbspmv_status rc = refuse_spmv_only(p)) return rc;
    const cb::DeviceLayout &L = p->A.lay;
    if (row) std::memcpy(row, L.val_row.data(), L.nvals * 4);
    if (col) std::memcpy(col, L.val_col.data(), L.nvals * 4);
    if (first_input)
        for (int64_t v = 0; v < L.nvals; ++v)
            first_input[v] = L.vsrc_ptr[v + 1] > L.vsrc_ptr[v] ? L.vsrc[L.vsrc_ptr[v]] : -1;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_input_slots(const cbspmv_plan *p, int64_t *slot) {
    if (!p || !slot) return fail(CBSPMV_ERR_INVALID, "null argument");
    if (cbspmv_status rc = refuse_spmv_only(p)) return rc;
    std::memcpy(slot, p->A.lay.input_slot.data(), p->host.nnz * sizeof(int64_t));
    return CBSPMV_OK;
}

cbspmv_status cbspmv_info_get(const cbspmv_plan *p, cbspmv_info *info) {
    if (!p || !info) return fail(CBSPMV_ERR_INVALID, "null argument");
    const cb::HostCB &g = p->host;
    cbspmv_info I;
    std::memset(&I, 0, sizeof(I));
    I.m = g.m;
    I.n = g.n;
    I.nnz = g.nnz;
    I.gb_m = g.gb_m;
    I.gb_n = g.gb_n;
    I.gb_nnzb = g.nnzb;
    I.gather_flag = g.gather_flag;
    I.direct_coo_columns = g.direct;
    I.compact_coo_indices = g.compact;
    I.load_balanced = g.balanced;
    I.unit_values = g.unit_values;
    I.super_sparse_blocks = g.super_sparse;
    I.analyzed_blocks = g.analyzed;
    I.super_sparse_ratio = g.ratio;
    I.load_stddev_before = g.sd_before;
    I.load_stddev_after = g.sd_after;
    int64_t c[6];
    block_counts(p, c);
    I.coo_blocks = c[0];
    I.csr_blocks = c[1];
    I.dense_blocks = c[2];
    I.uniform_blocks = c[3];
    I.segments = c[4];
    I.patterns = c[5];
    I.stored_values = p->A.lay.nvals;
    I.tiles = (int64_t)p->A.lay.tiles.size();
    I.split_rows = p->A.lay.split_rows;
    I.device_bytes = (int64_t)(p->A.lay.tiles.size() * sizeof(cb::TileDesc) +
                               p->A.lay.blocks.size() * sizeof(cb::BlockDesc) +
                               p->A.lay.payload.size() + p->A.lay.block_cols.size() * 4) +
                     p->A.rs_bytes + p->A.bal_bytes;
    I.algorithmic_bytes = p->A.lay.alg_bytes;
    I.rowseg_bytes = p->A.rs_bytes;
    I.scratch_bytes = (int64_t)(p->A.lay.slots * p->A.lay.bs * vsize(p) +
                                (p->A.lay.gb_m + 4) * 4);
    *info = I;
    return CBSPMV_OK;
}

namespace {
// Raw device-layout arrays, for host-side checks of the layout:
// dev_tiles (u32, 8 per tile), dev_blocks (u32, 4 per block), dev_payload
// (bytes), dev_values (stored values as double, device order).
int64_t export_device(const cb::DeviceLayout &L, const std::string &k, void *out) {
    auto raw = [&](const void *src, size_t bytes, size_t unit) -> int64_t {
        if (out && bytes) std::memcpy(out, src, bytes);
        return (int64_t)(bytes / unit);
    };
    if (k == "dev_tiles")
        return raw(L.tiles.data(), L.tiles.size() * sizeof(cb::TileDesc), 4);
    if (k == "dev_blocks")
        return raw(L.blocks.data(), L.blocks.size() * sizeof(cb::BlockDesc), 4);
    if (k == "dev_payload") return raw(L.payload.data(), L.payload.size(), 1);
    if (k == "dev_values") {
        if (out)
            for (int64_t v = 0; v < L.nvals; ++v) {
                double x;
                if (L.f32) {
                    float f;
                    std::memcpy(&f, L.payload.data() + L.val_off[v], 4);
                    x = f;
                } else {
                    std::memcpy(&x, L.payload.data() + L.val_off[v], 8);
                }
                ((double *)out)[v] = x;
            }
        return L.nvals;
    }
    // the row-segment stream built for W resident warps: "rs_<field>:<W>"
    if (k.rfind("rs_", 0) == 0) {
        const size_t colon = k.find(':');
        if (colon == std::string::npos) return -1;
        const int64_t warps = std::atoll(k.c_str() + colon + 1);
        const std::string f = k.substr(3, colon - 3);
        cb::RowSegHost R;
        if (warps <= 0 || !cb::build_rowseg(L, warps, R).empty()) return -1;
        const int32_t sizes[6] = {R.nch, R.M, R.nseg, R.nord, R.G, R.W};
        if (f == "sizes") return raw(sizes, sizeof sizes, 4);
        if (f == "chunks") return raw(R.chunks.data(), R.chunks.size(), 1);
        if (f == "meta") return raw(R.meta.data(), R.meta.size() * 4, 4);
        if (f == "spans") return raw(R.spans.data(), R.spans.size() * 4, 4);
        if (f == "rowmap") return raw(R.rowmap.data(), R.rowmap.size() * 4, 4);
        if (f == "empty") return raw(R.empty.data(), R.empty.size() * 4, 4);
        if (f == "vpos") return raw(R.vpos.data(), R.vpos.size() * 4, 4);
        if (f == "wbase") return raw(R.wbase.data(), R.wbase.size() * 4, 4);
    }
    return -1;
}
}  // namespace

// An SpMV-only plan has the device layout's geometry and payload but no host
// block arrays and no per-value arrays: those names give -1.
bool exportable(const cbspmv_plan *p, const std::string &k) {
    if (!p->spmv_only) return true;
    const bool ok = k == "dev_tiles" || k == "dev_blocks" || k == "dev_payload" ||
                    k.rfind("rs_", 0) == 0;
    if (!ok) fail(CBSPMV_ERR_STATE, "plan loaded from an SpMV-only plan file: no " + k);
    return ok;
}

namespace {
// The balanced schedule's stream of A (plans built with row_owned = 0):
// bal_rows, bal_cols (uint32, 4 per quad), bal_vals (the value type) and
// bal_gstart (int64, per group its first quad, then the quad count).
int64_t export_balanced(const cbspmv_plan *p, const std::string &k, void *out) {
    cb::BalancedHost B;
    if (!cb::build_balanced(p->A.lay, p->host, B).empty()) return -1;
    auto raw = [&](const void *src, size_t bytes, size_t unit) -> int64_t {
        if (out && bytes) std::memcpy(out, src, bytes);
        return (int64_t)(bytes / unit);
    };
    if (k == "bal_rows") return raw(B.rows.data(), B.rows.size() * 4, 4);
    if (k == "bal_cols") return raw(B.cols.data(), B.cols.size() * 4, 4);
    if (k == "bal_vals") return raw(B.vals.data(), B.vals.size(), B.f32 ? 4 : 8);
    if (k == "bal_gstart") return raw(B.gstart.data(), B.gstart.size() * 8, 8);
    return -1;
}
}  // namespace

int64_t cbspmv_export(const cbspmv_plan *p, const char *name, void *out) {
    if (!p || !name) return -1;
    const std::string k(name);
    if (k.rfind("bal_", 0) == 0) return p->spmv_only ? -1 : export_balanced(p, k, out);
    if (!exportable(p, k)) return -1;
    if (k.rfind("dev_", 0) == 0 || k.rfind("rs_", 0) == 0)
        return export_device(p->A.lay, k, out);
    return cb::export_array(p->host, k, out);
}

int64_t cbspmv_export_t(const cbspmv_plan *p, const char *name, void *out) {
    if (!p || !name || !p->has_t) return -1;
    const std::string k(name);
    if (!exportable(p, k)) return -1;
    if (k.rfind("dev_", 0) == 0 || k.rfind("rs_", 0) == 0)
        return export_device(p->AT.lay, k, out);
    return cb::export_array(p->host_t, k, out);
}

void cbspmv_export_scalars(const cbspmv_plan *p, int transpose, int64_t *out12,
                           double *out3) {
    const cb::HostCB &g = transpose ? p->host_t : p->host;
    const int64_t s[12] = {g.m, g.n, g.nnz, g.gb_m, g.gb_n, g.nnzb,
                           g.gather_flag, g.direct, g.compact, g.super_sparse,
                           g.analyzed, g.balanced};
    std::memcpy(out12, s, sizeof(s));
    out3[0] = g.ratio;
    out3[1] = g.sd_before;
    out3[2] = g.sd_after;
}

cbspmv_status cbspmv_destroy(cbspmv_plan *p) {
    delete p;
    return CBSPMV_OK;
}

size_t cbspmv_last_error(char *buf, size_t len) {
    if (buf && len) {
        const size_t n = std::min(len - 1, g_error.size());
        std::memcpy(buf, g_error.data(), n);
        buf[n] = 0;
    }
    return g_error.size();
}

int64_t cbspmv_launch_count(void) { return cb::kernel_launches(); }

}  // extern "C"

// ---- batches ---------------------------------------------------------------

// All matrices of a batch run in one launch: their views are a device table,
// their tiles concatenated (toff) and cut into scheduling units (ustart) the
// launch's warps take from a counter.
struct cbspmv_batch {
    std::vector<cbspmv_plan *> plans;  // in the caller's order
    std::vector<cb::MatView> views;    // host copy of the device table
    int bs = 16, f32 = 0, device = -1;
    bool bound = false;
    cb::MatView *d_views = nullptr;
    int64_t *d_toff = nullptr, *d_ustart = nullptr;
    int32_t *d_uorder = nullptr;    // queue order of the units
    int64_t ntot = 0, nunits = 0;   // tiles and scheduling units
    uint32_t *d_sched = nullptr;    // 2 scheduler words (unit counter, warps out)
    uint32_t *herr = nullptr, *derr = nullptr;  // error word (host-mapped)
    uint32_t tile_cap = 16;         // shared buffer bytes: every plan's largest tile
    cudaStream_t cap[8] = {};
    cudaEvent_t ev[9] = {};
    cudaGraphExec_t exec[2] = {};
    // over the row-segment streams (every plan has one, nrhs <= 16): the
    // matrices' table, segments {matrix, first chunk, end chunk, -} in queue
    // order with their meta, scheduler words, empty rows {matrix, row}, the
    // batch's spans, counters and partial slots
    bool rs_mode = false;
    std::vector<cb::RsBatchMat> rmats;
    cb::RsBatchMat *d_rmats = nullptr;
    int4 *d_rsegs = nullptr, *d_rmeta = nullptr, *d_rspans = nullptr;
    int32_t *d_rcnt = nullptr, nrseg = 0;
    uint32_t *d_rsched = nullptr;   // 2 scheduler words (next segment, warps out)
    int2 *d_rempty = nullptr;
    void *d_rpart = nullptr;
    int64_t rwarps = 0, nrempty = 0;
    ~cbspmv_batch() {
        for (cudaGraphExec_t &g : exec)
            if (g) cudaGraphExecDestroy(g);
        for (cudaEvent_t &e : ev)
            if (e) cudaEventDestroy(e);
        for (cudaStream_t &c : cap)
            if (c) cudaStreamDestroy(c);
        for (void *p : {(void *)d_toff, (void *)d_ustart, (void *)d_uorder, (void *)d_sched,
                        (void *)d_views, (void *)d_rmats, (void *)d_rsegs, (void *)d_rmeta,
                        (void *)d_rspans, (void *)d_rsched, (void *)d_rcnt, (void *)d_rempty,
                        d_rpart})
            if (p) cudaFree(p);
        if (herr) cudaFreeHost(herr);
    }
};

namespace {

// Reports (once) that a batch launch gave up a bounded device wait, and
// resets the plans' arrival counters and the batch's scheduler words.
cbspmv_status batch_device_error(cbspmv_batch *b, cudaStream_t st) {
    if (!b->herr) return CBSPMV_OK;
    volatile uint32_t *w = b->herr;
    if (*w == 0) return CBSPMV_OK;
    *w = 0;
    for (cbspmv_plan *p : b->plans)
        if (p->A.counters)
            CB_CUDA(cudaMemsetAsync(p->A.counters, 0, (p->A.lay.gb_m + 4) * sizeof(int32_t), st),
                    "reset scratch after a device error");
    CB_CUDA(cudaMemsetAsync(b->d_sched, 0, 16, st), "reset scratch after a device error");
    return fail(CBSPMV_ERR_DEVICE,
                "a bounded device wait gave up in an earlier batch launch: its outputs are "
                "incomplete; the batch's scratch was reset");
}

cbspmv_status batch_check(cbspmv_batch *b, bool need_bound, cudaStream_t st) {
    if (!b) return fail(CBSPMV_ERR_INVALID, "null batch");
    if (need_bound && !b->bound) return fail(CBSPMV_ERR_STATE, "batch has no bound x/y arrays");
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != b->device) return fail(CBSPMV_ERR_STATE, "batch was created on another device");
    return batch_device_error(b, st);
}

cbspmv_status batch_each(cbspmv_batch *b, cudaStream_t st) {
    for (size_t k = 0; k < b->plans.size(); ++k) {
        const cb::MatView &v = b->views[k];
        cbspmv_status rc = run_side(b->plans[k], b->plans[k]->A, v.x, v.y, v.nrhs, v.ldx,
                                    v.ldy, st);
        if (rc) return rc;
    }
    return CBSPMV_OK;
}

template <typename V>
cudaError_t upload_raw(const std::vector<V> &h, V **d) {
    const size_t n = std::max<size_t>(1, h.size());
    cudaError_t e = cudaMalloc((void **)d, n * sizeof(V));
    if (e == cudaSuccess) e = cudaMemset(*d, 0, n * sizeof(V));
    if (e == cudaSuccess && !h.empty())
        e = cudaMemcpy(*d, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice);
    return e;
}

// The batch over the row-segment streams, when every plan has one and takes
// at most 16 right-hand sides: each matrix's chunks cut into segments of
// about one eighth of a resident warp's share of the work (a chunk costs its
// lanes per entry), queued by lanes per entry (most first: warps of one SM
// then mostly run one code path) and taken by the warps from a counter, so
// one launch runs every matrix and balances itself; each segment has its own
// meta and the batch its own spans.
cbspmv_status batch_rowseg_setup(cbspmv_batch *b, const int *nrhs) {
    const int count = (int)b->plans.size();
    for (int k = 0; k < count; ++k) {
        const DevSide &s = b->plans[k]->A;
        if (!s.d.rs.chunks || s.rs_cinfo.empty() || nrhs[k] > cb::kRsSlotValues)
            return CBSPMV_OK;
    }
    const int64_t W = cb::rowseg_batch_warps(b->f32);
    if (W <= 0) return CBSPMV_OK;
    std::vector<int> g(count), order(count);
    double total = 0;
    for (int k = 0; k < count; ++k) {
        g[k] = cb::rs_lanes_per_entry(b->f32, nrhs[k]);
        total += (double)b->plans[k]->A.d.rs.nch * g[k];
    }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return g[a] > g[c]; });
    const double share = std::max(1.0, total / ((double)W * 8));
    std::vector<int32_t> segs, meta, spans;
    std::vector<int2> empty;
    for (int k : order) {
        const DevSide &s = b->plans[k]->A;
        const int64_t nch = s.d.rs.nch, seg0 = (int64_t)(segs.size() / 4);
        const int64_t per = std::max<int64_t>(1, (int64_t)std::llround(share / g[k]));
        std::vector<int64_t> cuts(1, 0);
        for (int64_t c = 0; c < nch; c += per) {
            const int64_t e = std::min(nch, c + per);
            segs.insert(segs.end(), {k, (int32_t)c, (int32_t)e, 0});
            cuts.push_back(e);
        }
        cb::rowseg_cut(s.rs_cinfo, cuts, seg0, k, meta, spans);
        for (int32_t r : s.rs_empty) empty.push_back(make_int2(k, r));
    }
    const size_t nseg = segs.size() / 4, nspan = spans.size() / 4;
    const size_t vsz = b->f32 ? 4 : 8;
    cudaError_t e = upload_raw(segs, (int32_t **)&b->d_rsegs);
    if (e == cudaSuccess) e = upload_raw(meta, (int32_t **)&b->d_rmeta);
    if (e == cudaSuccess) e = upload_raw(spans, (int32_t **)&b->d_rspans);
    if (e == cudaSuccess) e = upload_raw(std::vector<uint32_t>(2, 0u), &b->d_rsched);
    if (e == cudaSuccess) e = upload_raw(std::vector<int32_t>(std::max<size_t>(1, nspan), 0),
                                         &b->d_rcnt);
    if (e == cudaSuccess) e = upload_raw(empty, &b->d_rempty);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_rpart, std::max<size_t>(1, 2 * nseg) * cb::kRsSlotValues * vsz);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_rmats, count * sizeof(cb::RsBatchMat));
    if (e != cudaSuccess) return cuda_fail(e, "allocate batch tables");
    b->rmats.assign(count, cb::RsBatchMat());
    for (int k = 0; k < count; ++k) {
        const cb::RowSegDev &r = b->plans[k]->A.d.rs;
        cb::RsBatchMat &m = b->rmats[k];
        m.chunks = r.chunks;
        m.rowmap = r.rowmap;
        m.nrhs = nrhs[k];
        m.nord = r.nord;
        m.g = g[k];
        m.unit = r.unit;
    }
    b->rwarps = W;
    b->nrseg = (int32_t)nseg;
    b->nrempty = (int64_t)empty.size();
    b->rs_mode = true;
    return CBSPMV_OK;
}

// One persistent launch over every matrix of the batch.
cbspmv_status batch_one(cbspmv_batch *b, cudaStream_t st) {
    if (b->rs_mode) {
        const cudaError_t e = cb::launch_rowseg_batch(
            b->f32, b->d_rmats, b->d_rsegs, b->d_rmeta, b->nrseg, b->d_rsched, b->rwarps,
            b->d_rempty, b->nrempty, b->d_rspans, b->d_rcnt, b->d_rpart, st);
        return e == cudaSuccess ? CBSPMV_OK : cuda_fail(e, "batch launch");
    }
    const cudaError_t e = cb::launch_batch(b->bs, b->f32, b->d_views, (int)b->plans.size(),
                                           b->d_toff, b->d_ustart, b->d_uorder, b->nunits,
                                           b->tile_cap, b->d_sched, b->derr, st);
    return e == cudaSuccess ? CBSPMV_OK : cuda_fail(e, "batch launch");
}

}  // namespace

extern "C" {

cbspmv_status cbspmv_batch_create(cbspmv_plan *const *plans, int count, const int *nrhs,
                                  cbspmv_batch **out) {
    if (!plans || !nrhs || !out || count < 1)
        return fail(CBSPMV_ERR_INVALID, "batch needs count >= 1 plans and nrhs values");
    *out = nullptr;
    int dev = -1;
    cudaGetDevice(&dev);
    for (int k = 0; k < count; ++k) {
        const cbspmv_plan *p = plans[k];
        if (!p) return fail(CBSPMV_ERR_INVALID, "null plan in batch");
        if (!p->uploaded) return fail(CBSPMV_ERR_STATE, "batch plan not uploaded");
        if (p->device != dev)
            return fail(CBSPMV_ERR_STATE, "batch plans must be uploaded to the current device");
        if (p->opts.block_size != plans[0]->opts.block_size ||
            p->opts.value_type != plans[0]->opts.value_type)
            return fail(CBSPMV_ERR_INVALID, "batch plans must share block size and value type");
        if (nrhs[k] < 1) return fail(CBSPMV_ERR_INVALID, "nrhs must be >= 1");
    }
    cbspmv_batch *b = new (std::nothrow) cbspmv_batch();
    if (!b) return fail(CBSPMV_ERR_ALLOC, "out of host memory");
    b->bs = plans[0]->opts.block_size;
    b->f32 = plans[0]->opts.value_type == CBSPMV_F32;
    b->device = dev;
    for (int k = 0; k < count; ++k) {
        cbspmv_status rc = ensure_partials(plans[k]->A, nrhs[k], vsize(plans[k]));
        if (rc) {
            delete b;
            return rc;
        }
        b->tile_cap = std::max(b->tile_cap, plans[k]->A.d.mcap);
    }
    std::vector<int64_t> toff(1, 0);
    for (int k = 0; k < count; ++k) {
        DevSide &s = plans[k]->A;
        b->plans.push_back(plans[k]);
        b->views.push_back(cb::mat_view(s.d, nullptr, nullptr, nrhs[k], nrhs[k], nrhs[k]));
        toff.push_back(toff.back() + (int64_t)s.lay.tiles.size());
    }
    b->ntot = toff.back();
    // Scheduling units by cost (a tile's entries and block values times its
    // passes over the right-hand sides): about eight per resident warp, cut
    // at block-row starts once a unit holds its share, anywhere at twice
    // that; queued by lane split, costliest first within one, so the launch
    // does not end on a long unit.
    std::vector<int64_t> cost(b->ntot);
    double total = 0;
    for (int k = 0; k < count; ++k) {
        const DevSide &s = plans[k]->A;
        const uint32_t *t8 = reinterpret_cast<const uint32_t *>(s.lay.tiles.data());
        const uint32_t *b4 = reinterpret_cast<const uint32_t *>(s.lay.blocks.data());
        for (int64_t t = 0; t < (int64_t)s.lay.tiles.size(); ++t)
            total += (double)(cost[toff[k] + t] = cb::ms_tile_cost_rhs(t8 + 8 * t, b4, nrhs[k],
                                                                       b->f32));
    }
    const double share =
        total / (double)(std::max<int64_t>(1, cb::ms_warps(b->bs, b->f32, b->tile_cap)) * 8);
    std::vector<int64_t> all;
    std::vector<double> ucost;
    std::vector<int> uclass;  // lane split of the unit's first matrix
    auto lane_class = [&](int r) {
        const int V = b->f32 ? 4 : 2, need = (std::min(r, 16) + V - 1) / V;
        return need <= 1 ? 0 : need <= 2 ? 1 : 2;
    };
    double acc = 0;
    for (int k = 0; k < count; ++k) {
        const DevSide &s = plans[k]->A;
        const uint32_t *t8 = reinterpret_cast<const uint32_t *>(s.lay.tiles.data());
        for (int64_t t = 0; t < (int64_t)s.lay.tiles.size(); ++t) {
            const uint32_t *d = t8 + 8 * t;
            const bool row_start = d[5] == 0xffffffffu || d[5] == d[6];
            // (a unit holds two tiles at least, but the last: the kernel stages
            // two tiles ahead across one unit boundary)
            const bool two = !all.empty() && toff[k] + t - all.back() >= 2;
            if (all.empty() || (two && ((acc >= share && row_start) || acc >= 2 * share))) {
                if (!all.empty()) ucost.push_back(acc);
                all.push_back(toff[k] + t);
                uclass.push_back(lane_class(nrhs[k]));
                acc = 0;
            }
            acc += (double)cost[toff[k] + t];
        }
    }
    if (!all.empty()) ucost.push_back(acc);
    b->nunits = (int64_t)all.size();
    all.push_back(b->ntot);
    std::vector<int32_t> order(b->nunits);
    std::iota(order.begin(), order.end(), 0);
    // by lane split first, so the warps on one SM mostly run the same code
    // (the instruction cache), then costliest first
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t c) {
        return uclass[a] != uclass[c] ? uclass[a] > uclass[c] : ucost[a] > ucost[c];
    });
    cudaError_t e = cudaMalloc((void **)&b->d_ustart, all.size() * sizeof(int64_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_ustart, all.data(), all.size() * sizeof(int64_t),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_toff, toff.size() * sizeof(int64_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_toff, toff.data(), toff.size() * sizeof(int64_t),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !order.empty())
        e = cudaMalloc((void **)&b->d_uorder, order.size() * sizeof(int32_t));
    if (e == cudaSuccess && !order.empty())
        e = cudaMemcpy(b->d_uorder, order.data(), order.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_sched, 16);
    if (e == cudaSuccess) e = cudaMemset(b->d_sched, 0, 16);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_views, count * sizeof(cb::MatView));
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&b->herr, 16, cudaHostAllocMapped);
    if (e == cudaSuccess) {
        std::memset(b->herr, 0, 16);
        e = cudaHostGetDevicePointer((void **)&b->derr, b->herr, 0);
    }
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "allocate batch tables");
    }
    if (cbspmv_status rc = batch_rowseg_setup(b, nrhs)) {
        delete b;
        return rc;
    }
    *out = b;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_batch_bind(cbspmv_batch *b, const void *const *x, void *const *y,
                                void *stream) {
    cbspmv_status rc = batch_check(b, false, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    if (!x || !y) return fail(CBSPMV_ERR_INVALID, "null x or y array");
    for (size_t k = 0; k < b->plans.size(); ++k) {
        const DevSide &s = b->plans[k]->A;
        if ((s.lay.m > 0 && !y[k]) || (s.lay.n > 0 && !x[k]))
            return fail(CBSPMV_ERR_INVALID, "null x or y in batch");
        cb::MatView &v = b->views[k];
        v = cb::mat_view(s.d, x[k], y[k], v.nrhs, v.nrhs, v.nrhs);
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    CB_CUDA(cudaMemcpyAsync(b->d_views, b->views.data(), b->views.size() * sizeof(cb::MatView),
                            cudaMemcpyHostToDevice, st),
            "upload batch table");
    if (b->rs_mode) {
        for (size_t k = 0; k < b->plans.size(); ++k) {
            cb::RsBatchMat &m = b->rmats[k];
            const int V = b->f32 ? 4 : 2;
            m.x = x[k];
            m.y = y[k];
            m.ldx = m.ldy = m.nrhs;
            m.xvec = m.nrhs % V == 0 && reinterpret_cast<uintptr_t>(x[k]) % 16 == 0;
            m.yvec = m.nrhs % V == 0 && reinterpret_cast<uintptr_t>(y[k]) % 16 == 0;
        }
        CB_CUDA(cudaMemcpyAsync(b->d_rmats, b->rmats.data(),
                                b->rmats.size() * sizeof(cb::RsBatchMat), cudaMemcpyHostToDevice,
                                st),
                "upload batch table");
    }
    CB_CUDA(cudaStreamSynchronize(st), "upload batch table");
    if (b->exec[1]) {  // captured with the old pointers
        cudaGraphExecDestroy(b->exec[1]);
        b->exec[1] = nullptr;
    }
    b->bound = true;
    return CBSPMV_OK;
}

cbspmv_status cbspmv_batch_run(cbspmv_batch *b, void *stream) {
    cbspmv_status rc = batch_check(b, true, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    return batch_one(b, static_cast<cudaStream_t>(stream));
}

cbspmv_status cbspmv_batch_run_each(cbspmv_batch *b, void *stream) {
    cbspmv_status rc = batch_check(b, true, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    return batch_each(b, static_cast<cudaStream_t>(stream));
}

cbspmv_status cbspmv_batch_graph_launch(cbspmv_batch *b, int per_matrix, void *stream) {
    cbspmv_status rc = batch_check(b, true, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    const int mode = per_matrix ? 1 : 0;
    if (!b->exec[mode]) {
        for (int q = 0; q < 8; ++q)
            if (!b->cap[q]) CB_CUDA(cudaStreamCreateWithFlags(&b->cap[q], cudaStreamNonBlocking),
                                    "create capture stream");
        for (int q = 0; q < 9; ++q)
            if (!b->ev[q]) CB_CUDA(cudaEventCreateWithFlags(&b->ev[q], cudaEventDisableTiming),
                                   "create capture event");
        // one eager run first: launchers configure their kernels on first use
        rc = mode ? batch_each(b, b->cap[0]) : batch_one(b, b->cap[0]);
        if (rc) return rc;
        CB_CUDA(cudaStreamSynchronize(b->cap[0]), "batch warm-up");
        CB_CUDA(cudaStreamBeginCapture(b->cap[0], cudaStreamCaptureModeRelaxed), "begin capture");
        cbspmv_status crc = CBSPMV_OK;
        if (!mode) {
            crc = batch_one(b, b->cap[0]);
        } else {  // fork into 8 branches, round-robin over the matrices, join
            cudaEventRecord(b->ev[8], b->cap[0]);
            for (int q = 1; q < 8; ++q) cudaStreamWaitEvent(b->cap[q], b->ev[8], 0);
            for (size_t k = 0; k < b->plans.size() && !crc; ++k) {
                const cb::MatView &v = b->views[k];
                crc = run_side(b->plans[k], b->plans[k]->A, v.x, v.y, v.nrhs, v.ldx, v.ldy,
                               b->cap[k % 8]);
            }
            for (int q = 1; q < 8; ++q) {
                cudaEventRecord(b->ev[q], b->cap[q]);
                cudaStreamWaitEvent(b->cap[0], b->ev[q], 0);
            }
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->cap[0], &graph);
        if (crc) {
            if (graph) cudaGraphDestroy(graph);
            return crc;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "end capture");
        const cudaError_t ie = cudaGraphInstantiate(&b->exec[mode], graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            b->exec[mode] = nullptr;
            return cuda_fail(ie, "instantiate batch graph");
        }
    }
    CB_CUDA(cudaGraphLaunch(b->exec[mode], static_cast<cudaStream_t>(stream)), "graph launch");
    return CBSPMV_OK;
}

cbspmv_status cbspmv_batch_check(cbspmv_batch *b, void *stream) {
    if (!b) return fail(CBSPMV_ERR_INVALID, "null batch");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    CB_CUDA(cudaStreamSynchronize(st), "batch check: synchronize");
    return batch_check(b, false, st);
}

cbspmv_status cbspmv_batch_destroy(cbspmv_batch *b) {
    delete b;
    return CBSPMV_OK;
}

}  // extern "C"
