// Test infrastructure: a thin extern "C" driver around the REFERENCE's own host
// code, compiled straight from its headers (cb-spmv-dcu/src/coo2block.h,
// format.h, macros.h, utils.h) by oracle/Makefile into oracle/_ref/.  It is the
// pin for the oracle restatement (oracle/cb_oracle.cpp) and the reference arm
// of the benchmark (its CPU SpMV, cb-spmv-dcu/src/utils.h:85-136).
//
// Block size, row ownership and waves per workgroup are compile-time macros in
// the reference (macros.h:38-97, Makefile:4-7), so the Makefile builds one
// shared object per configuration.  No reference source is copied here; the
// headers are included from where they lie.
#include "coo2block.h"
#include "utils.h"

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct RefHandle {
    GLOBAL_BLOCK gb;
    // payload in final block order, flattened (see oracle/cb_dump.h)
    std::vector<uint32_t> pay_u32;
    std::vector<double> pay_f64;
    std::vector<int64_t> pay_u32_off, pay_f64_off;
    std::vector<int32_t> bidx_origin, bidx_end, bidx_nnz;
    std::vector<int32_t> type_i32, seg_direct_i32, seg_uniform_i32,
        row_uniform_i32;
    RefHandle(int m, int n, int nnz) : gb(m, n, nnz) {}
};

void flatten(RefHandle &h) {
    const GLOBAL_BLOCK &g = h.gb;
    const int nb = g.gb_nnzb;
    h.pay_u32_off.assign(nb + 1, 0);
    h.pay_f64_off.assign(nb + 1, 0);
    for (int i = 0; i < nb; ++i) {
        h.pay_u32_off[i] = (int64_t)h.pay_u32.size();
        h.pay_f64_off[i] = (int64_t)h.pay_f64.size();
        if (g.nnz_per_blk[i] <= 0) continue;
        const int old = g.block_idx_array[i].origin_idx;
        const int type = g.type_per_blk[i] & BLOCK_TYPE_MASK;
        if (type == COO) {
            const COO_BLOCK_COMP &b = g.data_per_coo_blk_comp.at(old);
            for (auto v : b.idx) h.pay_u32.push_back((uint32_t)v);
            for (auto v : b.val) h.pay_f64.push_back(v);
        } else if (type == CSR) {
            const CSR_BLOCK &b = g.data_per_csr_blk.at(old);
            for (auto v : b.row_ptr) h.pay_u32.push_back((uint32_t)v);
            for (auto v : b.col_idx) h.pay_u32.push_back((uint32_t)v);
            for (auto v : b.val) h.pay_f64.push_back(v);
        } else if (type == DENSE) {
            const DENSE_BLOCK &b = g.data_per_dense_blk.at(old);
            for (auto v : b.val) h.pay_f64.push_back(v);
        }
    }
    h.pay_u32_off[nb] = (int64_t)h.pay_u32.size();
    h.pay_f64_off[nb] = (int64_t)h.pay_f64.size();
    for (const BLOCK_IDX &b : g.block_idx_array) {
        h.bidx_origin.push_back(b.origin_idx);
        h.bidx_end.push_back(b.end_idx);
        h.bidx_nnz.push_back(b.blk_nnz);
    }
    for (auto t : g.type_per_blk) h.type_i32.push_back(t);
    for (auto t : g.segment_direct) h.seg_direct_i32.push_back(t);
    for (auto t : g.segment_uniform) h.seg_uniform_i32.push_back(t);
    for (auto t : g.block_row_uniform) h.row_uniform_i32.push_back(t);
}

template <class T>
int64_t put(const std::vector<T> &v, void *out) {
    if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(T));
    return (int64_t)v.size();
}

}  // namespace

extern "C" {

int cbdump_block_size(void) { return BLOCK_SIZE; }
int cbdump_row_owned(void) { return CB_ROW_OWNED; }
int cbdump_waves_per_block(void) { return WARP_PER_BLOCK; }

// Runs the reference's coo2block_gather (coo2block.h:628) on a row-sorted COO.
void *cbdump_build(int m, int n, int nnz, const int *row, const int *col,
                   const double *val) {
    RefHandle *h = new RefHandle(m, n, nnz);
    coo2block_gather(row, col, val, h->gb);
    flatten(*h);
    return h;
}

void cbdump_free(void *handle) { delete static_cast<RefHandle *>(handle); }

// Scalars: [m, n, nnz, gb_m, gb_n, gb_nnzb, gather_flag, direct_coo_columns,
// compact_coo_indices, super_sparse_blocks, analyzed_blocks, load_balanced]
void cbdump_scalars(void *handle, int64_t *out12, double *out3) {
    const GLOBAL_BLOCK &g = static_cast<RefHandle *>(handle)->gb;
    const int64_t s[12] = {g.mtx_m, g.mtx_n, g.mtx_nnz, g.gb_m, g.gb_n,
                           g.gb_nnzb, g.gather_flag, g.direct_coo_columns,
                           g.compact_coo_indices, g.super_sparse_blocks,
                           g.analyzed_blocks, g.load_balanced};
    std::memcpy(out12, s, sizeof(s));
    out3[0] = g.super_sparse_ratio;
    out3[1] = g.load_stddev_before;
    out3[2] = g.load_stddev_after;
}

// Copies the named array into out (if non-null) and returns its length.
// int32 arrays unless noted: pay_u32 (uint32), pay_f64 (double),
// pay_u32_off / pay_f64_off (int64).  Unknown name: -1.
int64_t cbdump_array(void *handle, const char *name, void *out) {
    RefHandle &h = *static_cast<RefHandle *>(handle);
    const GLOBAL_BLOCK &g = h.gb;
    const std::string k(name);
    if (k == "gb_row_idx") return put(g.gb_row_idx, out);
    if (k == "gb_col_idx") return put(g.gb_col_idx, out);
    if (k == "gb_row_ptr") return put(g.gb_row_ptr, out);
    if (k == "nnz_per_blk") return put(g.nnz_per_blk, out);
    if (k == "type_per_blk") return put(h.type_i32, out);
    if (k == "segment_rows") return put(g.segment_rows, out);
    if (k == "segment_begin") return put(g.segment_begin, out);
    if (k == "segment_end") return put(g.segment_end, out);
    if (k == "segment_direct") return put(h.seg_direct_i32, out);
    if (k == "segment_uniform") return put(h.seg_uniform_i32, out);
    if (k == "block_row_uniform") return put(h.row_uniform_i32, out);
    if (k == "flat_row_ptr") return put(g.flat_row_ptr, out);
    if (k == "flat_col_idx") return put(g.flat_col_idx, out);
    if (k == "pattern_row_ptr") return put(g.pattern_row_ptr, out);
    if (k == "pattern_col_idx") return put(g.pattern_col_idx, out);
    if (k == "pattern_output_ptr") return put(g.pattern_output_ptr, out);
    if (k == "pattern_output_rows") return put(g.pattern_output_rows, out);
    if (k == "block_cols_offset") return put(g.block_cols_offset, out);
    if (k == "block_cols") return put(g.block_cols, out);
    if (k == "bidx_origin") return put(h.bidx_origin, out);
    if (k == "bidx_end") return put(h.bidx_end, out);
    if (k == "bidx_nnz") return put(h.bidx_nnz, out);
    if (k == "pay_u32") return put(h.pay_u32, out);
    if (k == "pay_f64") return put(h.pay_f64, out);
    if (k == "pay_u32_off") return put(h.pay_u32_off, out);
    if (k == "pay_f64_off") return put(h.pay_f64_off, out);
    return -1;
}

// ---- the reference's CPU SpMV (utils.h:85-136), for timing and checking ----
struct RefSpmv {
    std::vector<int> row, col;
    std::vector<ValType> val, x, y;
};

void *cbref_spmv_prepare(int m, int n, int64_t nnz, const int *row,
                         const int *col, const double *val, const double *x) {
    RefSpmv *s = new RefSpmv;
    s->row.assign(row, row + nnz);
    s->col.assign(col, col + nnz);
    s->val.assign(val, val + nnz);
    s->x.assign(x, x + n);
    s->y.assign(m, 0.0);
    return s;
}

void cbref_spmv_set_y(void *ctx, const double *y) {
    RefSpmv *s = static_cast<RefSpmv *>(ctx);
    std::memcpy(s->y.data(), y, s->y.size() * sizeof(double));
}

// One call of check_results_consistency: recomputes y serially from the COO
// and compares it against the stored y (abs 1e-3 + rel 1e-4).  Returns 1 on
// PASS.  This is the whole CPU implementation the reference ships.
int cbref_spmv_check(void *ctx) {
    RefSpmv *s = static_cast<RefSpmv *>(ctx);
    return check_results_consistency(s->row, s->col, s->val, s->x, s->y) ? 1
                                                                         : 0;
}

void cbref_spmv_free(void *ctx) { delete static_cast<RefSpmv *>(ctx); }

}  // extern "C"
