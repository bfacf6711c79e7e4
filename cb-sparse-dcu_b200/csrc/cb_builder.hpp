// Host CB builder: the structure the reference calls GLOBAL_BLOCK
// (cb-spmv-dcu/src/format.h:62-104), built from a row-sorted COO with the
// reference's rules (coo2block.h:628-670) but parallel and map-free.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace cb {

enum : int { kCOO = 0, kCSR = 1, kDENSE = 3, kTypeMask = 0x7f, kUniform = 0x80 };

struct BuildOpts {
    int bs = 16;
    int row_owned = 1;
    int waves = 4;
    int dense_sixteenths = 15;
    int force_coo64 = 0;
};

// Everything the reference keeps in GLOBAL_BLOCK, with the per-block payload
// maps (data_per_coo_blk_comp / csr / dense, keyed by pre-balance block id)
// flattened: block o's payload is pay_u32[u32_off[o] .. u32_off[o+1]) and
// pay_f64[f64_off[o] .. f64_off[o+1]) in the reference's units (COO: idx;
// CSR: row_ptr then col_idx; DENSE: no u32, bs*bs values row-major).
struct HostCB {
    BuildOpts o;
    int64_t m = 0, n = 0, nnz = 0, gb_m = 0, gb_n = 0, nnzb = 0;
    int gather_flag = 0, direct = 0, compact = 0, balanced = 0;
    int64_t super_sparse = 0, analyzed = 0;
    double ratio = 0, sd_before = 0, sd_after = 0;

    std::vector<int32_t> gb_row, gb_col, nnz_blk, type_blk, gb_row_ptr;
    std::vector<int32_t> seg_rows, seg_begin, seg_end, seg_direct, seg_uniform,
        row_uniform;
    std::vector<int32_t> flat_row_ptr, flat_col, pat_row_ptr, pat_col,
        pat_out_ptr, pat_out_rows;
    std::vector<int32_t> block_cols_offset, block_cols;
    std::vector<int32_t> bidx_origin, bidx_end, bidx_nnz;

    int64_t nnzb_orig = 0;  // blocks before balance padding
    std::vector<int64_t> u32_off, f64_off;  // per original block, size+1
    std::vector<uint32_t> pay_u32;
    std::vector<double> pay_f64;
    // input nonzeros summed into each stored value, in summation order:
    // src[src_ptr[v] .. src_ptr[v+1]) for value v of pay_f64
    std::vector<int64_t> src_ptr;
    std::vector<int32_t> src;

    int unit_values = 0;  // cb-spmv-dcu.hpp:1105-1127
};

// Returns "" on success, else an error message; *code gets a cbspmv_status.
std::string build_cb(const BuildOpts &o, int64_t m, int64_t n, int64_t nnz,
                     const int32_t *row, const int32_t *col, const double *val,
                     HostCB &out, int *code);

// Array export under the oracle's dump names (cbdump_array semantics).
int64_t export_array(const HostCB &g, const std::string &name, void *out);

}  // namespace cb
