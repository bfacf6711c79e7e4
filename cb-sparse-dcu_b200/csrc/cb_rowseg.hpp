// Row-segment stream: a second device layout of a plan's stored entries,
// sorted by row (power-law and other scattered matrices, where the blocks
// hold a few entries each, run fastest on it; CSR and DENSE blocks are
// expanded into entries).
//
// The stored entries, sorted by (row, column), are cut into CHUNKS of
// 32 x kRsK entries: lane l of a warp takes the kRsK consecutive entries
// l*kRsK .. l*kRsK+kRsK-1 of a chunk and adds them up in registers along its
// rows; one segmented shuffle scan per chunk joins the rows that run across
// lanes.  Each entry is one u32 index word and one value:
//
//   word = column | bit 31 when the entry starts a new non-empty row
//
// so a lane finds its rows by counting row starts (an exclusive scan of the
// lanes' counts) from the chunk's running row: no row index is stored.  A
// chunk is [u32 words in 4-word vectors | T values in 16-byte vectors],
// vector q of lane l at q*32 + l, so each warp load is one coalesced 512-byte
// access.
//
// Chunks are grouped in SEGMENTS of M consecutive chunks, about one segment
// per resident warp (equal entry counts: balanced by construction).  A row
// that crosses segment boundaries is a SPAN: each of its segments leaves a
// partial sum in a slot (2 s: the segment's first row, 2 s + 1: its last),
// and the last segment to arrive on the span's counter adds the slots in
// segment order and stores y, so results do not depend on timing.
// Each CTA also holds a WINDOW of x in shared memory: kRsWindowBytes of
// consecutive columns from wbase[b], chosen on the host to cover the most
// entries of the CTA's segments; an entry whose column lies in its CTA's
// window carries bit 30 and reads x from there (a shared-memory gather costs
// a few wavefronts per warp where 32 scattered global loads cost 32 L1 tag
// lookups).  The segments are assigned to CTAs for a grid of G CTAs fixed at
// build time, so every launch uses that grid.
// Rows are counted as ORDINALS of the non-empty rows (rowmap maps them back
// when some rows are empty; those rows are listed in `empty` and zeroed).
// The entry count is padded to whole chunks with entries of value 0 on
// column 0 that start one extra ordinal (nord), whose sum is never stored.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "cb_layout.hpp"

namespace cb {

constexpr int kRsK = 4;            // entries per lane per chunk
constexpr int kRsWarps = 32;       // warps per CTA (one CTA per SM)
constexpr int kRsBatchWarps = 24;  // the batch kernel's (more registers per thread)
constexpr int kRsGvWarps = 16;     // the fused adjoint's (its gradient's registers)
constexpr uint32_t kRsStart = 1u << 31;   // word: the entry starts a row
constexpr uint32_t kRsWin = 1u << 30;    // word: x[column] is in the CTA's window
constexpr uint32_t kRsColMask = (1u << 30) - 1;
constexpr int64_t kRsWindowBytes = int64_t(128) << 10;
constexpr int64_t kRsMaxCols = int64_t(1) << 30;

inline int rs_chunk_entries() { return 32 * kRsK; }
// unit-valued layouts (every stored value 1) keep no values: words only
inline int64_t rs_chunk_bytes(int f32, int unit = 0) {
    return 32 * kRsK * (4 + (unit ? 0 : f32 ? 4 : 8));
}

// Byte offset, inside the chunk buffer, of the value of stream entry e.
inline int64_t rs_value_offset(int64_t e, int f32) {
    const int64_t C = 32 * kRsK, c = e / C, i = e % C, l = i / kRsK, j = i % kRsK;
    const int64_t vsz = f32 ? 4 : 8, nv = 16 / vsz;  // values per 16-byte vector
    const int64_t pos = (j / nv) * 32 * nv + l * nv + j % nv;
    return c * rs_chunk_bytes(f32) + 4 * C + pos * vsz;
}

struct RowSegHost {
    int f32 = 0;
    int unit = 0;           // no values in the chunks (every stored value is 1)
    int64_t m = 0, n = 0;
    int32_t nch = 0;        // chunks
    int32_t M = 0;          // chunks per segment
    int32_t nseg = 0;
    int32_t nord = 0;       // non-empty rows
    int32_t G = 0;          // CTAs of every launch
    int32_t W = 0;          // window length in values
    std::vector<int32_t> wbase;    // per CTA: first column of its window
    // per chunk: ordinal running before its first entry, its first entry
    // starts a row, row starts in it, ordinal of its last entry (what any
    // other segmentation needs: a batch cuts its own)
    std::vector<int32_t> cinfo;
    std::vector<uint8_t> chunks;
    std::vector<int32_t> meta;     // per segment: ord0, starts_row, head span, tail span
    std::vector<int32_t> spans;    // per span: first segment, last segment, ordinal, 0
    std::vector<int32_t> rowmap;   // ordinal -> row (empty when every row is non-empty)
    std::vector<int32_t> empty;    // rows with no stored entry
    std::vector<int32_t> vpos;     // per stored value (device order): its stream entry,
                                   // or empty without per-value offsets
    int64_t alg_bytes = 0;
};

// Whether the layout takes the row-segment stream: stored entries, columns
// below 2^30, rows below 2^31 (CSR and DENSE blocks are expanded into
// entries).  rowseg_all_coo: every block is a COO block (the automatic choice
// for one right-hand side then takes the stream; otherwise the tile kernels,
// which read CSR/DENSE blocks with fewer index bytes).
bool rowseg_applies(const DeviceLayout &L);
bool rowseg_all_coo(const DeviceLayout &L);

// Segment meta and spans of the segmentation `cuts` (chunk boundaries,
// increasing, cuts.front() == 0, cuts.back() == nch) of one stream from its
// chunk summaries: per segment {ordinal before, starts a row, head span, tail
// span} appended to meta (span ids offset by the spans already there), per
// span {first segment, last segment, ordinal, tag} appended to spans
// (segment ids offset by seg0).
void rowseg_cut(const std::vector<int32_t> &cinfo, const std::vector<int64_t> &cuts,
                int64_t seg0, int32_t tag, std::vector<int32_t> &meta,
                std::vector<int32_t> &spans);

// Builds the stream from the tiles' COO sections (row, column and value of
// every entry) for `warps` resident warps (G = warps / kRsWarps CTAs); vpos only when the layout has its
// per-value offsets (val_off).  Every plan of one matrix and value type gets
// the same stream, so the same sums.  Returns "" or an error.
std::string build_rowseg(const DeviceLayout &L, int64_t warps, RowSegHost &R);

// The balanced (non-row-owned) schedule of a plan built with row_owned = 0:
// the stored entries in the plan's block order -- the reference's balanced
// order (the builder's permutation, coo2block.h:382-498) when it balanced
// (nnz >= 10000), else the build order -- sorted by row within a block, grouped
// as the reference groups blocks (waves_per_block blocks per group, its CTA)
// and padded to quads of 4 entries with skip entries (row kBalSkip).  A warp
// takes whole groups and adds each run of one row into y with an atomic
// (the reference's accumulate_output without CB_ROW_OWNED,
// cb-spmv-dcu.hpp:149-157), so the sums' order is not fixed.
constexpr uint32_t kBalSkip = 0xffffffffu;
struct BalancedHost {
    int f32 = 0;
    int64_t nquads = 0;
    std::vector<uint32_t> rows, cols;  // 4 per quad
    std::vector<uint8_t> vals;         // 4 values per quad
    std::vector<int64_t> eoff;         // per entry: its value's payload offset (-1: skip)
    std::vector<int64_t> gstart;       // per group: first quad, then the quad count
};
// "" or an error (no permutation, unit values: the plan keeps the row-owned
// kernels).
std::string build_balanced(const DeviceLayout &L, const HostCB &g, BalancedHost &B);

}  // namespace cb
