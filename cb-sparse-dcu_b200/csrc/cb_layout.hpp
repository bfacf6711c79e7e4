// Device layout of a built CB structure: what the sm_100a kernels read.
//
// The reference packs one buffer with per-block pointers (cb-spmv-dcu.hpp:
// 1130-1348).  Here the unit of work is a TILE: up to kTileBlocks consecutive
// blocks of ONE block row (and at most kTileEntries COO entries), processed by
// one warp.  A tile's payload is contiguous and 16-byte aligned:
//
//   [COO section]  u32 idx[E] | pad16 | T val[E] | pad16
//                  idx = (row_in_block << 27) | original column (resolved
//                  through the gather list at build time, so the kernel does
//                  no dependent lookup for COO entries)
//   [per CSR block] IdxT row_ptr[bs+1] | IdxT col[k] | pad16 | T val[k] | pad16
//                  (IdxT = u8 for bs=16, u16 for bs=32; col is block-local
//                  in the block's column space: gathered when gather_flag)
//   [per DENSE block] T val[bs*bs] row-major | pad16
//
// Block rows longer than one tile are split; each of their tiles writes bs
// partial sums to a scratch slot and the last tile to arrive (a per-block-row
// counter) adds the partials in tile order and stores y.  Rows of empty block
// rows are covered by tiles with no blocks, which store zeros.
#pragma once

#include <cstdint>
#include <vector>

#include "cb_builder.hpp"

namespace cb {

constexpr int kTileBlocks = 32;
// Tile payload cap in bytes, [bs 16, bs 32][f32, f64]: at least one block of
// the largest kind (bs 32 FP64 CSR: 9.7 KB) and a whole COO section of 512
// entries.
constexpr int64_t kTileBytes[2][2] = {{4096, 6144}, {8192, 12288}};
constexpr int kTileEntries = 512;        // tile entry cap (the direct kernel's default)
constexpr int kTileEntriesStream = 256;  // the streaming kernel's default
constexpr int kColBits = 27;  // COO idx: column in bits 0..26
constexpr int64_t kMaxCols = int64_t(1) << kColBits;

// Position of the e-th entry (in (row, column) order) of a tile's COO
// section of E entries.  The section is cut into 32 lane slices of
// consecutive entries -- K = ceil(E / 32) entries for the first
// q = E - 32 (K - 1) lanes, K - 1 for the rest -- and entry j of lane l's
// slice is stored at position 32 j + l.  A warp that reads positions
// 32 j + lane (j = 0, 1, ...; valid while below E) is coalesced and gives
// each lane its slice in order; the positions fill [0, E) exactly.
inline int64_t coo_slice_pos(int64_t e, int64_t E) {
    const int64_t K = (E + 31) / 32, q = E - 32 * (K - 1);
    const int64_t l = e < q * K ? e / K : q + (e - q * K) / (K - 1);
    const int64_t j = e < q * K ? e % K : (e - q * K) % (K - 1);
    return 32 * j + l;
}

// 8 x u32 per tile
struct TileDesc {
    uint32_t block_begin;  // first block (device order)
    uint32_t block_row;
    uint32_t counts;       // nblocks | ncoo_blocks << 8 | nxt << 16
    uint32_t payload16;    // payload offset in 16-byte units
    uint32_t coo_entries;  // E
    uint32_t slot;         // partial slot, 0xffffffff when the row is whole
    uint32_t first_slot;   // first slot of this block row
    uint32_t row_tiles;    // tiles of this block row
};

// 4 x u32 per block (device order: within a tile COO blocks first)
struct BlockDesc {
    uint32_t off;    // COO: first entry in the tile; else byte offset in tile
    uint32_t meta;   // type | uniform<<2 | nnz<<3 | valid_cols<<14 | steps<<20
    uint32_t xbase;  // gather: index of first gathered column in block_cols;
                     // otherwise first column (gb_col * bs)
    uint32_t gb_col;
};

inline uint32_t meta_type(uint32_t m) { return m & 3u; }
inline uint32_t meta_nnz(uint32_t m) { return (m >> 3) & 2047u; }

struct DeviceLayout {
    int bs = 16;
    int f32 = 0;  // value type of the payload
    int unit = 0;  // every value is 1: no value arrays, DENSE blocks as bitmasks
    int gather = 0;
    int64_t m = 0, n = 0, gb_m = 0;
    std::vector<TileDesc> tiles;
    std::vector<BlockDesc> blocks;
    std::vector<uint8_t> payload;
    std::vector<int32_t> block_cols;  // only when gather and CSR/DENSE exist
    int64_t slots = 0;                // partial slots (tiles of split rows)
    int64_t split_rows = 0;
    int max_row_tiles = 0;
    int64_t max_entries = 0;          // largest COO section (entries) of a tile
    int64_t max_tile_bytes = 0;       // largest tile payload (bytes)
    double coo_share = 1.0;           // share of stored entries in COO blocks
    // stored values in device order
    int64_t nvals = 0;
    std::vector<uint64_t> val_off;   // byte offset of each value in payload
    std::vector<int32_t> val_row, val_col;
    std::vector<int64_t> vsrc_ptr;   // input nonzeros of each value, in the
    std::vector<int32_t> vsrc;       // builder's summation order
    std::vector<int64_t> input_slot; // per input nonzero: its value
    // algorithmic bytes of one launch (nrhs = 1), padding excluded
    int64_t alg_bytes = 0;
};

// Returns "" or an error; *code receives a cbspmv_status.
// kernel: 0 auto, 1 streaming, 2 direct -- the default tile size follows the
// kernel family (256 COO entries for the streaming kernel, 512 otherwise; the
// automatic choice is streaming when most stored entries are in COO blocks).
// unit = 1: when every stored value is 1 (g.unit_values), store no values and
// DENSE blocks as bs*bs-bit masks (the reference's UNIT_VALUES,
// cb-spmv-dcu.hpp:1105-1127).
std::string build_layout(const HostCB &g, int f32, int tile_entries, int kernel, int unit,
                         DeviceLayout &L, int *code);

// Cost-balanced contiguous split of the tiles over `warps` warps (the
// streaming kernel's load balance): part[w] .. part[w+1] are warp w's tiles.
std::vector<uint32_t> partition_tiles(const DeviceLayout &L, int64_t warps);

}  // namespace cb
