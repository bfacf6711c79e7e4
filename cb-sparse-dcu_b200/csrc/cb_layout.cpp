// Device layout construction (see cb_layout.hpp).  Decodes every block of the
// reference-encoded structure (the four COO index encodings of
// coo2block.h:232-248, CSR row_ptr/col_idx, dense images) and re-packs it
// tile by tile.  Parallel over block rows: a first pass sizes every block
// row's tiles, a second pass writes them at their prefix-sum offsets.
#include "cb_layout.hpp"

#include <omp.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <string>

#include "cbspmv.h"

namespace cb {
namespace {

inline int64_t a16(int64_t x) { return (x + 15) & ~int64_t(15); }

struct Ctx {
    const HostCB &g;
    int bs, bits, vsz, isz, emax, max_xt;
    int unit = 0;       // values all 1: no value arrays, DENSE blocks as bitmasks
    int64_t max_bytes;  // tile payload cap (a larger single block is a tile alone)
    std::vector<int64_t> rowptr;  // device block order grouped by block row
    std::vector<int64_t> order;   // final block indices
    explicit Ctx(const HostCB &h) : g(h) {}

    int32_t origin(int64_t i) const { return g.bidx_origin[i]; }
    int type(int64_t i) const { return g.type_blk[i] & kTypeMask; }
    int64_t k(int64_t i) const { return g.nnz_blk[i]; }
    bool is_coo(int64_t i) const { return type(i) == kCOO; }
    int64_t coo_bytes(int64_t E) const { return a16(E * 4) + (unit ? 0 : a16(E * vsz)); }
    int64_t payload_bytes(int64_t i) const {
        const int64_t kk = k(i);
        if (type(i) == kCSR) return a16((bs + 1 + kk) * isz) + (unit ? 0 : a16(kk * vsz));
        return unit ? (int64_t)bs * bs / 8 : (int64_t)bs * bs * vsz;  // dense
    }
    int64_t alg_payload(int64_t i) const {
        const int64_t kk = k(i);
        if (type(i) == kCOO) return kk * (4 + (unit ? 0 : vsz));
        if (type(i) == kCSR) return (bs + 1 + kk) * isz + (unit ? 0 : kk * vsz);
        return unit ? (int64_t)bs * bs / 8 : (int64_t)bs * bs * vsz;
    }
    int64_t nvals(int64_t i) const {
        return type(i) == kDENSE ? (int64_t)bs * bs : k(i);
    }
    int64_t valid_cols(int64_t i) const {
        const int64_t R = g.gb_row[i], c0 = (int64_t)g.gb_col[i] * bs;
        const int64_t width = g.gather_flag
            ? g.block_cols_offset[R + 1] - g.block_cols_offset[R]
            : g.n;
        return std::max<int64_t>(0, std::min<int64_t>(bs, width - c0));
    }
    int64_t resolve(int64_t i, int64_t local) const {
        const int64_t R = g.gb_row[i], c = (int64_t)g.gb_col[i] * bs + local;
        return g.gather_flag ? g.block_cols[g.block_cols_offset[R] + c] : c;
    }
};

// Greedy split of one block row's blocks (device order [b0, b1)) into tiles.
// fn(tile_begin, tile_end) for each tile, in order; COO blocks first inside.
// A tile also ends before its payload (COO section plus CSR/DENSE payloads)
// would pass max_bytes, so a tile fits the multi-right-hand-side kernel's
// shared-memory buffer.
template <class Fn>
void split_row(const Ctx &c, int64_t b0, int64_t b1, Fn fn) {
    int64_t s = b0, nb = 0, e = 0, nxt = 0, xbytes = 0;
    auto bytes = [&](int64_t ee, int64_t xb) { return c.coo_bytes(ee) + xb; };
    for (int64_t p = b0; p < b1; ++p) {
        const int64_t i = c.order[p];
        const bool coo = c.is_coo(i);
        const int64_t e2 = coo ? e + c.k(i) : e;
        const int64_t x2 = coo ? xbytes : xbytes + c.payload_bytes(i);
        const bool full = nb == kTileBlocks || (coo && e2 > c.emax) ||
                          (!coo && nxt == c.max_xt) ||
                          (nb > 0 && bytes(e2, x2) > c.max_bytes);
        if (full) {
            fn(s, p);
            s = p;
            nb = e = nxt = xbytes = 0;
        }
        ++nb;
        if (coo) {
            e += c.k(i);
        } else {
            ++nxt;
            xbytes += c.payload_bytes(i);
        }
    }
    fn(s, b1);  // also the single empty tile of an empty block row
}

struct RowTotals {
    int64_t tiles = 0, blocks = 0, bytes = 0, vals = 0, alg = 0, bcols = 0;
    int64_t xblocks = 0;  // CSR and DENSE blocks (the kernels read their descriptors)
};

}  // namespace

std::string build_layout(const HostCB &g, int f32, int tile_entries, int kernel, int unit,
                         DeviceLayout &L, int *code) {
    *code = CBSPMV_ERR_UNSUPPORTED;
    if (g.n > kMaxCols)
        return "the device layout stores columns in 27 bits (n <= 2^27)";
    if ((int64_t)g.nnzb > INT32_MAX) return "too many blocks";
    *code = CBSPMV_OK;
    Ctx c(g);
    c.bs = g.o.bs;
    c.bits = c.bs == 16 ? 4 : 5;
    c.vsz = f32 ? 4 : 8;
    c.unit = unit && g.unit_values ? 1 : 0;
    c.isz = c.bs == 16 ? 1 : 2;
    int64_t auto_emax = kTileEntries;
    if (kernel != 2) {
        int64_t coo_e = 0, all_e = 0;
        for (int64_t i = 0; i < g.nnzb; ++i) {
            if (g.nnz_blk[i] <= 0) continue;
            all_e += g.nnz_blk[i];
            if ((g.type_blk[i] & kTypeMask) == kCOO) coo_e += g.nnz_blk[i];
        }
        if (kernel == 1 || 2 * coo_e >= all_e) auto_emax = kTileEntriesStream;
    }
    c.emax = tile_entries > 0 ? std::max(64, std::min(tile_entries, kTileEntries))
                              : (int)auto_emax;
    // the streaming kernel holds a whole tile's entries in registers
    if (auto_emax == kTileEntriesStream) c.emax = std::min(c.emax, kTileEntriesStream);
    c.max_xt = c.bs == 16 ? 16 : 8;
    c.max_bytes = kTileBytes[c.bs == 16 ? 0 : 1][f32 ? 0 : 1];
    const int bs = c.bs, vsz = c.vsz, isz = c.isz;
    const int64_t gb_m = g.gb_m;

    // group real blocks by block row, keeping final order inside a row
    c.rowptr.assign(gb_m + 1, 0);
    for (int64_t i = 0; i < g.nnzb; ++i)
        if (g.nnz_blk[i] > 0 && g.gb_row[i] >= 0) c.rowptr[g.gb_row[i] + 1]++;
    for (int64_t R = 0; R < gb_m; ++R) c.rowptr[R + 1] += c.rowptr[R];
    c.order.resize(c.rowptr[gb_m]);
    {
        std::vector<int64_t> cur(c.rowptr.begin(), c.rowptr.end() - 1);
        for (int64_t i = 0; i < g.nnzb; ++i)
            if (g.nnz_blk[i] > 0 && g.gb_row[i] >= 0)
                c.order[cur[g.gb_row[i]]++] = i;
    }
    // within a tile, COO blocks come first: make that the device order by
    // reordering each tile's range (stable)
    // pass 1: per block row totals
    std::vector<RowTotals> tot(gb_m);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t R = 0; R < gb_m; ++R) {
        RowTotals t;
        split_row(c, c.rowptr[R], c.rowptr[R + 1], [&](int64_t s, int64_t e) {
            t.tiles++;
            int64_t E = 0;
            for (int64_t p = s; p < e; ++p) {
                const int64_t i = c.order[p];
                t.blocks++;
                t.vals += c.nvals(i);
                t.alg += c.alg_payload(i);
                if (c.is_coo(i)) {
                    E += c.k(i);
                } else {
                    t.xblocks++;
                    t.bytes += c.payload_bytes(i);
                    if (g.gather_flag) t.bcols += c.valid_cols(i);
                }
            }
            t.bytes += c.coo_bytes(E);
        });
        tot[R] = t;
    }
    std::vector<RowTotals> pre(gb_m + 1);
    for (int64_t R = 0; R < gb_m; ++R) {
        pre[R + 1].tiles = pre[R].tiles + tot[R].tiles;
        pre[R + 1].blocks = pre[R].blocks + tot[R].blocks;
        pre[R + 1].bytes = pre[R].bytes + tot[R].bytes;
        pre[R + 1].vals = pre[R].vals + tot[R].vals;
        pre[R + 1].alg = pre[R].alg + tot[R].alg;
        pre[R + 1].bcols = pre[R].bcols + tot[R].bcols;
        pre[R + 1].xblocks = pre[R].xblocks + tot[R].xblocks;
    }
    const RowTotals &T = pre[gb_m];
    if (T.bytes / 16 > (int64_t)UINT32_MAX || T.tiles > INT32_MAX) {
        *code = CBSPMV_ERR_UNSUPPORTED;
        return "device payload above 64 GiB";
    }
    // split-row slots
    std::vector<int64_t> slot0(gb_m + 1, 0);
    int64_t split_rows = 0;
    int max_row_tiles = 1;
    for (int64_t R = 0; R < gb_m; ++R) {
        const int64_t nt = tot[R].tiles;
        slot0[R + 1] = slot0[R] + (nt > 1 ? nt : 0);
        split_rows += nt > 1;
        max_row_tiles = std::max<int>(max_row_tiles, (int)nt);
    }

    L = DeviceLayout();
    L.bs = bs;
    L.f32 = f32;
    L.unit = c.unit;
    L.gather = g.gather_flag;
    L.m = g.m;
    L.n = g.n;
    L.gb_m = gb_m;
    L.tiles.resize(T.tiles);
    L.blocks.resize(T.blocks);
    L.payload.assign(T.bytes, 0);
    L.slots = slot0[gb_m];
    L.split_rows = split_rows;
    L.max_row_tiles = max_row_tiles;
    L.nvals = T.vals;
    L.val_off.resize(T.vals);
    L.val_row.resize(T.vals);
    L.val_col.resize(T.vals);
    L.vsrc_ptr.assign(T.vals + 1, 0);
    L.vsrc.resize(g.src.size());
    L.input_slot.assign(g.nnz, -1);
    if (g.gather_flag && T.bcols > 0) L.block_cols = g.block_cols;

    // value-source counts first, so vsrc_ptr can be a prefix sum
    std::vector<int64_t> vcount(T.vals, 0);
    auto each_value_src = [&](int64_t i, auto fn) {
        // fn(local value index, global stored value index)
        const int32_t o = c.origin(i);
        for (int64_t q = 0; q < c.nvals(i); ++q) fn(q, g.f64_off[o] + q);
    };
    // pass 2: write tiles
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t R = 0; R < gb_m; ++R) {
        int64_t tile = pre[R].tiles, blk = pre[R].blocks;
        int64_t byte = pre[R].bytes, val = pre[R].vals;
        int64_t t_in_row = 0;
        const int64_t nt = tot[R].tiles;
        std::vector<int64_t> tb;
        std::vector<double> sorted_val;
        auto put_tile_val = [&](int64_t at_byte, double x) {
            if (f32) {
                const float f = (float)x;
                std::memcpy(L.payload.data() + at_byte, &f, 4);
            } else {
                std::memcpy(L.payload.data() + at_byte, &x, 8);
            }
        };
        split_row(c, c.rowptr[R], c.rowptr[R + 1], [&](int64_t s, int64_t e) {
            tb.clear();
            for (int64_t p = s; p < e; ++p)
                if (c.is_coo(c.order[p])) tb.push_back(c.order[p]);
            const int64_t ncoo = (int64_t)tb.size();
            for (int64_t p = s; p < e; ++p)
                if (!c.is_coo(c.order[p])) tb.push_back(c.order[p]);
            int64_t E = 0;
            for (int64_t q = 0; q < ncoo; ++q) E += c.k(tb[q]);
            TileDesc &td = L.tiles[tile];
            td.block_begin = (uint32_t)blk;
            td.block_row = (uint32_t)R;
            td.counts = (uint32_t)tb.size() | (uint32_t)ncoo << 8 |
                        (uint32_t)(tb.size() - ncoo) << 16;
            td.payload16 = (uint32_t)(byte / 16);
            td.coo_entries = (uint32_t)E;
            td.slot = nt > 1 ? (uint32_t)(slot0[R] + t_in_row) : 0xffffffffu;
            td.first_slot = nt > 1 ? (uint32_t)slot0[R] : 0xffffffffu;
            td.row_tiles = (uint32_t)nt;
            uint8_t *base = L.payload.data() + byte;
            uint32_t *idx = (uint32_t *)base;
            const int64_t vals_at = a16(E * 4);
            int64_t xoff = c.coo_bytes(E);  // CSR/dense payloads
            int64_t e0 = 0;
            for (size_t q = 0; q < tb.size(); ++q) {
                const int64_t i = tb[q];
                const int32_t o = c.origin(i);
                const int ty = c.type(i);
                const int64_t kk = c.k(i);
                const uint32_t *pu = g.pay_u32.data() + g.u32_off[o];
                BlockDesc &bd = L.blocks[blk + q];
                const int64_t vc = c.valid_cols(i);
                bd.xbase = g.gather_flag
                    ? (uint32_t)(g.block_cols_offset[R] + (int64_t)g.gb_col[i] * bs)
                    : (uint32_t)((int64_t)g.gb_col[i] * bs);
                bd.gb_col = (uint32_t)g.gb_col[i];
                uint32_t steps = 0;
                const uint32_t uni = (g.type_blk[i] & kUniform) ? 1u : 0u;
                if (ty == kCOO) {
                    bd.off = (uint32_t)e0;
                    int run = 0, maxrun = 0, prev = -1;
                    for (int64_t q2 = 0; q2 < kk; ++q2) {
                        const uint32_t w = pu[q2];
                        uint32_t r;
                        int64_t col;
                        if (g.compact) {
                            r = (w >> 12) & (bs - 1);
                            col = w & 0xfff;
                        } else if (g.direct) {
                            r = (w >> 16) & (bs - 1);
                            col = w & 0xffff;
                        } else {
                            r = (w >> c.bits) & (bs - 1);
                            col = c.resolve(i, w & (bs - 1));
                        }
                        run = ((int)r == prev) ? run + 1 : 1;
                        prev = (int)r;
                        maxrun = std::max(maxrun, run);
                        idx[e0 + q2] = (r << kColBits) | (uint32_t)col;
                        const int64_t v = val + (e0 + q2);
                        L.val_row[v] = (int32_t)(R * bs + r);
                        L.val_col[v] = (int32_t)col;
                    }
                    while ((1 << steps) < maxrun) ++steps;
                } else {
                    bd.off = (uint32_t)xoff;
                    uint8_t *pb = L.payload.data() + byte + xoff;
                    if (ty == kCSR) {
                        for (int64_t q2 = 0; q2 < bs + 1 + kk; ++q2) {
                            const uint32_t w = pu[q2];
                            if (isz == 1)
                                pb[q2] = (uint8_t)w;
                            else
                                ((uint16_t *)pb)[q2] = (uint16_t)w;
                        }
                    }
                    xoff += c.payload_bytes(i);
                }
                bd.meta = (uint32_t)ty | uni << 2 | (uint32_t)kk << 3 |
                          (uint32_t)vc << 14 | steps << 20;
                if (ty == kCOO) e0 += kk;
            }
            // The tile's COO section holds the entries of all of its COO
            // blocks sorted by (row, column) (keys are unique: distinct blocks
            // hold distinct columns), cut into 32 lane slices of consecutive
            // entries (coo_slice_pos), so a lane's entries never go down a row
            // and a row's entries are one run of lanes.  Stored value v keeps
            // its block-major number; only its payload position moves.
            if (E > 0) {
                std::vector<uint64_t> key((size_t)E);
                sorted_val.resize((size_t)E);
                for (int64_t q2 = 0; q2 < E; ++q2)
                    key[q2] = (uint64_t)idx[q2] << 16 | (uint64_t)q2;
                std::sort(key.begin(), key.end());
                int64_t e1 = 0;
                for (size_t q = 0; q < (size_t)ncoo; ++q) {
                    const int64_t i = tb[q];
                    const double *pf = g.pay_f64.data() + g.f64_off[c.origin(i)];
                    for (int64_t q2 = 0; q2 < c.k(i); ++q2, ++e1) sorted_val[e1] = pf[q2];
                }
                for (int64_t q2 = 0; q2 < E; ++q2) {
                    const int64_t from = (int64_t)(key[q2] & 0xffff);
                    const int64_t pos = coo_slice_pos(q2, E);
                    idx[pos] = (uint32_t)(key[q2] >> 16);
                    if (c.unit) {  // no value arrays: nothing to place
                        L.val_off[val + from] = 0;
                        continue;
                    }
                    const int64_t at = byte + vals_at + pos * vsz;
                    put_tile_val(at, sorted_val[from]);
                    L.val_off[val + from] = (uint64_t)at;
                }
            }
            // value slots of CSR/DENSE blocks come after the tile's COO values
            int64_t v = val + E;
            int64_t xo = c.coo_bytes(E);
            for (size_t q = ncoo; q < tb.size(); ++q) {
                const int64_t i = tb[q];
                const int32_t o = c.origin(i);
                const int ty = c.type(i);
                const int64_t kk = c.k(i);
                const uint32_t *pu = g.pay_u32.data() + g.u32_off[o];
                const double *pf = g.pay_f64.data() + g.f64_off[o];
                const int64_t vc = c.valid_cols(i);
                const int64_t vals_here = ty == kCSR ? a16((bs + 1 + kk) * isz) : 0;
                const int64_t nv = c.nvals(i);
                for (int64_t q2 = 0; q2 < nv; ++q2) {
                    const int64_t at = byte + xo + vals_here + q2 * vsz;
                    const double x = pf[q2];
                    if (c.unit) {  // CSR: no values; DENSE: bit q2 of the bitmask
                        if (ty != kCSR && x == 1.0)
                            L.payload[byte + xo + q2 / 8] |= (uint8_t)(1u << (q2 % 8));
                        L.val_off[v + q2] = 0;
                    } else if (f32) {
                        const float f = (float)x;
                        std::memcpy(L.payload.data() + at, &f, 4);
                        L.val_off[v + q2] = (uint64_t)at;
                    } else {
                        std::memcpy(L.payload.data() + at, &x, 8);
                        L.val_off[v + q2] = (uint64_t)at;
                    }
                    int64_t r, col;
                    if (ty == kCSR) {
                        r = 0;
                        while ((int64_t)pu[r + 1] <= q2) ++r;
                        col = c.resolve(i, pu[bs + 1 + q2]);
                    } else {
                        r = q2 / bs;
                        const int64_t lc = q2 % bs;
                        col = lc < vc ? c.resolve(i, lc) : -1;
                    }
                    const int64_t grow = R * bs + r;
                    L.val_row[v + q2] = grow < g.m ? (int32_t)grow : -1;
                    L.val_col[v + q2] = (int32_t)col;
                }
                v += nv;
                xo += c.payload_bytes(i);
            }
            // value sources, in the same device value order
            int64_t vv = val;
            for (size_t q = 0; q < tb.size(); ++q) {
                const int64_t i = tb[q];
                if (!c.is_coo(i)) continue;
                each_value_src(i, [&](int64_t, int64_t gv) {
                    vcount[vv++] = g.src_ptr[gv + 1] - g.src_ptr[gv];
                });
            }
            for (size_t q = ncoo; q < tb.size(); ++q) {
                const int64_t i = tb[q];
                each_value_src(i, [&](int64_t, int64_t gv) {
                    vcount[vv++] = g.src_ptr[gv + 1] - g.src_ptr[gv];
                });
            }
            val = vv;
            blk += (int64_t)tb.size();
            byte += c.coo_bytes(E);
            for (size_t q = ncoo; q < tb.size(); ++q) byte += c.payload_bytes(tb[q]);
            ++tile;
            ++t_in_row;
        });
    }
    for (int64_t v = 0; v < T.vals; ++v) L.vsrc_ptr[v + 1] = L.vsrc_ptr[v] + vcount[v];
    // fill sources in a second sweep over blocks in device value order
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t R = 0; R < gb_m; ++R) {
        int64_t val = pre[R].vals;
        std::vector<int64_t> tb;
        split_row(c, c.rowptr[R], c.rowptr[R + 1], [&](int64_t s, int64_t e) {
            tb.clear();
            for (int64_t p = s; p < e; ++p)
                if (c.is_coo(c.order[p])) tb.push_back(c.order[p]);
            for (int64_t p = s; p < e; ++p)
                if (!c.is_coo(c.order[p])) tb.push_back(c.order[p]);
            for (int64_t i : tb) {
                each_value_src(i, [&](int64_t, int64_t gv) {
                    int64_t w = L.vsrc_ptr[val];
                    for (int64_t z = g.src_ptr[gv]; z < g.src_ptr[gv + 1]; ++z) {
                        L.vsrc[w++] = g.src[z];
                        L.input_slot[g.src[z]] = val;
                    }
                    ++val;
                });
            }
        });
    }
    {
        int64_t coo_e = 0, all_e = 0;
        for (const TileDesc &t : L.tiles) {
            L.max_entries = std::max<int64_t>(L.max_entries, t.coo_entries);
            coo_e += t.coo_entries;
        }
        // tiles are contiguous in the payload, in order
        for (size_t t = 0; t < L.tiles.size(); ++t) {
            const int64_t end = t + 1 < L.tiles.size() ? (int64_t)L.tiles[t + 1].payload16 * 16
                                                       : (int64_t)L.payload.size();
            L.max_tile_bytes =
                std::max<int64_t>(L.max_tile_bytes, end - (int64_t)L.tiles[t].payload16 * 16);
        }
        for (const BlockDesc &bd : L.blocks) all_e += meta_nnz(bd.meta);
        L.coo_share = all_e > 0 ? (double)coo_e / (double)all_e : 1.0;
    }
    // algorithmic bytes: tile descriptors, CSR/DENSE block descriptors (COO
    // blocks need none: their entries carry row and column), payload without
    // padding, gather-list reads of CSR/DENSE x tiles, x once, y once
    // (split-row partial sums are scratch traffic, not counted)
    L.alg_bytes = T.tiles * (int64_t)sizeof(TileDesc) +
                  T.xblocks * (int64_t)sizeof(BlockDesc) + T.alg + T.bcols * 4 +
                  g.n * vsz + g.m * vsz;
    return "";
}

std::vector<uint32_t> partition_tiles(const DeviceLayout &L, int64_t warps) {
    const int64_t nt = (int64_t)L.tiles.size();
    std::vector<double> cost(nt);
    double total = 0;
    for (int64_t t = 0; t < nt; ++t) {
        const TileDesc &d = L.tiles[t];
        double c = 96.0 + d.coo_entries;  // per-tile overhead in entry units
        const uint32_t nb = d.counts & 0xff, ncoo = (d.counts >> 8) & 0xff;
        for (uint32_t q = ncoo; q < nb; ++q) c += 1.5 * meta_nnz(L.blocks[d.block_begin + q].meta);
        cost[t] = c;
        total += c;
    }
    std::vector<uint32_t> part(warps + 1, (uint32_t)nt);
    part[0] = 0;
    double acc = 0;
    int64_t w = 1;
    for (int64_t t = 0; t < nt && w < warps; ++t) {
        acc += cost[t];
        while (w < warps && acc >= total * (double)w / (double)warps) part[w++] = (uint32_t)(t + 1);
    }
    return part;
}

}  // namespace cb
