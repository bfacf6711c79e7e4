// Host build of the row-segment stream (layout in cb_rowseg.hpp).
#include "cb_rowseg.hpp"

#include <algorithm>
#include <climits>
#include <cstring>
#include <utility>

namespace cb {

namespace {
int64_t a16_64(int64_t x) { return (x + 15) & ~int64_t(15); }
}  // namespace

bool rowseg_applies(const DeviceLayout &L) {
    return L.nvals > 0 && L.n <= kRsMaxCols && L.m < (int64_t(1) << 31);
}

bool rowseg_all_coo(const DeviceLayout &L) {
    for (const BlockDesc &b : L.blocks)
        if (meta_type(b.meta) != 0) return false;  // a CSR or DENSE block
    return true;
}

void rowseg_cut(const std::vector<int32_t> &cinfo, const std::vector<int64_t> &cuts,
                int64_t seg0, int32_t tag, std::vector<int32_t> &meta,
                std::vector<int32_t> &spans) {
    const int64_t nseg = (int64_t)cuts.size() - 1;
    int32_t open = -1;
    for (int64_t s = 0; s < nseg; ++s) {
        const int64_t c0 = cuts[(size_t)s], c1 = cuts[(size_t)s + 1];
        const int32_t *f = &cinfo[(size_t)(4 * c0)];
        int32_t mt[4] = {f[0], f[1], -1, -1};
        int64_t nfl = 0;
        for (int64_t c = c0; c < c1; ++c) nfl += cinfo[(size_t)(4 * c + 2)];
        if (s > 0 && !f[1] && open >= 0) {  // the first row goes on from segment s - 1
            mt[2] = open;
            spans[(size_t)(4 * open + 1)] = (int32_t)(seg0 + s);
        }
        const bool cont = s + 1 < nseg && !cinfo[(size_t)(4 * cuts[(size_t)s + 1] + 1)];
        if (!cont) {
            open = -1;
        } else if (nfl > 0 || mt[2] < 0) {  // the last row starts here: a new span
            open = (int32_t)(spans.size() / 4);
            spans.insert(spans.end(), {(int32_t)(seg0 + s), (int32_t)(seg0 + s),
                                       cinfo[(size_t)(4 * (c1 - 1) + 3)], tag});
            mt[3] = open;
        }
        meta.insert(meta.end(), mt, mt + 4);
    }
}

// Every stored entry of the tiles with the payload offset of its value: the
// COO sections, then CSR blocks (row pointers, block-local columns resolved
// through the gather list) and DENSE blocks (columns below the block's valid
// count; unit-valued layouts: the bits set in the mask).
void tile_entries(const DeviceLayout &L, std::vector<int32_t> &erow, std::vector<int32_t> &ecol,
                  std::vector<int64_t> &eoff) {
    const int64_t m = L.m;
    const int unit = L.unit;
    const int64_t vsz = L.f32 ? 4 : 8;
    erow.reserve((size_t)L.nvals);
    ecol.reserve((size_t)L.nvals);
    eoff.reserve((size_t)L.nvals);
    const int bs = L.bs;
    const int64_t isz = bs == 16 ? 1 : 2;
    for (const TileDesc &t : L.tiles) {
        const int64_t E = t.coo_entries, base = (int64_t)t.payload16 * 16;
        const uint32_t *idx = reinterpret_cast<const uint32_t *>(L.payload.data() + base);
        const int64_t vals = base + a16_64(4 * E);  // (none when unit)
        for (int64_t q = 0; q < E; ++q) {
            erow.push_back((int32_t)((int64_t)t.block_row * bs + (idx[q] >> kColBits)));
            ecol.push_back((int32_t)(idx[q] & ((1u << kColBits) - 1)));
            eoff.push_back(vals + q * vsz);
        }
        const uint32_t nb = t.counts & 0xffu, ncoo = (t.counts >> 8) & 0xffu;
        for (uint32_t j = ncoo; j < nb; ++j) {
            const BlockDesc &bd = L.blocks[(size_t)t.block_begin + j];
            const int64_t pb = base + bd.off;
            // (the valid-column field can carry a bit of an oversized raw
            // entry count of a DENSE block built from duplicates: clamp)
            const uint32_t k = meta_nnz(bd.meta);
            const uint32_t valid = std::min<uint32_t>((bd.meta >> 14) & 63u, (uint32_t)bs);
            auto col_of = [&](int64_t c) -> int32_t {
                return L.gather ? L.block_cols[(size_t)bd.xbase + (size_t)c]
                                : (int32_t)(bd.xbase + c);
            };
            if (meta_type(bd.meta) == 1) {  // CSR
                const uint8_t *p8 = L.payload.data() + pb;
                auto at = [&](int64_t i) -> int64_t {
                    return isz == 1 ? p8[i] : reinterpret_cast<const uint16_t *>(p8)[i];
                };
                const int64_t cv = pb + a16_64((bs + 1 + (int64_t)k) * isz);
                for (int64_t r = 0; r < bs; ++r) {
                    const int64_t row = (int64_t)t.block_row * bs + r;
                    for (int64_t q = at(r); q < at(r + 1); ++q) {
                        if (row >= m) continue;
                        erow.push_back((int32_t)row);
                        ecol.push_back(col_of(at(bs + 1 + q)));
                        eoff.push_back(cv + q * vsz);
                    }
                }
            } else {  // DENSE, row-major bs x bs
                for (int64_t r = 0; r < bs; ++r) {
                    const int64_t row = (int64_t)t.block_row * bs + r;
                    if (row >= m) continue;
                    for (int64_t c = 0; c < (int64_t)valid; ++c) {
                        const int64_t i = r * bs + c;
                        if (unit && !((L.payload[(size_t)(pb + i / 8)] >> (i % 8)) & 1)) continue;
                        erow.push_back((int32_t)row);
                        ecol.push_back(col_of(c));
                        eoff.push_back(pb + i * vsz);
                    }
                }
            }
        }
    }
}

std::string build_rowseg(const DeviceLayout &L, int64_t warps, RowSegHost &R) {
    if (!rowseg_applies(L)) return "the layout does not take the row-segment stream";
    const int64_t m = L.m, C = rs_chunk_entries();
    const int f32 = L.f32;
    const int unit = L.unit;
    const int64_t vsz = f32 ? 4 : 8, CB = rs_chunk_bytes(f32, unit);
    R = RowSegHost();
    R.f32 = f32;
    R.unit = unit;
    R.m = m;
    R.n = L.n;
    std::vector<int32_t> erow, ecol;
    std::vector<int64_t> eoff;
    tile_entries(L, erow, ecol, eoff);
    const int64_t nv = (int64_t)erow.size();
    if (nv == 0) return "row-segment stream: no entries";
    for (int64_t k2 = 0; k2 < nv; ++k2)  // every gather stays inside x, every row inside y
        if (ecol[(size_t)k2] < 0 || ecol[(size_t)k2] >= L.n || erow[(size_t)k2] < 0 ||
            erow[(size_t)k2] >= m)
            return "row-segment stream: an entry outside the matrix";
    // entries by (row, column): counting sort on rows, then columns
    std::vector<int64_t> rp((size_t)m + 1, 0);
    for (int64_t v = 0; v < nv; ++v) ++rp[(size_t)erow[v] + 1];
    for (int64_t r = 0; r < m; ++r) rp[r + 1] += rp[r];
    std::vector<int64_t> order((size_t)nv);
    {
        std::vector<int64_t> at(rp.begin(), rp.end() - 1);
        for (int64_t v = 0; v < nv; ++v) order[(size_t)at[(size_t)erow[v]]++] = v;
    }
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t r = 0; r < m; ++r)
        std::sort(order.begin() + rp[r], order.begin() + rp[r + 1],
                  [&](int64_t a, int64_t b) { return ecol[a] < ecol[b]; });
    // ordinals of the non-empty rows
    int64_t nord = 0;
    for (int64_t r = 0; r < m; ++r) nord += rp[r + 1] > rp[r];
    R.nord = (int32_t)nord;
    if (nord < m) {
        R.rowmap.reserve((size_t)nord);
        for (int64_t r = 0; r < m; ++r) {
            if (rp[r + 1] > rp[r])
                R.rowmap.push_back((int32_t)r);
            else
                R.empty.push_back((int32_t)r);
        }
    }
    const int64_t nch = (nv + C - 1) / C;
    R.nch = (int32_t)nch;
    R.chunks.assign((size_t)(nch * CB), 0);
    // words, values and per-entry ordinals; padding: value 0 on column 0,
    // the first padding entry starting the extra ordinal nord
    std::vector<int32_t> epos((size_t)nv);  // each entry's place in the stream
    std::vector<int32_t> ordv((size_t)(nch * C));
    std::vector<uint8_t> start((size_t)(nch * C), 0);
    int64_t ord = 0;
    for (int64_t e = 0; e < nch * C; ++e) {
        uint32_t word;
        if (e < nv) {
            const int64_t v = order[(size_t)e];
            const bool st = e > 0 && erow[v] != erow[order[(size_t)e - 1]];
            ord += st;
            start[(size_t)e] = st;
            word = (uint32_t)ecol[v] | (st ? kRsStart : 0u);
            if (!unit)
                std::memcpy(R.chunks.data() + rs_value_offset(e, f32),
                            L.payload.data() + eoff[v], (size_t)vsz);
            epos[(size_t)v] = (int32_t)e;
        } else {
            const bool st = e == nv;
            ord = st ? nord : ord;
            start[(size_t)e] = st;
            word = st ? kRsStart : 0u;
        }
        ordv[(size_t)e] = (int32_t)ord;
        // with 4 entries per lane the words of a chunk are in entry order
        const int64_t c = e / C, i = e % C;
        std::memcpy(R.chunks.data() + c * CB + 4 * i, &word, 4);
    }
    // chunk summaries, then segments of M chunks, about one per warp
    R.cinfo.assign((size_t)(4 * nch), 0);
    for (int64_t c = 0; c < nch; ++c) {
        int32_t *ci = &R.cinfo[(size_t)(4 * c)];
        const int64_t e0 = c * C;
        ci[0] = ordv[(size_t)e0] - start[(size_t)e0];
        ci[1] = start[(size_t)e0];
        for (int64_t e = e0; e < e0 + C; ++e) ci[2] += start[(size_t)e];
        ci[3] = ordv[(size_t)(e0 + C - 1)];
    }
    const int64_t M = std::max<int64_t>(1, (nch + std::max<int64_t>(warps, 1) - 1) /
                                               std::max<int64_t>(warps, 1));
    const int64_t nseg = (nch + M - 1) / M;
    R.M = (int32_t)M;
    R.nseg = (int32_t)nseg;
    {
        std::vector<int64_t> cuts;
        for (int64_t s0 = 0; s0 < nseg; ++s0) cuts.push_back(s0 * M);
        cuts.push_back(nch);
        rowseg_cut(R.cinfo, cuts, 0, 0, R.meta, R.spans);
    }
    // the CTAs' windows of x: per CTA, the W consecutive columns holding the
    // most of its entries (a sliding window over its sorted columns)
    const int64_t G = std::max<int64_t>(1, std::max<int64_t>(warps, 1) / kRsWarps);
    const int64_t W = kRsWindowBytes / vsz;
    R.G = (int32_t)G;
    R.W = (int32_t)W;
    R.wbase.assign((size_t)G, 0);
    std::vector<int32_t> cols;
    for (int64_t b = 0; b < G; ++b) {
        const int64_t s0 = b * nseg / G, s1 = (b + 1) * nseg / G;
        const int64_t e0 = std::min(nv, s0 * M * C), e1 = std::min(nv, s1 * M * C);
        if (e0 >= e1) continue;
        cols.clear();
        for (int64_t e = e0; e < e1; ++e) cols.push_back(ecol[order[(size_t)e]]);
        std::sort(cols.begin(), cols.end());
        size_t best = 0, lo = 0;
        int32_t wb = cols[0];
        for (size_t hi = 0; hi < cols.size(); ++hi) {
            while ((int64_t)cols[hi] - cols[lo] >= W) ++lo;
            if (hi - lo + 1 > best) {
                best = hi - lo + 1;
                wb = cols[lo];
            }
        }
        R.wbase[(size_t)b] = wb;
        for (int64_t e = e0; e < e1; ++e) {
            const int64_t col = ecol[order[(size_t)e]];
            if (col >= wb && col < wb + W) {
                const int64_t c = e / C, i = e % C;
                uint32_t word;
                std::memcpy(&word, R.chunks.data() + c * CB + 4 * i, 4);
                word |= kRsWin;
                std::memcpy(R.chunks.data() + c * CB + 4 * i, &word, 4);
            }
        }
    }
    // per stored value (device order) its stream entry, for value updates:
    // stored value v sits at payload offset val_off[v] (absent from plans
    // loaded from SpMV-only files, which take no new values)
    if (!unit && (int64_t)L.val_off.size() == L.nvals) {
        std::vector<std::pair<int64_t, int32_t>> by_off((size_t)nv);
        for (int64_t k = 0; k < nv; ++k) by_off[(size_t)k] = {eoff[(size_t)k], epos[(size_t)k]};
        std::sort(by_off.begin(), by_off.end());
        R.vpos.resize((size_t)L.nvals);
        for (int64_t v = 0; v < L.nvals; ++v) {
            const int64_t off = (int64_t)L.val_off[v];
            auto it = std::lower_bound(by_off.begin(), by_off.end(),
                                       std::make_pair(off, INT32_MIN));
            // a DENSE slot outside the valid columns or rows has no entry
            R.vpos[(size_t)v] = it != by_off.end() && it->first == off ? it->second : -1;
        }
    }
    R.alg_bytes = L.alg_bytes;
    return "";
}

}  // namespace cb

namespace cb {

std::string build_balanced(const DeviceLayout &L, const HostCB &g, BalancedHost &B) {
    if (g.o.row_owned || L.unit) return "the plan is row-owned or stores no values";
    if (L.n > kRsMaxCols || L.m >= (int64_t(1) << 31)) return "matrix too large";
    const int bs = L.bs, W = g.o.waves;
    const int64_t vsz = L.f32 ? 4 : 8;
    B = BalancedHost();
    B.f32 = L.f32;
    std::vector<int32_t> erow, ecol;
    std::vector<int64_t> eoff;
    tile_entries(L, erow, ecol, eoff);
    const int64_t ne = (int64_t)erow.size();
    for (int64_t k = 0; k < ne; ++k)
        if (ecol[(size_t)k] < 0 || ecol[(size_t)k] >= L.n || erow[(size_t)k] < 0 ||
            erow[(size_t)k] >= L.m)
            return "balanced stream: an entry outside the matrix";
    // each entry's block (block row, block column in the gathered space) and
    // that block's place in the block order: sorted tables searched by
    // binary search (the gather lists can be as long as the entries)
    std::vector<std::pair<int32_t, int32_t>> gcol;  // per block row: (column, position), by column
    if (g.gather_flag) {
        gcol.resize(g.block_cols.size());
        for (int64_t R = 0; R < g.gb_m; ++R) {
            const int32_t o0 = g.block_cols_offset[(size_t)R], o1 = g.block_cols_offset[(size_t)R + 1];
            for (int32_t q = o0; q < o1; ++q) gcol[(size_t)q] = {g.block_cols[(size_t)q], q - o0};
            std::sort(gcol.begin() + o0, gcol.begin() + o1);
        }
    }
    std::vector<std::pair<uint64_t, int64_t>> bkey;  // ((block row, block column), index), sorted
    const int64_t nb = (int64_t)g.gb_row.size();
    for (int64_t i = 0; i < nb; ++i)
        if (g.gb_row[(size_t)i] >= 0)
            bkey.push_back({(uint64_t)g.gb_row[(size_t)i] << 32 | (uint32_t)g.gb_col[(size_t)i], i});
    std::sort(bkey.begin(), bkey.end());
    std::vector<int64_t> blk((size_t)ne);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t k = 0; k < ne; ++k) {
        const int64_t R = erow[(size_t)k] / bs;
        int64_t C = -1;
        if (g.gather_flag) {
            const auto b0 = gcol.begin() + g.block_cols_offset[(size_t)R];
            const auto b1 = gcol.begin() + g.block_cols_offset[(size_t)R + 1];
            const auto it = std::lower_bound(b0, b1, std::make_pair(ecol[(size_t)k], INT32_MIN));
            if (it != b1 && it->first == ecol[(size_t)k]) C = it->second / bs;
        } else {
            C = ecol[(size_t)k] / bs;
        }
        const uint64_t key = (uint64_t)R << 32 | (uint32_t)C;
        const auto it = std::lower_bound(bkey.begin(), bkey.end(), std::make_pair(key, INT64_MIN));
        if (C < 0 || it == bkey.end() || it->first != key) {
            bad |= 1;
            blk[(size_t)k] = -1;
        } else {
            blk[(size_t)k] = it->second;
        }
    }
    if (bad) return "balanced stream: an entry outside every block";
    // entries by (balanced block, row, column)
    std::vector<int64_t> order((size_t)ne);
    for (int64_t k = 0; k < ne; ++k) order[(size_t)k] = k;
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        if (blk[(size_t)a] != blk[(size_t)b]) return blk[(size_t)a] < blk[(size_t)b];
        if (erow[(size_t)a] != erow[(size_t)b]) return erow[(size_t)a] < erow[(size_t)b];
        return ecol[(size_t)a] < ecol[(size_t)b];
    });
    // groups of W consecutive balanced blocks (the reference's CTAs), each
    // padded to whole quads with skip entries
    const int64_t ngroups = (nb + W - 1) / W;
    B.gstart.assign((size_t)ngroups + 1, 0);
    int64_t k = 0, quads = 0;
    for (int64_t gi = 0; gi < ngroups; ++gi) {
        B.gstart[(size_t)gi] = quads;
        const int64_t k0 = k;
        while (k < ne && blk[(size_t)order[(size_t)k]] / W == gi) ++k;
        const int64_t cnt = k - k0, nq = (cnt + 3) / 4;
        for (int64_t e = 0; e < nq * 4; ++e) {
            const bool real = e < cnt;
            const int64_t v = real ? order[(size_t)(k0 + e)] : -1;
            B.rows.push_back(real ? (uint32_t)erow[(size_t)v] : kBalSkip);
            B.cols.push_back(real ? (uint32_t)ecol[(size_t)v] : 0u);
            B.eoff.push_back(real ? eoff[(size_t)v] : -1);
        }
        quads += nq;
    }
    B.gstart[(size_t)ngroups] = quads;
    B.nquads = quads;
    B.vals.assign((size_t)(quads * 4 * vsz), 0);
    for (int64_t e = 0; e < quads * 4; ++e)
        if (B.eoff[(size_t)e] >= 0)
            std::memcpy(B.vals.data() + e * vsz, L.payload.data() + B.eoff[(size_t)e],
                        (size_t)vsz);
    return "";
}

}  // namespace cb
