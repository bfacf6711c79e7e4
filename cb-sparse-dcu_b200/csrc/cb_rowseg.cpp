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
    if (L.nvals <= 0 || L.n > kRsMaxCols || L.m >= (int64_t(1) << 31)) return false;
    for (const BlockDesc &b : L.blocks)
        if (meta_type(b.meta) != 0) return false;  // a CSR or DENSE block
    return true;
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
    // the entries of the tiles' COO sections (every block is a COO block):
    // row, column and the payload offset of the value
    int64_t nv = 0;
    for (const TileDesc &t : L.tiles) nv += t.coo_entries;
    if (nv != L.nvals) return "row-segment stream: COO entries and stored values differ";
    std::vector<int32_t> erow((size_t)nv), ecol((size_t)nv);
    std::vector<int64_t> eoff((size_t)nv);
    {
        int64_t k = 0;
        for (const TileDesc &t : L.tiles) {
            const int64_t E = t.coo_entries, base = (int64_t)t.payload16 * 16;
            const uint32_t *idx = reinterpret_cast<const uint32_t *>(L.payload.data() + base);
            const int64_t vals = base + a16_64(4 * E);  // (none when unit)
            for (int64_t q = 0; q < E; ++q, ++k) {
                erow[(size_t)k] = (int32_t)((int64_t)t.block_row * L.bs + (idx[q] >> kColBits));
                ecol[(size_t)k] = (int32_t)(idx[q] & ((1u << kColBits) - 1));
                eoff[(size_t)k] = vals + q * vsz;
            }
        }
    }
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
            eoff[v] = -1 - e;  // from here on: the entry's place in the stream
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
    // segments of M chunks, about one per warp
    const int64_t M = std::max<int64_t>(1, (nch + std::max<int64_t>(warps, 1) - 1) /
                                               std::max<int64_t>(warps, 1));
    const int64_t nseg = (nch + M - 1) / M;
    R.M = (int32_t)M;
    R.nseg = (int32_t)nseg;
    R.meta.assign((size_t)(4 * nseg), -1);
    int32_t open = -1;
    for (int64_t s = 0; s < nseg; ++s) {
        const int64_t e0 = s * M * C, e1 = std::min(nch, (s + 1) * M) * C - 1;
        int32_t *mt = &R.meta[(size_t)(4 * s)];
        mt[0] = ordv[(size_t)e0] - start[(size_t)e0];
        mt[1] = start[(size_t)e0];
        int64_t nfl = 0;
        for (int64_t e = e0; e <= e1; ++e) nfl += start[(size_t)e];
        if (s > 0 && !start[(size_t)e0]) {  // the first row goes on from segment s - 1
            if (open < 0) return "row-segment spans out of order";
            mt[2] = open;
            R.spans[(size_t)(4 * open + 1)] = (int32_t)s;
        }
        const bool cont = s + 1 < nseg && !start[(size_t)((s + 1) * M * C)];
        if (!cont) {
            open = -1;
        } else if (nfl > 0 || mt[2] < 0) {  // the last row starts here: a new span
            open = (int32_t)(R.spans.size() / 4);
            R.spans.insert(R.spans.end(), {(int32_t)s, (int32_t)s, ordv[(size_t)e1], 0});
            mt[3] = open;
        }
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
    if (!unit && (int64_t)L.val_off.size() == nv) {
        std::vector<std::pair<int64_t, int32_t>> by_off((size_t)nv);
        {
            int64_t k = 0;
            for (const TileDesc &t : L.tiles) {
                const int64_t E = t.coo_entries, base = (int64_t)t.payload16 * 16;
                for (int64_t q = 0; q < E; ++q, ++k)
                    by_off[(size_t)k] = {base + a16_64(4 * E) + q * vsz,
                                         (int32_t)(-1 - eoff[(size_t)k])};
            }
        }
        std::sort(by_off.begin(), by_off.end());
        R.vpos.resize((size_t)nv);
        for (int64_t v = 0; v < nv; ++v) {
            const int64_t off = (int64_t)L.val_off[v];
            auto it = std::lower_bound(by_off.begin(), by_off.end(),
                                       std::make_pair(off, INT32_MIN));
            if (it == by_off.end() || it->first != off)
                return "row-segment stream: a stored value outside the COO sections";
            R.vpos[(size_t)v] = it->second;
        }
    }
    R.alg_bytes = L.alg_bytes;
    return "";
}

}  // namespace cb
