// Host CB builder (see cb_builder.hpp).  Produces the reference's
// GLOBAL_BLOCK content bit for bit; the reference steps each function
// follows are cited beside it.  Differences are only in how the work is done:
// block rows are independent once the input is row-sorted, so discovery,
// gathering and encoding run in parallel per block row, and the hash maps of
// the reference (coo2block.h:87, :567) are replaced by per-row open-addressing
// tables and a hash of each row's column pattern.
#include "cb_builder.hpp"

#include <omp.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <queue>
#include <unordered_map>

#include "cbspmv.h"

namespace cb {
namespace {

constexpr int kWave = 64;  // the reference's wavefront, fixed in its rules

int bits_of(int bs) {
    int b = 0;
    while ((1 << b) < bs) ++b;
    return b;
}

// Small open-addressing map int -> int for one block row.
struct RowMap {
    std::vector<int32_t> key, value;
    uint32_t mask = 0;
    void reset(int64_t expected) {
        uint32_t cap = 16;
        while (cap < 2 * expected) cap <<= 1;
        if (key.size() < cap) {
            key.resize(cap);
            value.resize(cap);
        }
        mask = cap - 1;
        std::fill(key.begin(), key.begin() + cap, -1);
    }
    // returns the slot's value reference and whether it was inserted
    int32_t &find(int32_t k, bool &inserted) {
        uint32_t h = (uint32_t)k * 2654435761u;
        for (uint32_t i = h & mask;; i = (i + 1) & mask) {
            if (key[i] == k) {
                inserted = false;
                return value[i];
            }
            if (key[i] == -1) {
                key[i] = k;
                inserted = true;
                return value[i];
            }
        }
    }
};

// coo2block_pre_metadata (coo2block.h:77-121).  With rows sorted, blocks are
// discovered block row by block row, and inside a row in order of first touch,
// which is the reference's global first-touch order.
void discover(HostCB &g, const std::vector<int64_t> &rs, const int32_t *colv,
              std::vector<int32_t> &lid, std::vector<int64_t> &base) {
    const int bs = g.o.bs;
    const int64_t gb_m = g.gb_m;
    std::vector<int32_t> nb(gb_m, 0);
    std::vector<int32_t> tmpcol(g.nnz);
    lid.resize(g.nnz);
#pragma omp parallel
    {
        RowMap map;
#pragma omp for schedule(dynamic, 16)
        for (int64_t R = 0; R < gb_m; ++R) {
            const int64_t s = rs[R], e = rs[R + 1];
            if (s == e) continue;
            map.reset(e - s);
            int32_t count = 0;
            for (int64_t i = s; i < e; ++i) {
                const int32_t bj = colv[i] / bs;
                bool ins;
                int32_t &v = map.find(bj, ins);
                if (ins) {
                    v = count;
                    tmpcol[s + count] = bj;
                    ++count;
                }
                lid[i] = v;
            }
            nb[R] = count;
        }
    }
    base.assign(gb_m + 1, 0);
    for (int64_t R = 0; R < gb_m; ++R) base[R + 1] = base[R] + nb[R];
    g.nnzb = base[gb_m];
    g.gb_row.assign(g.nnzb, 0);
    g.gb_col.assign(g.nnzb, 0);
    g.nnz_blk.assign(g.nnzb, 0);
    g.type_blk.assign(g.nnzb, kCOO);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t R = 0; R < gb_m; ++R) {
        const int64_t s = rs[R], e = rs[R + 1];
        for (int32_t j = 0; j < nb[R]; ++j) {
            g.gb_row[base[R] + j] = (int32_t)R;
            g.gb_col[base[R] + j] = tmpcol[s + j];
        }
        for (int64_t i = s; i < e; ++i) g.nnz_blk[base[R] + lid[i]]++;
    }
}

// gather (coo2block.h:7-61): sorted distinct columns of every block row, and
// each nonzero's position in its row's list.
void gather_columns(HostCB &g, const std::vector<int64_t> &rs,
                    const int32_t *col, std::vector<int32_t> &gcol) {
    const int64_t gb_m = g.gb_m;
    std::vector<std::vector<int32_t>> lists(gb_m);
    gcol.resize(g.nnz);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t R = 0; R < gb_m; ++R) {
        const int64_t s = rs[R], e = rs[R + 1];
        std::vector<int32_t> &l = lists[R];
        l.assign(col + s, col + e);
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
        for (int64_t i = s; i < e; ++i)
            gcol[i] = (int32_t)(std::lower_bound(l.begin(), l.end(), col[i]) -
                                l.begin());
    }
    g.block_cols_offset.assign(gb_m + 1, 0);
    for (int64_t R = 0; R < gb_m; ++R)
        g.block_cols_offset[R + 1] =
            g.block_cols_offset[R] + (int32_t)lists[R].size();
    g.block_cols.resize(g.block_cols_offset[gb_m]);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t R = 0; R < gb_m; ++R)
        std::copy(lists[R].begin(), lists[R].end(),
                  g.block_cols.begin() + g.block_cols_offset[R]);
}

struct BlockIn {  // one block's nonzeros in input order (COO_BLOCK_ORIG)
    std::vector<int32_t> r, c, src;
    std::vector<double> v;
    void clear() {
        r.clear();
        c.clear();
        v.clear();
        src.clear();
    }
};

struct RowOut {  // encoded payload of one block row, blocks in order
    std::vector<uint32_t> u32;
    std::vector<double> f64;
    std::vector<int32_t> src;
    std::vector<int32_t> src_cnt;  // per value
    std::vector<int64_t> u32_len, f64_len;
};

// uniform test of the dense image built by summing entries in input order
// (coo2block.h:292-305 and :320-327): every row equals row 0.
bool dense_uniform(const std::vector<double> &dense, int bs) {
    for (int r = 1; r < bs; ++r)
        for (int c = 0; c < bs; ++c)
            if (!(dense[r * bs + c] == dense[c])) return false;
    return true;
}

// Rows of the dense image all equal, for a block whose (r, c) pairs are
// distinct: the image holds 0.0 + v at each entry and 0.0 elsewhere.  `ord`
// lists the entries sorted by (r, c).
bool sparse_uniform(const BlockIn &b, const std::vector<int> &ord, int bs) {
    // count entries whose image value is nonzero, per row
    int cnt[64] = {0};
    for (int j : ord)
        if ((0.0 + b.v[j]) != 0.0) cnt[b.r[j]]++;
    for (int r = 1; r < bs; ++r)
        if (cnt[r] != cnt[0]) return false;
    if (cnt[0] == 0) return true;
    // compare each row's nonzero (col, value) sequence with row 0's
    std::vector<std::pair<int, double>> row0;
    size_t p = 0;
    const size_t k = ord.size();
    while (p < k && b.r[ord[p]] == 0) {
        const int j = ord[p++];
        if ((0.0 + b.v[j]) != 0.0) row0.push_back({b.c[j], 0.0 + b.v[j]});
    }
    for (int r = 1; r < bs; ++r) {
        size_t q = 0;
        while (p < k && b.r[ord[p]] == r) {
            const int j = ord[p++];
            const double val = 0.0 + b.v[j];
            if (val == 0.0) continue;
            if (q >= row0.size() || row0[q].first != b.c[j] ||
                !(row0[q].second == val))
                return false;
            ++q;
        }
        if (q != row0.size()) return false;
    }
    return true;
}

// coo2block_post (coo2block.h:154-380) for one block.
void encode_block(const HostCB &g, int64_t bid, const BlockIn &b, bool ext,
                  RowOut &out, int32_t &type, int32_t &nnz_out,
                  std::vector<int> &ord, std::vector<double> &dense) {
    const int bs = g.o.bs, bits = bits_of(bs);
    const int dense_thr = bs * bs * g.o.dense_sixteenths / 16;
    const int k = (int)b.r.size();
    const size_t u0 = out.u32.size(), f0 = out.f64.size();
    const bool coo = k <= kWave / 2 || (ext && k <= kWave);
    if (coo) {
        ord.resize(k);
        for (int j = 0; j < k; ++j) ord[j] = j;
        std::sort(ord.begin(), ord.end(), [&b](int l, int r) {
            if (b.r[l] != b.r[r]) return b.r[l] < b.r[r];
            return b.c[l] < b.c[r];
        });
        bool dup = false;
        const int32_t R = g.gb_row[bid];
        for (int q = 0; q < k; ++q) {
            const int j = ord[q];
            const uint32_t rr = (uint32_t)b.r[j], cc = (uint32_t)b.c[j];
            uint32_t idx;
            if (g.compact || g.direct) {
                const int32_t gathered = g.gb_col[bid] * bs + (int32_t)cc;
                const uint32_t oc =
                    (uint32_t)g.block_cols[g.block_cols_offset[R] + gathered];
                idx = g.compact ? ((rr << 12) | oc) : ((rr << 16) | oc);
            } else {
                idx = (rr << bits) | cc;
            }
            if (out.u32.size() > u0 && out.u32.back() == idx) {
                out.f64.back() += b.v[j];
                out.src.push_back(b.src[j]);
                out.src_cnt.back()++;
                dup = true;
            } else {
                out.u32.push_back(idx);
                out.f64.push_back(b.v[j]);
                out.src.push_back(b.src[j]);
                out.src_cnt.push_back(1);
            }
        }
        const int kk = (int)(out.u32.size() - u0);
        if (bs != 64 && ((g.direct && !g.compact) || bs == 32)) {
            const int rs = g.direct ? 16 : bits;
            const int ps = g.direct ? 16 + bits : 10;
            const uint32_t lm = g.direct ? (1u << (ps + 5)) : 0x8000u;
            const uint32_t mask = (uint32_t)bs - 1;
            uint32_t *p = out.u32.data() + u0;
            bool longrows = false;
            int s = 0;
            while (s < kk) {
                const uint32_t r0 = (p[s] >> rs) & mask;
                int e = s + 1;
                while (e < kk && ((p[e] >> rs) & mask) == r0) ++e;
                for (int q = 0; s + q < e; ++q) p[s + q] |= (uint32_t)(q << ps);
                longrows = longrows || (e - s) > 8;
                s = e;
            }
            if (longrows)
                for (int q = 0; q < kk; ++q) p[q] |= lm;
        }
        bool uni;
        if (dup) {
            dense.assign(bs * bs, 0.0);
            for (int j = 0; j < k; ++j) dense[b.r[j] * bs + b.c[j]] += b.v[j];
            uni = dense_uniform(dense, bs);
        } else {
            uni = sparse_uniform(b, ord, bs);
        }
        type = kCOO | (uni ? kUniform : 0);
        nnz_out = kk;
    } else if (k >= dense_thr) {
        dense.assign(bs * bs, 0.0);
        std::vector<int32_t> cnt(bs * bs + 1, 0);
        for (int j = 0; j < k; ++j) {
            dense[b.r[j] * bs + b.c[j]] += b.v[j];
            cnt[b.r[j] * bs + b.c[j] + 1]++;
        }
        out.f64.insert(out.f64.end(), dense.begin(), dense.end());
        for (int q = 0; q < bs * bs; ++q) out.src_cnt.push_back(cnt[q + 1]);
        for (int q = 0; q < bs * bs; ++q) cnt[q + 1] += cnt[q];
        const size_t s0 = out.src.size();
        out.src.resize(s0 + k);
        for (int j = 0; j < k; ++j)
            out.src[s0 + cnt[b.r[j] * bs + b.c[j]]++] = b.src[j];
        type = kDENSE | (dense_uniform(dense, bs) ? kUniform : 0);
        nnz_out = k;
    } else {
        std::vector<uint32_t> rp(bs + 1, 0), ci(k);
        std::vector<double> cv(k);
        std::vector<int32_t> cs(k);
        for (int j = 0; j < k; ++j) rp[b.r[j]]++;
        uint32_t sum = 0;
        for (int r = 0; r < bs; ++r) {
            const uint32_t t = rp[r];
            rp[r] = sum;
            sum += t;
        }
        rp[bs] = (uint32_t)k;
        std::vector<uint32_t> cur(rp);
        for (int j = 0; j < k; ++j) {
            const uint32_t d = cur[b.r[j]]++;
            ci[d] = (uint32_t)b.c[j];
            cv[d] = b.v[j];
            cs[d] = b.src[j];
        }
        bool uni = true;
        const uint32_t len0 = rp[1] - rp[0];
        for (int r = 1; r < bs && uni; ++r) {
            const uint32_t beg = rp[r], len = rp[r + 1] - beg;
            if (len != len0) {
                uni = false;
                break;
            }
            for (uint32_t q = 0; q < len; ++q)
                uni = uni && ci[beg + q] == ci[q] && cv[beg + q] == cv[q];
        }
        out.u32.insert(out.u32.end(), rp.begin(), rp.end());
        out.u32.insert(out.u32.end(), ci.begin(), ci.end());
        out.f64.insert(out.f64.end(), cv.begin(), cv.end());
        out.src.insert(out.src.end(), cs.begin(), cs.end());
        out.src_cnt.insert(out.src_cnt.end(), (size_t)k, 1);
        type = kCSR | (uni ? kUniform : 0);
        nnz_out = k;
    }
    out.u32_len.push_back((int64_t)(out.u32.size() - u0));
    out.f64_len.push_back((int64_t)(out.f64.size() - f0));
}

// Gathers each block row's nonzeros per block (pre_payload, coo2block.h:123-146)
// and calls fn(local block index, BlockIn) in block order.
template <class Fn>
void for_blocks_of_row(const HostCB &g, int64_t R, const std::vector<int64_t> &rs,
                       const std::vector<int64_t> &base,
                       const std::vector<int32_t> &lid, const int32_t *row,
                       const int32_t *colv, const double *val,
                       std::vector<int32_t> &cnt, std::vector<int32_t> &order,
                       BlockIn &b, Fn fn) {
    const int bs = g.o.bs;
    const int64_t s = rs[R], e = rs[R + 1];
    const int32_t nb = (int32_t)(base[R + 1] - base[R]);
    if (nb == 0) return;
    cnt.assign(nb + 1, 0);
    for (int64_t i = s; i < e; ++i) cnt[lid[i] + 1]++;
    for (int32_t j = 0; j < nb; ++j) cnt[j + 1] += cnt[j];
    order.resize(e - s);
    {
        std::vector<int32_t> cur(cnt.begin(), cnt.end() - 1);
        for (int64_t i = s; i < e; ++i) order[cur[lid[i]]++] = (int32_t)(i - s);
    }
    for (int32_t j = 0; j < nb; ++j) {
        b.clear();
        const int64_t bid = base[R] + j;
        const int32_t r0 = (int32_t)R * bs, c0 = g.gb_col[bid] * bs;
        for (int32_t q = cnt[j]; q < cnt[j + 1]; ++q) {
            const int64_t i = s + order[q];
            b.r.push_back(row[i] - r0);
            b.c.push_back(colv[i] - c0);
            b.v.push_back(val[i]);
            b.src.push_back((int32_t)i);
        }
        fn(j, b);
    }
}

void build_segments(HostCB &g) {  // coo2block.h:500-544
    const int W = g.o.waves;
    g.gb_row_ptr.assign(g.gb_m + 1, 0);
    for (int32_t r : g.gb_row) g.gb_row_ptr[r + 1]++;
    for (int64_t r = 0; r < g.gb_m; ++r) g.gb_row_ptr[r + 1] += g.gb_row_ptr[r];
    if (!g.o.row_owned) return;
    g.row_uniform.assign(g.gb_m, 1);
    std::vector<uint8_t> has(g.gb_m, 0);
    for (int64_t b = 0; b < g.nnzb; ++b) {
        const int32_t r = g.gb_row[b];
        has[r] = 1;
        g.row_uniform[r] = g.row_uniform[r] && (g.type_blk[b] & kUniform);
    }
    for (int64_t r = 0; r < g.gb_m; ++r) {
        const int32_t beg = g.gb_row_ptr[r], end = g.gb_row_ptr[r + 1];
        const bool uni = has[r] && g.row_uniform[r];
        const bool direct = g.nnz < 10000 || uni;
        const int32_t count =
            end == beg ? 0 : direct ? 1 : (end - beg + W - 1) / W;
        for (int32_t s = 0; s < count; ++s) {
            const int32_t sb = direct ? beg : beg + s * W;
            g.seg_rows.push_back((int32_t)r);
            g.seg_begin.push_back(sb);
            g.seg_end.push_back(direct ? end : std::min(sb + W, end));
            g.seg_direct.push_back(direct);
            g.seg_uniform.push_back(uni);
        }
    }
}

double load_stddev(const std::vector<int64_t> &loads) {
    double sum = 0;
    for (auto l : loads) sum += (double)l;
    const double mean = sum / (double)loads.size();
    double var = 0;
    for (auto l : loads) var += ((double)l - mean) * ((double)l - mean);
    return std::sqrt(var / (double)loads.size());
}

struct BlockIdx {  // BLOCK_IDX (format.h:34-48)
    int blk_nnz, origin_idx, end_idx;
};

// coo2block_banlance (coo2block.h:382-498).  std::sort with the reference's
// comparator keeps its order among blocks of equal nnz; the least-loaded
// queue is ordered by (load, index), a total order, so any heap agrees.
void balance(HostCB &g) {
    const int W = g.o.waves;
    const int64_t nb0 = g.nnzb;
    std::vector<BlockIdx> a(nb0);
    for (int64_t i = 0; i < nb0; ++i) a[i] = {g.nnz_blk[i], (int)i, 0};
    std::vector<int64_t> before((nb0 + W - 1) / W, 0);
    for (int64_t i = 0; i < nb0; ++i) before[i / W] += g.nnz_blk[i];
    g.sd_before = load_stddev(before);
    std::sort(a.begin(), a.end(),
              [](BlockIdx x, BlockIdx y) { return x.blk_nnz > y.blk_nnz; });
    int64_t nb = nb0;
    if (nb % W) {
        const int pad = W - (int)(nb % W);
        for (int q = 0; q < pad; ++q) a.push_back({0, INT_MAX, -1});
        nb += pad;
    }
    const int64_t ctas = nb / W;
    struct Item {
        int64_t total;
        int64_t index;
        int count;
        bool operator>(const Item &o) const {
            return total == o.total ? index > o.index : total > o.total;
        }
    };
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> pq;
    for (int64_t j = 0; j < ctas; ++j) pq.push({0, j, 0});
    for (int64_t i = 0; i < nb; ++i) {
        Item t = pq.top();
        pq.pop();
        a[i].end_idx = (int)(t.index * W + t.count);
        t.total += a[i].blk_nnz;
        t.count++;
        if (t.count < W) pq.push(t);
    }
    std::sort(a.begin(), a.end(),
              [](BlockIdx x, BlockIdx y) { return x.end_idx < y.end_idx; });
    std::vector<int32_t> r(nb), c(nb), k(nb), t(nb);
    for (int64_t i = 0; i < nb; ++i) {
        const int o = a[i].origin_idx;
        if (o != INT_MAX) {
            r[i] = g.gb_row[o];
            c[i] = g.gb_col[o];
            k[i] = g.nnz_blk[o];
            t[i] = g.type_blk[o];
        } else {
            r[i] = c[i] = -1;
            k[i] = 0;
            t[i] = kCOO;
        }
    }
    std::vector<int64_t> after(ctas, 0);
    for (int64_t i = 0; i < nb; ++i) after[i / W] += a[i].blk_nnz;
    g.sd_after = load_stddev(after);
    g.balanced = 1;
    g.nnzb = nb;
    g.gb_row.swap(r);
    g.gb_col.swap(c);
    g.nnz_blk.swap(k);
    g.type_blk.swap(t);
    g.bidx_origin.resize(nb);
    g.bidx_end.resize(nb);
    g.bidx_nnz.resize(nb);
    for (int64_t i = 0; i < nb; ++i) {
        g.bidx_origin[i] = a[i].origin_idx;
        g.bidx_end[i] = a[i].end_idx;
        g.bidx_nnz[i] = a[i].blk_nnz;
    }
}

// coo2block_build_flat_csr and coo2block_build_patterns (coo2block.h:546-602).
// Rows are already sorted, so the flat CSR is the input order.  Patterns get
// ids in order of first appearance; rows are matched through a hash of their
// sorted column list, with an exact comparison on every hash hit.
void build_patterns(HostCB &g, const int32_t *row, const int32_t *col) {
    const int64_t m = g.m;
    g.flat_row_ptr.assign(m + 1, 0);
    for (int64_t i = 0; i < g.nnz; ++i) g.flat_row_ptr[row[i] + 1]++;
    for (int64_t r = 0; r < m; ++r) g.flat_row_ptr[r + 1] += g.flat_row_ptr[r];
    g.flat_col.assign(col, col + g.nnz);
    std::vector<int32_t> sorted(g.flat_col);
    std::vector<uint64_t> hash(m);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < m; ++r) {
        int32_t *b = sorted.data() + g.flat_row_ptr[r];
        int32_t *e = sorted.data() + g.flat_row_ptr[r + 1];
        std::sort(b, e);
        uint64_t h = 1469598103934665603ull ^ (uint64_t)(e - b);
        for (int32_t *p = b; p < e; ++p) {
            h ^= (uint64_t)(uint32_t)*p;
            h *= 1099511628211ull;
            h ^= h >> 29;
        }
        hash[r] = h;
    }
    std::vector<int32_t> pid(m);
    std::vector<int64_t> rep;  // representative row of each pattern
    std::unordered_map<uint64_t, std::vector<int32_t>> seen;
    seen.reserve((size_t)m * 2 + 1);
    for (int64_t r = 0; r < m; ++r) {
        auto &cand = seen[hash[r]];
        const int64_t len = g.flat_row_ptr[r + 1] - g.flat_row_ptr[r];
        int32_t found = -1;
        for (int32_t p : cand) {
            const int64_t q = rep[p];
            const int64_t ql = g.flat_row_ptr[q + 1] - g.flat_row_ptr[q];
            if (ql == len &&
                std::equal(sorted.begin() + g.flat_row_ptr[r],
                           sorted.begin() + g.flat_row_ptr[r + 1],
                           sorted.begin() + g.flat_row_ptr[q])) {
                found = p;
                break;
            }
        }
        if (found < 0) {
            found = (int32_t)rep.size();
            rep.push_back(r);
            cand.push_back(found);
        }
        pid[r] = found;
    }
    const int64_t np = (int64_t)rep.size();
    g.pat_row_ptr.assign(np + 1, 0);
    g.pat_out_ptr.assign(np + 1, 0);
    for (int64_t p = 0; p < np; ++p) {
        const int64_t q = rep[p];
        g.pat_row_ptr[p + 1] = g.pat_row_ptr[p] +
            (int32_t)(g.flat_row_ptr[q + 1] - g.flat_row_ptr[q]);
    }
    for (int64_t r = 0; r < m; ++r) g.pat_out_ptr[pid[r] + 1]++;
    for (int64_t p = 0; p < np; ++p) g.pat_out_ptr[p + 1] += g.pat_out_ptr[p];
    g.pat_col.resize(g.pat_row_ptr[np]);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t p = 0; p < np; ++p) {
        const int64_t q = rep[p];
        std::copy(sorted.begin() + g.flat_row_ptr[q],
                  sorted.begin() + g.flat_row_ptr[q + 1],
                  g.pat_col.begin() + g.pat_row_ptr[p]);
    }
    g.pat_out_rows.resize(m);
    std::vector<int32_t> cur(g.pat_out_ptr.begin(), g.pat_out_ptr.end() - 1);
    for (int64_t r = 0; r < m; ++r) g.pat_out_rows[cur[pid[r]]++] = (int32_t)r;
}

template <class T>
int64_t put(const std::vector<T> &v, void *out) {
    if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(T));
    return (int64_t)v.size();
}

}  // namespace

std::string build_cb(const BuildOpts &o, int64_t m, int64_t n, int64_t nnz,
                     const int32_t *row, const int32_t *col, const double *val,
                     HostCB &g, int *code) {
    *code = CBSPMV_ERR_INVALID;
    if (o.bs != 16 && o.bs != 32) return "block_size must be 16 or 32";
    if (o.waves < 1 || o.waves > 1024) return "waves_per_block must be in [1, 1024]";
    if (o.dense_sixteenths < 1 || o.dense_sixteenths > 16)
        return "dense_sixteenths must be in [1, 16]";
    if (m < 0 || n < 0 || nnz < 0) return "negative size";
    if (m > INT_MAX || n > INT_MAX || nnz > INT_MAX)
        return "sizes are int32 in the reference's structure (m, n, nnz < 2^31)";
    if (nnz > 0 && (!row || !col || !val)) return "null COO array";
    *code = CBSPMV_ERR_BOUNDS;
    {
        int64_t bad = -1;
#pragma omp parallel for reduction(max : bad)
        for (int64_t i = 0; i < nnz; ++i)
            if (row[i] < 0 || row[i] >= m || col[i] < 0 || col[i] >= n)
                bad = std::max(bad, i);
        if (bad >= 0)
            return "COO entry " + std::to_string(bad) + " is outside the matrix";
    }
    *code = CBSPMV_ERR_UNSORTED;
    {
        int64_t bad = -1;
#pragma omp parallel for reduction(max : bad)
        for (int64_t i = 1; i < nnz; ++i)
            if (row[i] < row[i - 1]) bad = std::max(bad, i);
        if (bad >= 0)
            return "COO rows must be non-decreasing (entry " +
                   std::to_string(bad) + ")";
    }
    *code = CBSPMV_OK;

    g = HostCB();
    g.o = o;
    g.m = m;
    g.n = n;
    g.nnz = nnz;
    const int bs = o.bs;
    g.gb_m = (m + bs - 1) / bs;
    g.gb_n = (n + bs - 1) / bs;

    // entry range of every block row
    std::vector<int64_t> rs(g.gb_m + 1, nnz);
#pragma omp parallel for
    for (int64_t R = 0; R <= g.gb_m; ++R)
        rs[R] = std::lower_bound(row, row + nnz, (int32_t)std::min<int64_t>(
                                     R * bs, INT_MAX)) - row;

    std::vector<int32_t> lid, gcol;
    std::vector<int64_t> base;
    discover(g, rs, col, lid, base);
    // gather_flag (coo2block.h:63-75)
    {
        int64_t small = 0;
        for (int64_t i = 0; i < g.nnzb; ++i) small += g.nnz_blk[i] <= 8;
        g.super_sparse = small;
        g.analyzed = g.nnzb;
        g.ratio = g.nnzb > 0 ? small * 1.0 / g.nnzb : 0.0;
    }
    const int32_t *colv = col;
    if (nnz >= 10 && g.ratio > 0.15) {
        g.gather_flag = 1;
        gather_columns(g, rs, col, gcol);
        colv = gcol.data();
        discover(g, rs, colv, lid, base);
    }
    g.direct = g.gather_flag && n <= 65535;
    g.compact = g.direct && bs == 16 && n <= 4095 && nnz < 10000;

    // extend_coo_to_wave64 (coo2block.h:162-191)
    int64_t cand = 0, bal = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : cand, bal)
    for (int64_t R = 0; R < g.gb_m; ++R) {
        const int64_t s = rs[R], e = rs[R + 1];
        const int32_t nb = (int32_t)(base[R + 1] - base[R]);
        if (nb == 0) continue;
        // per block: entry count and per-row counts for 33..64-entry blocks
        std::vector<int32_t> rowcnt;
        bool any = false;
        for (int32_t j = 0; j < nb; ++j) {
            const int32_t k = g.nnz_blk[base[R] + j];
            any = any || (k > kWave / 2 && k <= kWave);
        }
        if (!any) continue;
        rowcnt.assign((size_t)nb * bs, 0);
        for (int64_t i = s; i < e; ++i)
            rowcnt[(size_t)lid[i] * bs + (row[i] - R * bs)]++;
        for (int32_t j = 0; j < nb; ++j) {
            const int32_t k = g.nnz_blk[base[R] + j];
            if (k <= kWave / 2 || k > kWave) continue;
            int lo = INT_MAX, hi = 0;
            for (int r = 0; r < bs; ++r) {
                const int c = rowcnt[(size_t)j * bs + r];
                if (c > 0) {
                    lo = std::min(lo, c);
                    hi = std::max(hi, c);
                }
            }
            cand++;
            bal += (hi - lo) <= 1;
        }
    }
    const bool ext = o.force_coo64 || (cand > 0 && bal * 2 < cand);

    // encode every block (coo2block_post), in parallel per block row
    std::vector<RowOut> rows(g.gb_m);
#pragma omp parallel
    {
        std::vector<int32_t> cnt, order;
        std::vector<int> ord;
        std::vector<double> dense;
        BlockIn b;
#pragma omp for schedule(dynamic, 16)
        for (int64_t R = 0; R < g.gb_m; ++R) {
            RowOut &out = rows[R];
            for_blocks_of_row(g, R, rs, base, lid, row, colv, val, cnt, order,
                              b, [&](int32_t j, const BlockIn &blk) {
                                  const int64_t bid = base[R] + j;
                                  int32_t type, nz;
                                  encode_block(g, bid, blk, ext, out, type, nz,
                                               ord, dense);
                                  g.type_blk[bid] = type;
                                  g.nnz_blk[bid] = nz;
                              });
        }
    }
    // flatten per-row outputs (per original block id)
    g.nnzb_orig = g.nnzb;
    std::vector<int64_t> ru(g.gb_m + 1, 0), rf(g.gb_m + 1, 0), rsrc(g.gb_m + 1, 0);
    for (int64_t R = 0; R < g.gb_m; ++R) {
        ru[R + 1] = ru[R] + (int64_t)rows[R].u32.size();
        rf[R + 1] = rf[R] + (int64_t)rows[R].f64.size();
        rsrc[R + 1] = rsrc[R] + (int64_t)rows[R].src.size();
    }
    g.pay_u32.resize(ru[g.gb_m]);
    g.pay_f64.resize(rf[g.gb_m]);
    g.src.resize(rsrc[g.gb_m]);
    g.src_ptr.assign(rf[g.gb_m] + 1, 0);
    g.u32_off.assign(g.nnzb + 1, 0);
    g.f64_off.assign(g.nnzb + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t R = 0; R < g.gb_m; ++R) {
        const RowOut &out = rows[R];
        std::copy(out.u32.begin(), out.u32.end(), g.pay_u32.begin() + ru[R]);
        std::copy(out.f64.begin(), out.f64.end(), g.pay_f64.begin() + rf[R]);
        std::copy(out.src.begin(), out.src.end(), g.src.begin() + rsrc[R]);
        int64_t s = rsrc[R];
        for (size_t v = 0; v < out.src_cnt.size(); ++v) {
            s += out.src_cnt[v];
            g.src_ptr[rf[R] + v + 1] = s;
        }
        int64_t u = ru[R], f = rf[R];
        for (size_t j = 0; j < out.u32_len.size(); ++j) {
            g.u32_off[base[R] + j] = u;
            g.f64_off[base[R] + j] = f;
            u += out.u32_len[j];
            f += out.f64_len[j];
        }
    }
    g.u32_off[g.nnzb] = ru[g.gb_m];
    g.f64_off[g.nnzb] = rf[g.gb_m];
    rows.clear();
    rows.shrink_to_fit();

    // unit-value detection (cb-spmv-dcu.hpp:1105-1127)
    {
        int unit = 1;
#pragma omp parallel for reduction(min : unit)
        for (int64_t b = 0; b < g.nnzb; ++b) {
            const int t = g.type_blk[b] & kTypeMask;
            for (int64_t v = g.f64_off[b]; v < g.f64_off[b + 1]; ++v) {
                const double x = g.pay_f64[v];
                if (!(x == 1.0 || (t == kDENSE && x == 0.0))) unit = 0;
            }
        }
        g.unit_values = unit;
    }

    build_segments(g);
    if (!o.row_owned && nnz >= 10000) {
        balance(g);
    } else {
        g.bidx_origin.resize(g.nnzb);
        g.bidx_end.resize(g.nnzb);
        g.bidx_nnz.resize(g.nnzb);
        for (int64_t i = 0; i < g.nnzb; ++i) {
            g.bidx_origin[i] = g.bidx_end[i] = (int32_t)i;
            g.bidx_nnz[i] = g.nnz_blk[i];
        }
    }
    build_patterns(g, row, col);
    return "";
}

int64_t export_array(const HostCB &g, const std::string &k, void *out) {
    if (k == "gb_row_idx") return put(g.gb_row, out);
    if (k == "gb_col_idx") return put(g.gb_col, out);
    if (k == "gb_row_ptr") return put(g.gb_row_ptr, out);
    if (k == "nnz_per_blk") return put(g.nnz_blk, out);
    if (k == "type_per_blk") return put(g.type_blk, out);
    if (k == "segment_rows") return put(g.seg_rows, out);
    if (k == "segment_begin") return put(g.seg_begin, out);
    if (k == "segment_end") return put(g.seg_end, out);
    if (k == "segment_direct") return put(g.seg_direct, out);
    if (k == "segment_uniform") return put(g.seg_uniform, out);
    if (k == "block_row_uniform") return put(g.row_uniform, out);
    if (k == "flat_row_ptr") return put(g.flat_row_ptr, out);
    if (k == "flat_col_idx") return put(g.flat_col, out);
    if (k == "pattern_row_ptr") return put(g.pat_row_ptr, out);
    if (k == "pattern_col_idx") return put(g.pat_col, out);
    if (k == "pattern_output_ptr") return put(g.pat_out_ptr, out);
    if (k == "pattern_output_rows") return put(g.pat_out_rows, out);
    if (k == "block_cols_offset") return put(g.block_cols_offset, out);
    if (k == "block_cols") return put(g.block_cols, out);
    if (k == "bidx_origin") return put(g.bidx_origin, out);
    if (k == "bidx_end") return put(g.bidx_end, out);
    if (k == "bidx_nnz") return put(g.bidx_nnz, out);
    // payload in FINAL block order, as the reference packs it
    // (cb-spmv-dcu.hpp:1282-1346)
    if (k == "pay_u32" || k == "pay_f64" || k == "pay_u32_off" ||
        k == "pay_f64_off") {
        const bool is_u32 = k == "pay_u32" || k == "pay_u32_off";
        const bool offs = k == "pay_u32_off" || k == "pay_f64_off";
        const std::vector<int64_t> &off = is_u32 ? g.u32_off : g.f64_off;
        int64_t total = 0;
        std::vector<int64_t> o(g.nnzb + 1, 0);
        for (int64_t i = 0; i < g.nnzb; ++i) {
            const int32_t org = g.bidx_origin[i];
            const int64_t len = (g.nnz_blk[i] > 0 && org != INT_MAX)
                                    ? off[org + 1] - off[org]
                                    : 0;
            o[i] = total;
            total += len;
        }
        o[g.nnzb] = total;
        if (offs) return put(o, out);
        if (out) {
            for (int64_t i = 0; i < g.nnzb; ++i) {
                const int64_t len = o[i + 1] - o[i];
                if (!len) continue;
                const int32_t org = g.bidx_origin[i];
                if (is_u32)
                    std::memcpy((uint32_t *)out + o[i],
                                g.pay_u32.data() + off[org], len * 4);
                else
                    std::memcpy((double *)out + o[i],
                                g.pay_f64.data() + off[org], len * 8);
            }
        }
        return total;
    }
    return -1;
}

}  // namespace cb
