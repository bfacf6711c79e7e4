// ORACLE — test infrastructure, not product code.
//
// A deliberately plain, serial CPU restatement of the reference's CB-SpMV
// algorithm (xing-cong/CB-Sparse-DCU, cb-spmv-dcu/src/), used only by tests/,
// __graft_entry__.smoke() and the CPU-baseline leg of bench.py to CHECK the
// product.  It is pinned against the reference's own host code compiled from
// its headers (oracle/ref_driver.cpp -> oracle/_ref/) and against the golden
// fixtures under tests/golden/.
//
// Contents
//   * CB build: coo2block_gather (coo2block.h:628-670) and every step it calls,
//     with the reference's compile-time macros (macros.h:38-97) as run-time
//     options.  Output is exposed through the same cbdump_* ABI as
//     oracle/ref_driver.cpp so arrays can be compared one by one.
//   * The reference's CPU SpMV loop (utils.h:98-111), in double (as written)
//     and in long double with per-row absolute sums for tolerance checks.
//   * A decoder that evaluates y from the CB structure exactly as the device
//     kernels interpret it (cb-spmv-dcu.hpp:159-1084), to pin the meaning of
//     every index encoding.
//   * Adjoint references: g_x = A^T g and g_vals[k] = g[row_k] * x[col_k].
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

enum { kCOO = 0, kCSR = 1, kDENSE = 3, kTypeMask = 0x7f, kUniform = 0x80 };
constexpr int kWave = 64;  // the reference's wavefront (macros.h:77-78)

struct Opts {
    int bs = 16;               // CB_BLOCK_SIZE (macros.h:38)
    int row_owned = 1;         // CB_ROW_OWNED (Makefile:6)
    int waves = 4;             // CB_WAVES_PER_BLOCK (Makefile:5)
    int dense_sixteenths = 15; // CB_DENSE_SIXTEENTHS (macros.h:93)
    int force_coo64 = 0;       // CB_FORCE_COO64 (macros.h:90)
    int bits() const {
        int b = 0;
        while ((1 << b) < bs) ++b;
        return b;
    }
};

struct OrigBlock {  // COO_BLOCK_ORIG (format.h:12-18)
    std::vector<int> r, c;
    std::vector<double> v;
};
struct Payload {  // one finished block, in reference units
    std::vector<uint32_t> u32;  // COO idx | CSR row_ptr then col_idx
    std::vector<double> f64;    // values (DENSE: bs*bs row-major)
};
struct BlockIdx {  // BLOCK_IDX (format.h:34-48)
    int blk_nnz, origin_idx, end_idx;
};

struct CB {
    Opts o;
    int64_t m = 0, n = 0, nnz = 0, gb_m = 0, gb_n = 0, nnzb = 0;
    int gather_flag = 0, direct = 0, compact = 0, balanced = 0;
    int64_t super_sparse = 0, analyzed = 0;
    double ratio = 0, sd_before = 0, sd_after = 0;
    std::vector<int> gb_row, gb_col, gb_row_ptr, nnz_blk, type_blk;
    std::vector<int> seg_rows, seg_begin, seg_end, seg_direct, seg_uniform,
        row_uniform;
    std::vector<int> flat_row_ptr, flat_col, pat_row_ptr, pat_col, pat_out_ptr,
        pat_out_rows;
    std::vector<int> block_cols_offset, block_cols;
    std::vector<BlockIdx> bidx;
    std::vector<OrigBlock> orig;
    std::vector<Payload> pay;  // indexed by ORIGINAL (pre-balance) block id
    // flattened dump in final block order
    std::vector<uint32_t> d_u32;
    std::vector<double> d_f64;
    std::vector<int64_t> d_u32_off, d_f64_off;
    std::vector<int> d_origin, d_end, d_nnz;
};

// coo2block_pre_metadata (coo2block.h:77-121): blocks in first-touch order.
void pre_metadata(CB &g, const int *row, const int *col,
                  std::vector<int> &ids) {
    const int bs = g.o.bs;
    std::unordered_map<long long, int> map;
    ids.resize(g.nnz);
    for (int64_t i = 0; i < g.nnz; ++i) {
        const int bi = row[i] / bs, bj = col[i] / bs;
        const long long key = (long long)bi * g.gb_n + bj;
        auto it = map.find(key);
        int id;
        if (it == map.end()) {
            id = (int)g.nnzb++;
            map.emplace(key, id);
            g.gb_row.push_back(bi);
            g.gb_col.push_back(bj);
            g.nnz_blk.push_back(1);
            g.type_blk.push_back(kCOO);
        } else {
            id = it->second;
            g.nnz_blk[id]++;
        }
        ids[i] = id;
    }
}

// coo2block_pre_payload (coo2block.h:123-146)
void pre_payload(CB &g, const int *row, const int *col, const double *val,
                 const std::vector<int> &ids) {
    const int bs = g.o.bs;
    g.orig.assign(g.nnzb, OrigBlock());
    for (int64_t i = 0; i < g.nnz; ++i) {
        OrigBlock &b = g.orig[ids[i]];
        b.r.push_back(row[i] - g.gb_row[ids[i]] * bs);
        b.c.push_back(col[i] - g.gb_col[ids[i]] * bs);
        b.v.push_back(val[i]);
    }
}

// gather_flag (coo2block.h:63-75)
bool gather_decision(CB &g) {
    int64_t small = 0;
    for (int64_t i = 0; i < g.nnzb; ++i) small += g.nnz_blk[i] <= 8;
    g.super_sparse = small;
    g.analyzed = g.nnzb;
    g.ratio = g.nnzb > 0 ? small * 1.0 / g.nnzb : 0.0;
    return g.nnz >= 10 && g.ratio > 0.15;
}

// gather (coo2block.h:7-61): per block row, sorted unique original columns;
// every nonzero's column becomes its position in that list.
void gather_columns(CB &g, const int *row, const int *col,
                    std::vector<int> &gcol) {
    const int bs = g.o.bs;
    std::vector<std::vector<int>> lists(g.gb_m);
    for (int64_t i = 0; i < g.nnz; ++i) lists[row[i] / bs].push_back(col[i]);
    for (auto &l : lists) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
    }
    gcol.resize(g.nnz);
    for (int64_t i = 0; i < g.nnz; ++i) {
        const auto &l = lists[row[i] / bs];
        gcol[i] = (int)(std::lower_bound(l.begin(), l.end(), col[i]) -
                        l.begin());
    }
    g.block_cols_offset.assign(g.gb_m + 1, 0);
    for (int64_t r = 0; r < g.gb_m; ++r)
        g.block_cols_offset[r + 1] = g.block_cols_offset[r] + (int)lists[r].size();
    g.block_cols.clear();
    for (auto &l : lists) g.block_cols.insert(g.block_cols.end(), l.begin(), l.end());
}

bool rows_uniform(const std::vector<double> &dense, int bs) {
    for (int r = 1; r < bs; ++r)
        for (int c = 0; c < bs; ++c)
            if (!(dense[r * bs + c] == dense[c])) return false;
    return true;
}

// coo2block_post (coo2block.h:154-380): per-block format choice and encoding.
void post(CB &g) {
    const int bs = g.o.bs, bits = g.o.bits();
    const int dense_thr = bs * bs * g.o.dense_sixteenths / 16;
    g.direct = g.gather_flag && g.n <= 65535;
    g.compact = g.direct && bs == 16 && g.n <= 4095 && g.nnz < 10000;
    int cand = 0, bal = 0;
    for (const OrigBlock &b : g.orig) {
        const int k = (int)b.r.size();
        if (k <= kWave / 2 || k > kWave) continue;
        std::vector<int> cnt(bs, 0);
        for (int r : b.r) cnt[r]++;
        int lo = INT_MAX, hi = 0;
        for (int r = 0; r < bs; ++r)
            if (cnt[r] > 0) {
                lo = std::min(lo, cnt[r]);
                hi = std::max(hi, cnt[r]);
            }
        cand++;
        bal += (hi - lo) <= 1;
    }
    const bool ext = g.o.force_coo64 || (cand > 0 && bal * 2 < cand);
    g.pay.assign(g.nnzb, Payload());
    for (int64_t i = 0; i < g.nnzb; ++i) {
        const OrigBlock &b = g.orig[i];
        const int k = (int)b.r.size();
        Payload &p = g.pay[i];
        std::vector<double> dense(bs * bs, 0.0);
        for (int j = 0; j < k; ++j) dense[b.r[j] * bs + b.c[j]] += b.v[j];
        const bool coo = k <= kWave / 2 || (ext && k <= kWave);
        if (coo) {
            std::vector<int> order(k);
            for (int j = 0; j < k; ++j) order[j] = j;
            std::sort(order.begin(), order.end(), [&b](int l, int r) {
                if (b.r[l] != b.r[r]) return b.r[l] < b.r[r];
                return b.c[l] < b.c[r];
            });
            for (int j : order) {
                const uint32_t rr = (uint32_t)b.r[j], cc = (uint32_t)b.c[j];
                uint32_t idx;
                if (g.compact || g.direct) {
                    const int gathered = g.gb_col[i] * bs + (int)cc;
                    const uint32_t oc = (uint32_t)g.block_cols[
                        g.block_cols_offset[g.gb_row[i]] + gathered];
                    idx = g.compact ? ((rr << 12) | oc) : ((rr << 16) | oc);
                } else {
                    idx = (rr << bits) | cc;
                }
                if (!p.u32.empty() && p.u32.back() == idx) {
                    p.f64.back() += b.v[j];
                } else {
                    p.u32.push_back(idx);
                    p.f64.push_back(b.v[j]);
                }
            }
            const int kk = (int)p.u32.size();
            if (bs != 64 && ((g.direct && !g.compact) || bs == 32)) {
                const int rs = g.direct ? 16 : bits;
                const int ps = g.direct ? 16 + bits : 10;
                const uint32_t lm = g.direct ? (1u << (ps + 5)) : 0x8000u;
                const uint32_t mask = (uint32_t)bs - 1;
                bool longrows = false;
                int s = 0;
                while (s < kk) {
                    const uint32_t r0 = (p.u32[s] >> rs) & mask;
                    int e = s + 1;
                    while (e < kk && ((p.u32[e] >> rs) & mask) == r0) ++e;
                    for (int q = 0; s + q < e; ++q) p.u32[s + q] |= (uint32_t)(q << ps);
                    longrows = longrows || (e - s) > 8;
                    s = e;
                }
                if (longrows)
                    for (auto &x : p.u32) x |= lm;
            }
            g.type_blk[i] = kCOO | (rows_uniform(dense, bs) ? kUniform : 0);
            g.nnz_blk[i] = kk;
        } else if (g.nnz_blk[i] >= dense_thr) {
            p.f64 = dense;
            g.type_blk[i] = kDENSE | (rows_uniform(dense, bs) ? kUniform : 0);
        } else {
            std::vector<uint32_t> rp(bs + 1, 0), ci(k);
            std::vector<double> cv(k);
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
            p.u32 = rp;
            p.u32.insert(p.u32.end(), ci.begin(), ci.end());
            p.f64 = cv;
            g.type_blk[i] = kCSR | (uni ? kUniform : 0);
        }
    }
}

void build_row_ptr(CB &g) {  // coo2block.h:500-508
    g.gb_row_ptr.assign(g.gb_m + 1, 0);
    for (int r : g.gb_row) g.gb_row_ptr[r + 1]++;
    for (int64_t r = 0; r < g.gb_m; ++r) g.gb_row_ptr[r + 1] += g.gb_row_ptr[r];
}

void build_segments(CB &g) {  // coo2block.h:510-544
    const int W = g.o.waves;
    g.row_uniform.assign(g.gb_m, 1);
    std::vector<int> has(g.gb_m, 0);
    for (int64_t b = 0; b < g.nnzb; ++b) {
        const int r = g.gb_row[b];
        has[r] = 1;
        g.row_uniform[r] = g.row_uniform[r] && (g.type_blk[b] & kUniform);
    }
    for (int64_t r = 0; r < g.gb_m; ++r) {
        const int beg = g.gb_row_ptr[r], end = g.gb_row_ptr[r + 1];
        const bool uni = has[r] && g.row_uniform[r];
        const bool direct = g.nnz < 10000 || uni;
        const int count = end == beg ? 0 : direct ? 1 : (end - beg + W - 1) / W;
        for (int s = 0; s < count; ++s) {
            const int sb = direct ? beg : beg + s * W;
            g.seg_rows.push_back((int)r);
            g.seg_begin.push_back(sb);
            g.seg_end.push_back(direct ? end : std::min(sb + W, end));
            g.seg_direct.push_back(direct);
            g.seg_uniform.push_back(uni);
        }
    }
}

double load_stddev(const std::vector<long long> &loads) {
    double sum = 0;
    for (auto l : loads) sum += (double)l;
    const double mean = sum / loads.size();
    double var = 0;
    for (auto l : loads) var += (l - mean) * (l - mean);
    return std::sqrt(var / loads.size());
}

// coo2block_banlance (coo2block.h:382-498): sort blocks by nnz (descending,
// std::sort as the reference does, so ties fall the same way), pad to a
// multiple of W, then greedy least-loaded assignment of W blocks per CTA.
void balance(CB &g) {
    const int W = g.o.waves;
    const int64_t nb0 = g.nnzb;
    std::vector<BlockIdx> a(nb0);
    for (int64_t i = 0; i < nb0; ++i) a[i] = {g.nnz_blk[i], (int)i, 0};
    std::vector<long long> before((nb0 + W - 1) / W, 0);
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
    // min-heap on (total, index); both fields make the order total
    std::vector<long long> total(ctas, 0);
    std::vector<int> count(ctas, 0);
    std::map<std::pair<long long, int64_t>, int> heap;
    for (int64_t j = 0; j < ctas; ++j) heap[{0, j}] = 1;
    for (int64_t i = 0; i < nb; ++i) {
        auto it = heap.begin();
        const int64_t j = it->first.second;
        heap.erase(it);
        a[i].end_idx = (int)(j * W + count[j]);
        total[j] += a[i].blk_nnz;
        count[j]++;
        if (count[j] < W) heap[{total[j], j}] = 1;
    }
    std::sort(a.begin(), a.end(),
              [](BlockIdx x, BlockIdx y) { return x.end_idx < y.end_idx; });
    std::vector<int> r(nb), c(nb), k(nb), t(nb);
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
    std::vector<long long> after(ctas, 0);
    for (int64_t i = 0; i < nb; ++i) after[i / W] += a[i].blk_nnz;
    g.sd_after = load_stddev(after);
    g.balanced = 1;
    g.nnzb = nb;
    g.gb_row = r;
    g.gb_col = c;
    g.nnz_blk = k;
    g.type_blk = t;
    g.bidx = a;
}

void build_flat_csr(CB &g, const int *row, const int *col) {  // :546-561
    g.flat_row_ptr.assign(g.m + 1, 0);
    g.flat_col.resize(g.nnz);
    for (int64_t i = 0; i < g.nnz; ++i) g.flat_row_ptr[row[i] + 1]++;
    for (int64_t r = 0; r < g.m; ++r) g.flat_row_ptr[r + 1] += g.flat_row_ptr[r];
    std::vector<int> cur(g.flat_row_ptr);
    for (int64_t i = 0; i < g.nnz; ++i) g.flat_col[cur[row[i]]++] = col[i];
}

void build_patterns(CB &g) {  // :566-602, first-appearance pattern ids
    std::map<std::vector<int>, int> ids;
    std::vector<std::vector<int>> cols, rows;
    for (int64_t r = 0; r < g.m; ++r) {
        std::vector<int> c(g.flat_col.begin() + g.flat_row_ptr[r],
                           g.flat_col.begin() + g.flat_row_ptr[r + 1]);
        std::sort(c.begin(), c.end());
        auto ins = ids.emplace(c, (int)cols.size());
        if (ins.second) {
            cols.push_back(c);
            rows.emplace_back();
        }
        rows[ins.first->second].push_back((int)r);
    }
    g.pat_row_ptr.assign(cols.size() + 1, 0);
    g.pat_out_ptr.assign(cols.size() + 1, 0);
    for (size_t p = 0; p < cols.size(); ++p) {
        g.pat_col.insert(g.pat_col.end(), cols[p].begin(), cols[p].end());
        g.pat_out_rows.insert(g.pat_out_rows.end(), rows[p].begin(), rows[p].end());
        g.pat_row_ptr[p + 1] = (int)g.pat_col.size();
        g.pat_out_ptr[p + 1] = (int)g.pat_out_rows.size();
    }
}

void flatten(CB &g) {
    g.d_u32_off.assign(g.nnzb + 1, 0);
    g.d_f64_off.assign(g.nnzb + 1, 0);
    for (int64_t i = 0; i < g.nnzb; ++i) {
        g.d_u32_off[i] = (int64_t)g.d_u32.size();
        g.d_f64_off[i] = (int64_t)g.d_f64.size();
        if (g.nnz_blk[i] <= 0) continue;
        const Payload &p = g.pay[g.bidx[i].origin_idx];
        g.d_u32.insert(g.d_u32.end(), p.u32.begin(), p.u32.end());
        g.d_f64.insert(g.d_f64.end(), p.f64.begin(), p.f64.end());
    }
    g.d_u32_off[g.nnzb] = (int64_t)g.d_u32.size();
    g.d_f64_off[g.nnzb] = (int64_t)g.d_f64.size();
    for (const BlockIdx &b : g.bidx) {
        g.d_origin.push_back(b.origin_idx);
        g.d_end.push_back(b.end_idx);
        g.d_nnz.push_back(b.blk_nnz);
    }
}

// coo2block_gather (coo2block.h:628-670)
CB *build(const Opts &o, int m, int n, int64_t nnz, const int *row,
          const int *col, const double *val) {
    CB *gp = new CB;
    CB &g = *gp;
    g.o = o;
    g.m = m;
    g.n = n;
    g.nnz = nnz;
    g.gb_m = (m + o.bs - 1) / o.bs;
    g.gb_n = (n + o.bs - 1) / o.bs;
    std::vector<int> ids;
    pre_metadata(g, row, col, ids);
    if (gather_decision(g)) {
        std::vector<int> gcol;
        gather_columns(g, row, col, gcol);
        // GLOBAL_BLOCK::reset (format.h:115-183) keeps only the gather
        // statistics and the column lists
        g.nnzb = 0;
        g.gb_row.clear();
        g.gb_col.clear();
        g.nnz_blk.clear();
        g.type_blk.clear();
        g.gather_flag = 1;
        pre_metadata(g, row, gcol.data(), ids);
        pre_payload(g, row, gcol.data(), val, ids);
        post(g);
    } else {
        pre_payload(g, row, col, val, ids);
        post(g);
    }
    build_row_ptr(g);
    if (o.row_owned) build_segments(g);
    if (!o.row_owned && nnz >= 10000) {
        balance(g);
    } else {
        g.bidx.resize(g.nnzb);
        for (int64_t i = 0; i < g.nnzb; ++i)
            g.bidx[i] = {g.nnz_blk[i], (int)i, (int)i};
    }
    build_flat_csr(g, row, col);
    build_patterns(g);
    flatten(g);
    return gp;
}

template <class T>
int64_t put(const std::vector<T> &v, void *out) {
    if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(T));
    return (int64_t)v.size();
}

}  // namespace

extern "C" {

void *oracle_build(int bs, int row_owned, int waves, int dense_sixteenths,
                   int force_coo64, int m, int n, int64_t nnz, const int *row,
                   const int *col, const double *val) {
    Opts o;
    o.bs = bs;
    o.row_owned = row_owned;
    o.waves = waves;
    o.dense_sixteenths = dense_sixteenths;
    o.force_coo64 = force_coo64;
    if (bs < 2 || bs > 64 || (bs & (bs - 1))) return nullptr;
    return build(o, m, n, nnz, row, col, val);
}

void cbdump_free(void *h) { delete static_cast<CB *>(h); }

void cbdump_scalars(void *h, int64_t *out12, double *out3) {
    const CB &g = *static_cast<CB *>(h);
    const int64_t s[12] = {g.m, g.n, g.nnz, g.gb_m, g.gb_n, g.nnzb,
                           g.gather_flag, g.direct, g.compact, g.super_sparse,
                           g.analyzed, g.balanced};
    std::memcpy(out12, s, sizeof(s));
    out3[0] = g.ratio;
    out3[1] = g.sd_before;
    out3[2] = g.sd_after;
}

int64_t cbdump_array(void *h, const char *name, void *out) {
    CB &g = *static_cast<CB *>(h);
    const std::string k(name);
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
    if (k == "bidx_origin") return put(g.d_origin, out);
    if (k == "bidx_end") return put(g.d_end, out);
    if (k == "bidx_nnz") return put(g.d_nnz, out);
    if (k == "pay_u32") return put(g.d_u32, out);
    if (k == "pay_f64") return put(g.d_f64, out);
    if (k == "pay_u32_off") return put(g.d_u32_off, out);
    if (k == "pay_f64_off") return put(g.d_f64_off, out);
    return -1;
}

// y = A x by the reference's serial COO loop (utils.h:98-111), in double and
// in input order, as written.
void oracle_spmv_coo(int m, int64_t nnz, const int *row, const int *col,
                     const double *val, const double *x, double *y) {
    for (int i = 0; i < m; ++i) y[i] = 0.0;
    for (int64_t k = 0; k < nnz; ++k) y[row[k]] += val[k] * x[col[k]];
}

// Y = A X for nrhs right-hand sides (column-major, leading dims ldx/ldy) in
// long double, plus absrow[i * nrhs + j] = sum_k |a_ik x_kj| for tolerances.
void oracle_spmm_coo_ld(int m, int64_t nnz, const int *row, const int *col,
                        const double *val, int nrhs, const double *x,
                        int64_t ldx, double *y, int64_t ldy, double *absrow) {
    std::vector<long double> acc((size_t)m * nrhs, 0.0L), aa((size_t)m * nrhs, 0.0L);
    for (int64_t k = 0; k < nnz; ++k)
        for (int j = 0; j < nrhs; ++j) {
            const long double t = (long double)val[k] * x[(int64_t)j * ldx + col[k]];
            acc[(size_t)j * m + row[k]] += t;
            aa[(size_t)j * m + row[k]] += std::fabs(t);
        }
    for (int j = 0; j < nrhs; ++j)
        for (int i = 0; i < m; ++i) {
            y[(int64_t)j * ldy + i] = (double)acc[(size_t)j * m + i];
            if (absrow) absrow[(int64_t)j * m + i] = (double)aa[(size_t)j * m + i];
        }
}

// g_x = A^T g in long double (adjoint reference), same layout conventions.
void oracle_spmm_t_coo_ld(int n, int64_t nnz, const int *row, const int *col,
                          const double *val, int nrhs, const double *g,
                          int64_t ldg, double *gx, int64_t ldgx, double *absrow) {
    std::vector<long double> acc((size_t)n * nrhs, 0.0L), aa((size_t)n * nrhs, 0.0L);
    for (int64_t k = 0; k < nnz; ++k)
        for (int j = 0; j < nrhs; ++j) {
            const long double t = (long double)val[k] * g[(int64_t)j * ldg + row[k]];
            acc[(size_t)j * n + col[k]] += t;
            aa[(size_t)j * n + col[k]] += std::fabs(t);
        }
    for (int j = 0; j < nrhs; ++j)
        for (int i = 0; i < n; ++i) {
            gx[(int64_t)j * ldgx + i] = (double)acc[(size_t)j * n + i];
            if (absrow) absrow[(int64_t)j * n + i] = (double)aa[(size_t)j * n + i];
        }
}

// d(0.5||AX - T||^2)/d val_k summed over right-hand sides, with G = AX - T
// given:  gval[k] = sum_j G[row_k, j] * X[col_k, j]   (input nonzero order)
void oracle_grad_vals(int64_t nnz, const int *row, const int *col, int nrhs,
                      const double *g, int64_t ldg, const double *x,
                      int64_t ldx, double *gval) {
    for (int64_t k = 0; k < nnz; ++k) {
        long double s = 0;
        for (int j = 0; j < nrhs; ++j)
            s += (long double)g[(int64_t)j * ldg + row[k]] * x[(int64_t)j * ldx + col[k]];
        gval[k] = (double)s;
    }
}

// Evaluates y from a CB dump the way the device kernels read it
// (cb-spmv-dcu.hpp:328-578 COO/CSR/DENSE; :807-816 gather lookups; compact
// u16 (row<<12|col), direct (row<<16|col) and standard (row<<bits|col)
// encodings).  Works on any cbdump handle's arrays passed in explicitly, so it
// can decode the reference's own structure.
int oracle_cb_decode_spmv(int bs, int64_t m, int64_t nnzb, int gather_flag,
                          int direct, int compact, const int *gb_row,
                          const int *gb_col, const int *nnz_blk,
                          const int *type_blk, const int *block_cols_offset,
                          const int *block_cols, const uint32_t *pay_u32,
                          const int64_t *u32_off, const double *pay_f64,
                          const int64_t *f64_off, const double *x, double *y) {
    int bits = 0;
    while ((1 << bits) < bs) ++bits;
    const uint32_t mask = (uint32_t)bs - 1;
    std::vector<long double> acc(m, 0.0L);
    auto xcol = [&](int64_t b, uint32_t local) -> double {
        if (!gather_flag) return x[(int64_t)gb_col[b] * bs + local];
        return x[block_cols[block_cols_offset[gb_row[b]] +
                            (int64_t)gb_col[b] * bs + local]];
    };
    for (int64_t b = 0; b < nnzb; ++b) {
        if (nnz_blk[b] <= 0) continue;
        const int type = type_blk[b] & kTypeMask;
        const uint32_t *u = pay_u32 + u32_off[b];
        const double *v = pay_f64 + f64_off[b];
        const int64_t r0 = (int64_t)gb_row[b] * bs;
        if (type == kCOO) {
            for (int k = 0; k < nnz_blk[b]; ++k) {
                uint32_t r, c;
                double xv;
                if (compact) {
                    r = (u[k] >> 12) & mask;
                    c = u[k] & 0xfff;
                    xv = x[c];
                } else if (direct) {
                    r = (u[k] >> 16) & mask;
                    c = u[k] & 0xffff;
                    xv = x[c];
                } else {
                    r = (u[k] >> bits) & mask;
                    c = u[k] & mask;
                    xv = xcol(b, c);
                }
                if (r0 + r < m) acc[r0 + r] += (long double)v[k] * xv;
            }
        } else if (type == kCSR) {
            const uint32_t *rp = u, *ci = u + bs + 1;
            for (int r = 0; r < bs; ++r)
                for (uint32_t k = rp[r]; k < rp[r + 1]; ++k)
                    if (r0 + r < m) acc[r0 + r] += (long double)v[k] * xcol(b, ci[k]);
        } else if (type == kDENSE) {
            const int64_t width = gather_flag
                ? block_cols_offset[gb_row[b] + 1] - block_cols_offset[gb_row[b]]
                : INT64_MAX;
            for (int r = 0; r < bs; ++r)
                for (int c = 0; c < bs; ++c) {
                    if ((int64_t)gb_col[b] * bs + c >= width) continue;
                    if (v[r * bs + c] != 0.0 && r0 + r < m)
                        acc[r0 + r] += (long double)v[r * bs + c] * xcol(b, c);
                }
        } else {
            return -1;
        }
    }
    for (int64_t i = 0; i < m; ++i) y[i] = (double)acc[i];
    return 0;
}

}  // extern "C"
