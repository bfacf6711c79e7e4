// sm_100a multi-right-hand-side CB-SpMV and batches: Y = A X with X (n x nrhs)
// and Y (m x nrhs) row-major (leading dimensions ldx, ldy), over the same tile
// layout as the single-vector kernels (cb_kernels.cu); a batch runs many such
// products in one launch.
//
// cb_mstream_kernel: persistent warps take units of consecutive tiles (of one
// matrix, or of a batch's concatenated tile list) from a counter, one unit
// ahead, and double-buffer whole tile payloads -- COO section, CSR and DENSE
// payloads -- in shared memory with bulk asynchronous copies (TMA, no
// multicast): the next tiles are in flight while one is computed from shared
// memory.  Tile payloads are capped in size by the packer so two fit per warp.
//
// A lane carries V consecutive right-hand sides (4 FP32 / 2 FP64 values, one
// vector load of an x row where the layout allows it) and RL lanes share an
// entry, RL * V covering nrhs (more right-hand sides take several passes over
// the staged tile); G = 32 / RL entries per warp step.  The per-entry work --
// index decode, row runs, accumulator update -- is done once per V values.
// COO x gathers run one chunk ahead of the chunk being added up; CSR/DENSE
// blocks stage their x rows for up to 8 / RL blocks at a time.  Accumulators
// are lane-private (V values per lane and row); consecutive tiles of one block
// row inside a warp's range keep adding into them.

// Block rows split over several tiles: a row whose tiles all lie in one
// warp's range is stored directly; otherwise each warp's run leaves its sums
// in the slot of its first tile and the last run to arrive on the row's
// counter adds them in tile order.  No tile waits on another.  Every mbarrier
// wait is bounded; on give-up the error word is set and the warp stops after
// draining its own copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "cb_device.cuh"
#include "cb_kernels.hpp"

namespace cb {
namespace {

using dev::a16;
using dev::add_entries;
using dev::bulk_g2s;
using dev::dense_at;
using dev::fence_mbar_init;
using dev::fence_proxy_async;
using dev::kColMask;
using dev::kFull;
using dev::mbar_arrive;
using dev::mbar_arrive_tx;
using dev::mbar_init;
using dev::mbar_wait;
using dev::policy_evict_first;

constexpr int kMsWarps = 4;  // warps per CTA

// Per-warp shared memory: [acc | xt | mbar[2] | buf[2]], buf = `cap` bytes.
// acc: V values per lane and row (lane l, row r at acc[(r * 32 + l) * V]);
// xt: x rows of up to XB CSR/DENSE blocks, RL * V values per column.
template <typename T, int BS, int RL, int V>
struct MsLayout {
    static constexpr int XB = RL >= 8 ? 1 : 8 / RL;
    static constexpr uint32_t acc_bytes = BS * 32 * V * sizeof(T);
    static constexpr uint32_t xt_bytes = XB * BS * RL * V * sizeof(T);
    static constexpr uint32_t head = a16(acc_bytes + xt_bytes + 16);
    __host__ __device__ static uint32_t bytes(uint32_t cap) { return head + 2 * cap; }
};

// V consecutive values: one vector load where the layout allows it
template <typename T, int V>
__device__ __forceinline__ void ldg_v(const T *p, T *o) {
    if constexpr (V == 4 && sizeof(T) == 4) {
        const float4 f = __ldg(reinterpret_cast<const float4 *>(p));
        o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = f.w;
    } else if constexpr (V == 2 && sizeof(T) == 4) {
        const float2 f = __ldg(reinterpret_cast<const float2 *>(p));
        o[0] = f.x; o[1] = f.y;
    } else if constexpr (V == 2 && sizeof(T) == 8) {
        const double2 f = __ldg(reinterpret_cast<const double2 *>(p));
        o[0] = f.x; o[1] = f.y;
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) o[v] = __ldg(p + v);
    }
}
template <typename T, int V>
__device__ __forceinline__ void lds_v(const T *p, T *o) {
    if constexpr (V == 4 && sizeof(T) == 4) {
        const float4 f = *reinterpret_cast<const float4 *>(p);
        o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = f.w;
    } else if constexpr (V == 2 && sizeof(T) == 4) {
        const float2 f = *reinterpret_cast<const float2 *>(p);
        o[0] = f.x; o[1] = f.y;
    } else if constexpr (V == 2 && sizeof(T) == 8) {
        const double2 f = *reinterpret_cast<const double2 *>(p);
        o[0] = f.x; o[1] = f.y;
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) o[v] = p[v];
    }
}
template <typename T, int V>
__device__ __forceinline__ void sts_v(T *p, const T *o) {
    if constexpr (V == 4 && sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(o[0], o[1], o[2], o[3]);
    } else if constexpr (V == 2 && sizeof(T) == 4) {
        *reinterpret_cast<float2 *>(p) = make_float2(o[0], o[1]);
    } else if constexpr (V == 2 && sizeof(T) == 8) {
        *reinterpret_cast<double2 *>(p) = make_double2(o[0], o[1]);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) p[v] = o[v];
    }
}
template <typename T, int V>
__device__ __forceinline__ void acc_add(T *p, const T *s) {
    T o[V];
    lds_v<T, V>(p, o);
#pragma unroll
    for (int v = 0; v < V; ++v) o[v] += s[v];
    sts_v<T, V>(p, o);
}

// Adds one staged tile (payload at `buf`), right-hand sides j0 + [0, RL * V),
// into the warp's accumulators.  Lane (g, l) handles right-hand sides
// j0 + l * V + [0, V) of entries g, g + G, ...
template <typename T, int BS, int RL, int V, int KC>
__device__ __forceinline__ void ms_add(const MatView &M, const uint4 ta, const uint4 tb,
                                       const unsigned char *buf, int j0, T *acc, T *xt,
                                       int lane) {
    constexpr int G = 32 / RL;
    constexpr int RV = RL * V;
    constexpr int CH = G * KC;  // entries per chunk
    constexpr int XB = MsLayout<T, BS, RL, V>::XB;
    const int es = lane / RL, jl = lane % RL;
    const int jb = j0 + jl * V;
    T *myacc = &acc[lane * V];  // row r at myacc[r * 32 * V]
    const int ncoo = (ta.z >> 8) & 0xff;
    const int nxt = (ta.z >> 16) & 0xff;
    const int E = (int)tb.x;

    // COO entries, the next chunk's x gathers in flight during this chunk.
    // Tile entries are sorted by row, so a lane's slots never go down a row:
    // equal-row slots are summed in registers and each run adds once, all
    // accumulator loads ahead of the stores (distinct runs, distinct rows).
    // The section is stored in 32 lane slices of consecutive entries
    // (coo_slice_pos, cb_layout.hpp): slice s holds positions 32 j + s < E.
    // Lane group es takes slices es, es + G, ..., es + G (RL - 1) in turn --
    // its slots q = t Kt + j, slice es + G t, entry j -- so the rows of its
    // slots never decrease, and each slot step of the warp reads G
    // consecutive positions.
    const uint32_t *sidx = reinterpret_cast<const uint32_t *>(buf);
    const T *sval = reinterpret_cast<const T *>(buf + a16(4u * E));
    const int nv = max(0, min(V, M.nrhs - jb));  // this lane's right-hand sides
    const T *__restrict__ xr = static_cast<const T *>(M.x) + jb;
    const int Kt = (E + 31) >> 5;  // entries of the longest slices
    const int nslots = RL * Kt;
    auto positions = [&](int c0, int (&p_)[KC]) {  // slots c0 .. c0+KC-1 (E: none)
        int t = Kt ? c0 / Kt : RL, j = c0 - t * Kt;
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            p_[u] = t < RL ? 32 * j + es + G * t : E;
            if (++j == Kt) {
                j = 0;
                ++t;
            }
        }
    };
    uint32_t w[KC];
    T a[KC], xv[KC][V];
    int pc[KC];
    auto load = [&](const int (&p_)[KC], uint32_t (&w_)[KC], T (&a_)[KC], T (&x_)[KC][V]) {
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            const int e = p_[u];
            w_[u] = e < E ? sidx[e] : 0u;
            a_[u] = e < E ? (M.unit ? T(1) : sval[e]) : T(0);
        }
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            const int e = p_[u];
#pragma unroll
            for (int v = 0; v < V; ++v) x_[u][v] = T(0);
            if (e < E && nv > 0) {
                const T *p = xr + (size_t)(w_[u] & kColMask) * (size_t)M.ldx;
                if (M.xvec) {
                    ldg_v<T, V>(p, x_[u]);
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (v < nv) x_[u][v] = __ldg(p + v);
                }
            }
        }
    };
    if (E > 0) {
        positions(0, pc);
        load(pc, w, a, xv);
    }
    for (int c0 = 0; c0 < nslots; c0 += KC) {
        uint32_t w2[KC];
        T a2[KC], x2[KC][V];
        int pn[KC];
        positions(c0 + KC, pn);
        load(pn, w2, a2, x2);  // slots past the last load nothing
        // A slot with no entry (between two slices of the group, or past
        // the last) takes the row of the slot before it and adds 0, so equal
        // rows stay one run per chunk -- every run flushed below is a
        // distinct row, which lets all accumulator loads go ahead of the
        // stores.  A run is flushed only if it holds an entry.
        uint32_t r[KC];
        T s[KC][V];
        bool f[KC], has[KC];
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            const bool valid = pc[u] < E;
            r[u] = valid || u == 0 ? w[u] >> 27 : r[u > 0 ? u - 1 : 0];
            const bool same = u > 0 && r[u] == r[u > 0 ? u - 1 : 0];
            has[u] = valid || (same && has[u > 0 ? u - 1 : 0]);
#pragma unroll
            for (int v = 0; v < V; ++v)
                s[u][v] = fma(a[u], xv[u][v], same ? s[u > 0 ? u - 1 : 0][v] : T(0));
        }
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            const bool more = u + 1 < KC && r[u + 1 < KC ? u + 1 : u] == r[u];
            f[u] = has[u] && !more;
        }
        T o[KC][V];
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            if (f[u]) {
                lds_v<T, V>(myacc + r[u] * 32 * V, o[u]);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) o[u][v] = T(0);
            }
        }
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            if (f[u]) {
#pragma unroll
                for (int v = 0; v < V; ++v) o[u][v] += s[u][v];
                sts_v<T, V>(myacc + r[u] * 32 * V, o[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            w[u] = w2[u];
            a[u] = a2[u];
            pc[u] = pn[u];
#pragma unroll
            for (int v = 0; v < V; ++v) xv[u][v] = x2[u][v];
        }
    }

    // CSR and DENSE blocks, XB at a time (x rows of XB blocks fill xt)
    uint4 bd = make_uint4(0, 0, 0, 0);  // lane q: CSR/DENSE block q of the tile
    if (lane < nxt) bd = __ldg(&M.blocks[ta.x + ncoo + lane]);
    for (int jb0 = 0; jb0 < nxt; jb0 += XB) {
        const int nbg = min(XB, nxt - jb0);
        __syncwarp();  // the previous group is done with xt
        for (int i0 = 0; i0 < XB * BS * RV; i0 += 32) {
            const int idx = i0 + lane;  // idx % RV == lane % RV
            const int q = idx / (BS * RV), c = (idx / RV) % BS, j = j0 + idx % RV;
            const int src = jb0 + min(q, nbg - 1);
            const uint32_t xb = __shfl_sync(kFull, bd.z, src);
            const uint32_t mb = __shfl_sync(kFull, bd.y, src);
            if (q < nbg) {
                T xvv = T(0);
                if (c < (int)((mb >> 14) & 63) && j < M.nrhs) {
                    const int64_t col = M.gather ? (int64_t)__ldg(&M.block_cols[xb + c])
                                                 : (int64_t)(xb + c);
                    xvv = __ldg(static_cast<const T *>(M.x) + col * M.ldx + j);
                }
                xt[idx] = xvv;
            }
        }
        __syncwarp();
        for (int q = 0; q < nbg; ++q) {
            const uint32_t off = __shfl_sync(kFull, bd.x, jb0 + q);
            const uint32_t mb = __shfl_sync(kFull, bd.y, jb0 + q);
            const int k = (mb >> 3) & 2047;
            const unsigned char *pb = buf + off;
            const T *xq = xt + q * BS * RV + jl * V;  // column c at xq[c * RV]
            if ((mb & 3) == 1) {  // CSR
                using IdxT = typename std::conditional<BS == 16, uint8_t, uint16_t>::type;
                const IdxT *rp = reinterpret_cast<const IdxT *>(pb);
                const IdxT *ci = rp + BS + 1;
                const T *vv = reinterpret_cast<const T *>(
                    pb + a16((uint32_t)((BS + 1 + k) * sizeof(IdxT))));
                constexpr int L = G >= BS ? G / BS : 1;      // lanes per row
                constexpr int RS = G >= BS ? BS : G;          // rows in parallel
                for (int row = es / L; row < BS; row += RS) {
                    T sum[V], xx[V];
#pragma unroll
                    for (int v = 0; v < V; ++v) sum[v] = T(0);
                    for (int t = rp[row] + (G >= BS ? es % L : 0); t < rp[row + 1]; t += L) {
                        const T av = M.unit ? T(1) : vv[t];
                        lds_v<T, V>(xq + ci[t] * RV, xx);
#pragma unroll
                        for (int v = 0; v < V; ++v) sum[v] = fma(av, xx[v], sum[v]);
                    }
                    acc_add<T, V>(myacc + row * 32 * V, sum);
                    if (G >= BS) break;
                }
            } else {  // DENSE, row-major bs x bs; columns in a rotated order
                constexpr int L = G >= BS ? G / BS : 1;
                constexpr int RS = G >= BS ? BS : G;
                constexpr int W = BS / L;  // columns per lane
                for (int row = es / L; row < BS; row += RS) {
                    const int cb0 = (G >= BS ? es % L : 0) * W;
                    T sum[V], xx[V];
#pragma unroll
                    for (int v = 0; v < V; ++v) sum[v] = T(0);
#pragma unroll 4
                    for (int c = 0; c < W; ++c) {
                        const int cc = cb0 + ((c + row) % W);
                        const T av = dense_at<T, BS>(pb, M.unit, row, cc);
                        lds_v<T, V>(xq + cc * RV, xx);
#pragma unroll
                        for (int v = 0; v < V; ++v) sum[v] = fma(av, xx[v], sum[v]);
                    }
                    acc_add<T, V>(myacc + row * 32 * V, sum);
                    if (G >= BS) break;
                }
            }
        }
    }
    __syncwarp();
}

// Ends a run of `runlen` consecutive tiles of one block row (the last one
// tile index g of the launch's tile list, descriptors ta/tb), right-hand
// sides j0 + [0, RL * V): reduces the accumulators and stores Y, or for a
// row whose tiles are not all in this run leaves the run's sums in the slot
// of its first tile; the last run to arrive on the row's counter adds the
// row's runs in tile order.  With one pass per tile (passes == 1) runs start
// at the row's first tile and at every scheduling unit start inside the row
// (ustart[0 .. nunits), so the order does not depend on which warp ran which
// unit); with several passes every tile is a run.
template <typename T, int BS, int RL, int V>
__device__ __forceinline__ void ms_out(const MatView &M, const uint4 ta, const uint4 tb,
                                       int64_t g, int64_t runlen, int j0, int passes, T *acc,
                                       const int64_t *__restrict__ ustart, int64_t nunits,
                                       int lane) {
    constexpr int G = 32 / RL;
    constexpr int RV = RL * V;
    constexpr int NO = BS * RV;
    T *__restrict__ y = static_cast<T *>(M.y);
    const int64_t row0 = (int64_t)ta.y * BS;
    const bool whole = tb.y == 0xffffffffu || (passes == 1 && runlen == (int64_t)tb.w);
    const int64_t first = g - (int64_t)(tb.y - tb.z);  // the row's first tile
    const int64_t run0 = g - runlen + 1;
    T *part = static_cast<T *>(M.partials);
#pragma unroll 1
    for (int q = 0; q < (NO + 31) / 32; ++q) {
        const int o = lane + 32 * q;
        if (o < NO) {
            const int r = o / RV, jj = o % RV;
            T s0 = T(0), s1 = T(0);
#pragma unroll 8
            for (int t = 0; t < G; t += 2) {
                T *p0 = &acc[(r * 32 + ((t + r) % G) * RL) * V + jj];
                s0 += *p0;
                *p0 = T(0);
                if (t + 1 < G) {
                    T *p1 = &acc[(r * 32 + ((t + 1 + r) % G) * RL) * V + jj];
                    s1 += *p1;
                    *p1 = T(0);
                }
            }
            const T s = s0 + s1;
            const int jo = j0 + jj;
            if (jo < M.nrhs) {
                if (whole) {
                    if (row0 + r < M.m) y[(row0 + r) * M.ldy + jo] = s;
                } else {
                    const int64_t slot = (int64_t)tb.z + (run0 - first);
                    part[((size_t)slot * M.nrhs + jo) * BS + r] = s;
                }
            }
        }
    }
    if (whole) return;
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane == 0) {
        const int add = (int)runlen;
        const int old = atomicAdd(&M.counters[ta.y], add);
        last = old + add == (int)tb.w * passes;
    }
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    const int64_t end = first + (int64_t)tb.w;
    int64_t u0 = 0, u1 = nunits;  // the first unit starting after `first`
    while (u0 < u1) {
        const int64_t mid = (u0 + u1) >> 1;
        if (__ldg(&ustart[mid]) <= first) u0 = mid + 1; else u1 = mid;
    }
    for (int o = lane; o < BS * M.nrhs; o += 32) {
        const int r = o % BS, jj = o / BS;
        T tot = __ldcg(&part[((size_t)tb.z * M.nrhs + jj) * BS + r]);
        if (passes > 1) {
            for (uint32_t t = 1; t < tb.w; ++t)
                tot += __ldcg(&part[((size_t)(tb.z + t) * M.nrhs + jj) * BS + r]);
        } else {
            for (int64_t u = u0; u < nunits; ++u) {
                const int64_t b = __ldg(&ustart[u]);
                if (b >= end) break;
                tot += __ldcg(&part[((size_t)(tb.z + (b - first)) * M.nrhs + jj) * BS + r]);
            }
        }
        if (row0 + r < M.m) y[(row0 + r) * M.ldy + jj] = tot;
    }
    if (lane == 0) atomicExch(&M.counters[ta.y], 0);
}

// A position in the concatenated tile list: matrix k owns [lo, hi).
struct Cursor {
    int k = 0;
    int64_t lo = 0, hi = 0;
};

__device__ __forceinline__ void advance(Cursor &c, int64_t g, const int64_t *__restrict__ toff) {
    while (g >= c.hi) {
        ++c.k;
        c.lo = c.hi;
        c.hi = __ldg(&toff[c.k + 1]);
    }
}

// COO slots per lane in one chunk: about 16 (FP32) or 8 (FP64) gathered
// values in flight per lane
template <typename T>
__host__ __device__ constexpr int kc_for(int V) {
    return sizeof(T) == 4 ? (V == 1 ? 8 : (V == 2 ? 6 : 4)) : (V == 1 ? 6 : 4);
}

// Single matrix: mats == nullptr and `single` is the matrix (tiles
// [0, single.ntiles)).  Batch: mats[k] owns tiles [toff[k], toff[k+1]) of the
// launch's tile list; every matrix of one launch uses RL lanes x V values.
// Tiles come in units -- unit u is [ustart[u], ustart[u+1]).  dynamic = 0:
// warp w runs unit w (host cost-balanced ranges, one per warp).  dynamic = 1:
// units of at least two tiles but the last, boundaries at block-row starts
// where the host could place them, taken from a counter (sched[0]) one unit
// ahead; the warp whose exit completes sched[1] == number of warps resets
// both for the next launch.
template <typename T, int BS, int RL, int V>
__global__ void __launch_bounds__(kMsWarps * 32, 3)
    cb_mstream_kernel(const MatView single, const MatView *__restrict__ mats, int nmats,
                      const int64_t *__restrict__ toff, const int64_t *__restrict__ ustart,
                      int64_t nunits, int dynamic, uint32_t cap,
                      uint32_t *__restrict__ sched, uint32_t *__restrict__ err,
                      uint32_t limit) {
    using SL = MsLayout<T, BS, RL, V>;
    constexpr int RV = RL * V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char *wbase = smem_raw + (size_t)wib * SL::bytes(cap);
    T *acc = reinterpret_cast<T *>(wbase);
    T *xt = reinterpret_cast<T *>(wbase + SL::acc_bytes);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(wbase + SL::acc_bytes + SL::xt_bytes);
    unsigned char *const buf0 = wbase + SL::head;
    const uint64_t pol = policy_evict_first();

    for (int t = lane; t < BS * 32 * V; t += 32) acc[t] = T(0);
    if (lane == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    __syncwarp();

    const bool one = mats == nullptr;
    // units: lane 0 takes the next unit index with an atomic; the other
    // lanes learn it (shuffle) only when it is needed, about a unit later, so
    // the atomic's latency is hidden.  ua = unit being computed, [ua_s, ua_e)
    // its tiles; ub = the next unit.
    const int64_t gw = (int64_t)blockIdx.x * kMsWarps + wib;
    uint32_t ub_raw = 0;
    bool first_take = true;
    auto take = [&]() {
        if (dynamic) {
            if (lane == 0) ub_raw = atomicAdd(&sched[0], 1u);
        } else {  // the warp's own unit, then nothing
            ub_raw = first_take && gw < nunits ? (uint32_t)gw : (uint32_t)nunits;
        }
        first_take = false;
    };
    bool ub_known = false;
    int64_t ub = 0, ub_s = 0, ub_e = 0;
    auto resolve = [&]() {
        if (!ub_known) {
            ub = (int64_t)__shfl_sync(kFull, ub_raw, 0);
            if (ub < nunits) {
                ub_s = __ldg(&ustart[ub]);
                ub_e = __ldg(&ustart[ub + 1]);
            }
            ub_known = true;
        }
    };
    take();
    resolve();
    int64_t ua = ub, ua_s = ub_s, ua_e = ub_e;
    if (ua < nunits) {
        take();
        ub_known = false;
    }
    // the n-th tile after tile g of unit ua, following into unit ub (n <= 2;
    // units hold >= 2 tiles but the last); -1 past the warp's work
    auto ahead = [&](int64_t g, int n) -> int64_t {
        if (g + n < ua_e) return g + n;
        resolve();
        if (ub >= nunits) return -1;
        const int64_t h = ub_s + (g + n - ua_e);
        return h < ub_e ? h : -1;
    };

    // a matrix cursor for the tiles computed and one for the tiles staged
    auto locate = [&](Cursor &c, int64_t g) {
        if (one) {
            c.k = 0;
            c.lo = 0;
            c.hi = single.ntiles;
            return;
        }
        if (g >= c.lo && g < c.hi) return;
        if (g >= c.hi && c.hi > 0) {
            advance(c, g, toff);
            return;
        }
        int l = 0, h = nmats;  // the last matrix k with toff[k] <= g
        while (h - l > 1) {
            const int mid = (l + h) >> 1;
            if (__ldg(&toff[mid]) <= g) l = mid; else h = mid;
        }
        c.k = l;
        c.lo = __ldg(&toff[l]);
        c.hi = __ldg(&toff[l + 1]);
    };
    Cursor cs;
    cs.hi = 0;
    MatView M = single;
    int mk = -1;  // matrix held in M
    // what each buffer holds: the tile's matrix, its descriptors, and the
    // block row of the matrix's next tile
    int sk0 = 0, sk1 = 0;
    uint4 sa0 = make_uint4(0, 0, 0, 0), sb0 = sa0, sa1 = sa0, sb1 = sa0;
    uint32_t snext0 = 0xffffffffu, snext1 = 0xffffffffu;  // block row of tile g+1 (same matrix)

    auto stage = [&](int64_t g, int bi) {
        locate(cs, g);
        const MatView *V0 = one ? &single : &mats[cs.k];
        const uint4 *st_tiles = V0->tiles;
        const int64_t t = g - cs.lo;
        const uint4 a = __ldg(&st_tiles[2 * t]);
        const uint4 b = __ldg(&st_tiles[2 * t + 1]);
        const bool more = t + 1 < cs.hi - cs.lo;
        const uint4 an = more ? __ldg(&st_tiles[2 * (t + 1)]) : make_uint4(0, 0xffffffffu, 0, 0);
        const uint32_t e16 = more ? an.w : V0->pay16_end;
        if (bi) {
            sk1 = cs.k; sa1 = a; sb1 = b; snext1 = an.y;
        } else {
            sk0 = cs.k; sa0 = a; sb0 = b; snext0 = an.y;
        }
        if (lane == 0) {
            const uint32_t bytes = (e16 - a.w) * 16u;
            if (bytes == 0) {
                mbar_arrive(&mbar[bi]);
            } else {
                fence_proxy_async();  // the buffer's previous tile was read
                mbar_arrive_tx(&mbar[bi], bytes);
                bulk_g2s(buf0 + bi * cap, V0->payload + (size_t)a.w * 16, bytes, &mbar[bi], pol);
            }
        }
    };

    uint32_t phase = 0u, inflight = 0u;
    int bi = 0;
    int64_t runlen = 0;  // tiles of the current block row added so far
    if (ua < nunits) {
        int64_t g = ua_s;
        stage(g, 0);
        inflight |= 1u;
        const int64_t g1 = ahead(g, 1);
        if (g1 >= 0) {
            stage(g1, 1);
            inflight |= 2u;
        }
        for (;;) {
            // on give-up the copy into buffer bi may still be landing: leave
            // it marked in flight (same parity) for the drain below
            if (!mbar_wait(&mbar[bi], (phase >> bi) & 1u, err, limit)) break;
            phase ^= 1u << bi;
            inflight &= ~(1u << bi);
            const int k = bi ? sk1 : sk0;
            if (!one && k != mk) {
                M = mats[k];
                mk = k;
            }
            const uint4 ta = bi ? sa1 : sa0;
            const uint4 tb = bi ? sb1 : sb0;
            const uint32_t next_row = bi ? snext1 : snext0;
            // does this warp's next tile continue the block row in this unit?
            const bool cont = g + 1 < ua_e && next_row == ta.y;
            const unsigned char *buf = buf0 + bi * cap;
            const int passes = (M.nrhs + RV - 1) / RV;
            if (passes == 1) {
                ms_add<T, BS, RL, V, kc_for<T>(V)>(M, ta, tb, buf, 0, acc, xt, lane);
                ++runlen;
                if (!cont) {
                    ms_out<T, BS, RL, V>(M, ta, tb, g, runlen, 0, 1, acc, ustart, nunits, lane);
                    runlen = 0;
                }
            } else {
                for (int j0 = 0; j0 < M.nrhs; j0 += RV) {
                    ms_add<T, BS, RL, V, kc_for<T>(V)>(M, ta, tb, buf, j0, acc, xt, lane);
                    ms_out<T, BS, RL, V>(M, ta, tb, g, 1, j0, passes, acc, ustart, nunits,
                                         lane);
                }
            }
            __syncwarp();
            const int64_t g2 = ahead(g, 2);
            if (g2 >= 0) {
                stage(g2, bi);
                inflight |= 1u << bi;
            }
            bi ^= 1;
            if (g + 1 < ua_e) {
                ++g;
            } else {  // unit done: move to the next, take one more ahead
                resolve();
                ua = ub;
                ua_s = ub_s;
                ua_e = ub_e;
                if (ua >= nunits) break;
                take();
                ub_known = false;
                g = ua_s;
            }
        }
    }
    // never leave with a bulk copy still writing this warp's buffers
    for (int q = 0; q < 2; ++q)
        if ((inflight >> q) & 1u) mbar_wait(&mbar[q], (phase >> q) & 1u, err);
    __syncwarp();
    // count this warp out; the last one resets the unit counter
    if (lane == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(&sched[1], 1u);
        if (done == gridDim.x * kMsWarps - 1) {
            atomicExch(&sched[0], 0u);
            atomicExch(&sched[1], 0u);
        }
    }
}

template <typename T, int BS, int RL, int V>
cudaError_t ms_configure(uint32_t cap, size_t *smem) {
    *smem = (size_t)MsLayout<T, BS, RL, V>::bytes(cap) * kMsWarps;
    return dev_enable_smem(reinterpret_cast<const void *>(cb_mstream_kernel<T, BS, RL, V>),
                           *smem);
}

template <typename T, int BS, int RL, int V>
int64_t ms_warps_t(uint32_t cap) {
    size_t smem = 0;
    if (ms_configure<T, BS, RL, V>(cap, &smem) != cudaSuccess) return 0;
    const int resident = dev_resident(
        reinterpret_cast<const void *>(cb_mstream_kernel<T, BS, RL, V>), kMsWarps * 32, smem);
    return (int64_t)resident * dev_sms() * kMsWarps;
}

template <typename T, int BS, int RL, int V>
cudaError_t ms_launch_t(const MatView &single, const MatView *mats, int nmats,
                        const int64_t *toff, const int64_t *ustart, int64_t nunits, int dynamic,
                        uint32_t cap, uint32_t *sched, uint32_t *err, cudaStream_t stream) {
    size_t smem = 0;
    cudaError_t e = ms_configure<T, BS, RL, V>(cap, &smem);
    if (e != cudaSuccess) return e;
    if (cap % 16 || !sched || !err) return cudaErrorInvalidValue;
    if (nunits <= 0) return cudaSuccess;
    // dynamic: resident warps (or fewer); static: one warp per unit
    const int64_t w = dynamic ? std::min<int64_t>(ms_warps_t<T, BS, RL, V>(cap), nunits) : nunits;
    const int64_t ctas = (w + kMsWarps - 1) / kMsWarps;
    cb_mstream_kernel<T, BS, RL, V><<<(unsigned)ctas, kMsWarps * 32, smem, stream>>>(
        single, mats, nmats, toff, ustart, nunits, dynamic, cap, sched, err, wait_polls());
    note_launch();
    return cudaGetLastError();
}

// Calls f(T(), BS, RL, V) for the run-time class.
template <typename F>
auto by_class(int bs, int f32, MsClass c, F f) {
    auto with_t = [&](auto t, auto b) {
        using T = decltype(t);
        using I1 = std::integral_constant<int, 1>;
        using I2 = std::integral_constant<int, 2>;
        using VV = std::integral_constant<int, sizeof(T) == 4 ? 4 : 2>;
        if (c.V == 1) return f(t, b, I1(), I1());
        if (c.V == 2 && c.RL == 1 && sizeof(T) == 4) return f(t, b, I1(), I2());
        switch (c.RL) {
            case 1: return f(t, b, I1(), VV());
            case 2: return f(t, b, I2(), VV());
            case 4: return f(t, b, std::integral_constant<int, 4>(), VV());
            default: return f(t, b, std::integral_constant<int, 8>(), VV());
        }
    };
    if (bs == 16)
        return f32 ? with_t(float(), std::integral_constant<int, 16>())
                   : with_t(double(), std::integral_constant<int, 16>());
    return f32 ? with_t(float(), std::integral_constant<int, 32>())
               : with_t(double(), std::integral_constant<int, 32>());
}

}  // namespace

MsClass ms_class(int nrhs, int f32) {
    const int vmax = f32 ? 4 : 2;
    int R = 1;
    while (R < nrhs && R < 8 * vmax) R *= 2;
    MsClass c;
    c.V = std::min(vmax, R);
    c.RL = std::max(1, R / c.V);
    return c;
}

uint32_t ms_cap(int64_t max_tile_bytes) {
    return (uint32_t)std::max<int64_t>(16, (max_tile_bytes + 15) / 16 * 16);
}

MatView mat_view(const DevLayout &d, const void *x, void *y, int nrhs, int64_t ldx,
                 int64_t ldy) {
    MatView M;
    M.tiles = static_cast<const uint4 *>(d.tiles);
    M.blocks = static_cast<const uint4 *>(d.blocks);
    M.payload = d.payload;
    M.block_cols = d.block_cols;
    M.x = x;
    M.y = y;
    M.partials = d.partials;
    M.counters = d.counters;
    M.ntiles = d.ntiles;
    M.m = d.m;
    M.ldx = ldx;
    M.ldy = ldy;
    M.nrhs = nrhs;
    M.gather = d.gather;
    M.pay16_end = d.pay16_end;
    M.unit = d.unit;
    // vector x loads: rows aligned to V values and every V-group a lane reads
    // inside its row (ldx a multiple of V, and the last group within ldx)
    const MsClass c = ms_class(nrhs, d.f32);
    const size_t vsz = d.f32 ? 4 : 8;
    const int64_t vcols = (nrhs + c.V - 1) / c.V * c.V;
    M.xvec = c.V > 1 && reinterpret_cast<uintptr_t>(x) % (c.V * vsz) == 0 && ldx % c.V == 0 &&
             vcols <= ldx;
    return M;
}

int64_t ms_warps(int bs, int f32, uint32_t cap) {
    return by_class(bs, f32, ms_class(8, f32), [&](auto t, auto b, auto rl, auto v) {
        using T = decltype(t);
        return ms_warps_t<T, b(), rl(), v()>(cap);
    });
}

int64_t ms_tile_cost(const uint32_t *tile8, const uint32_t *blocks4) {
    const uint32_t counts = tile8[2];
    const uint32_t nb = counts & 0xff, ncoo = (counts >> 8) & 0xff;
    int64_t work = 64 + tile8[4];  // per-tile overhead + COO entries
    for (uint32_t q = ncoo; q < nb; ++q) work += (blocks4[4 * (tile8[0] + q) + 1] >> 3) & 2047;
    return work;
}

void ms_unit_starts(const uint32_t *tile8, int64_t ntiles, int64_t target, int64_t base,
                    std::vector<int64_t> &ustart) {
    for (int64_t t = 0; t < ntiles; ++t) {
        const uint32_t *d = tile8 + 8 * t;
        const bool row_start = d[5] == 0xffffffffu || d[5] == d[6];  // slot == first slot
        const int64_t count = ustart.empty() ? 0 : base + t - ustart.back();  // in the unit
        // a new unit at a block-row start once the unit is full, or anywhere
        // once it is twice as long (very long rows)
        if (ustart.empty() || (count >= target && row_start) || count >= 2 * target)
            ustart.push_back(base + t);
    }
}

cudaError_t launch_spmm(const DevLayout &d, const void *x, void *y, int nrhs, int64_t ldx,
                        int64_t ldy, cudaStream_t stream) {
    if (d.ntiles == 0) return cudaSuccess;
    if (!d.ustart) return cudaErrorInvalidValue;
    const MatView M = mat_view(d, x, y, nrhs, ldx, ldy);
    return by_class(d.bs, d.f32, ms_class(nrhs, d.f32), [&](auto t, auto b, auto rl, auto v) {
        using T = decltype(t);
        return ms_launch_t<T, b(), rl(), v()>(M, nullptr, 1, nullptr, d.ustart, d.nunits, 0,
                                              d.mcap, d.sched, d.err, stream);
    });
}

cudaError_t launch_batch(int bs, int f32, MsClass c, const MatView *mats, int nmats,
                         const int64_t *toff, const int64_t *ustart, int64_t nunits,
                         uint32_t cap, uint32_t *sched, cudaStream_t stream) {
    return by_class(bs, f32, c, [&](auto t, auto b, auto rl, auto v) {
        using T = decltype(t);
        return ms_launch_t<T, b(), rl(), v()>(MatView(), mats, nmats, toff, ustart, nunits, 1,
                                              cap, sched, sched + 2, stream);
    });
}

}  // namespace cb
