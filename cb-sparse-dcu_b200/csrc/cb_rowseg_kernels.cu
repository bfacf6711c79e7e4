// Row-segment stream kernels (layout in cb_rowseg.hpp) and the balanced
// schedule:
//   * cb_rowseg_kernel       y = A x, one right-hand side (below);
//   * cb_rowseg_mrhs_kernel  Y = A X, G lanes per entry, several right-hand
//                            sides (rs_mrhs_segment);
//   * cb_rowseg_gv_kernel    the fused adjoint: A^T G and the value gradient;
//   * cb_rowseg_batch_kernel every matrix of a batch in one launch;
//   * cb_balanced_kernel     plans built with row_owned = 0: the reference's
//                            block order, atomics into y;
//   * value refreshes after cbspmv_set_values.
//
// One right-hand side: one CTA of 32 warps per SM.  Per chunk a lane
//   * holds the NEXT chunk's words and values in registers, loaded with
//     coalesced 16-byte loads that do not allocate in L1 (L1 is left to the
//     x gathers) and are marked evict-first in L2 (x stays in L2),
//   * gathers x for its kRsK entries, all loads in flight at once: from the
//     CTA's window of x in shared memory (staged at the start) when the
//     entry's word says so, else from global memory,
//   * counts its row starts; an exclusive warp scan of the counts gives the
//     ordinal of the row it starts in,
//   * adds its entries along its rows in registers; a row that starts and
//     ends inside the lane is stored at once,
//   * joins the rows that run across lanes with one segmented inclusive scan
//     (reset at lanes holding a row start), carrying the chunk's last row into
//     the next chunk.
// The products of one row are added in entry order within a lane and in lane
// order across lanes, fixed by the layout: results are bitwise reproducible
// (the balanced schedule's atomics excepted).  The reference adds each entry
// into its row with an atomic (cb-spmv-dcu.hpp:423-426); the sums here are
// the same rows' sums.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "cb_device.cuh"
#include "cb_kernels.hpp"
#include "cb_rowseg.hpp"

namespace cb {
namespace {

using dev::kFull;

template <typename T> struct RsVec;
template <> struct RsVec<double> { using V = double2; static constexpr int n = 2; };
template <> struct RsVec<float> { using V = float4; static constexpr int n = 4; };

__device__ __forceinline__ uint4 ld_stream(const uint4 *p, uint64_t pol) {
    uint4 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ double2 ld_stream(const double2 *p, uint64_t pol) {
    double2 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
        : "=d"(r.x), "=d"(r.y)
        : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ float4 ld_stream(const float4 *p, uint64_t pol) {
    float4 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
        : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
        : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ void unpack(const double2 &v, double *o) {
    o[0] = v.x;
    o[1] = v.y;
}
__device__ __forceinline__ void unpack(const float4 &v, float *o) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}

// A row that crosses segments: this segment's part into its slot; the last
// part to arrive (acquire-release counter) adds the slots in segment order,
// stores y and resets the counter.  Called by one lane.
template <typename T>
__device__ __forceinline__ void rs_arrive(const RowSegDev &rs, T *__restrict__ y, int span,
                                          T v, int slot) {
    T *part = static_cast<T *>(rs.part);
    part[slot] = v;
    cuda::atomic_ref<int32_t, cuda::thread_scope_device> ctr(rs.counters[span]);
    const int old = ctr.fetch_add(1, cuda::memory_order_acq_rel);
    const int4 sp = __ldg(&rs.spans[span]);
    if (old + 1 == sp.y - sp.x + 1) {
        T tot = __ldcg(&part[2 * sp.x + 1]);
        for (int s = sp.x + 1; s <= sp.y; ++s) tot += __ldcg(&part[2 * s]);
        y[rs.rowmap ? __ldg(&rs.rowmap[sp.z]) : sp.z] = tot;
        ctr.store(0, cuda::memory_order_relaxed);
    }
}

template <typename T, bool UNIT>
__global__ void __launch_bounds__(kRsWarps * 32, 1)
    cb_rowseg_kernel(const RowSegDev rs, const T *__restrict__ x, T *__restrict__ y) {
    using V = typename RsVec<T>::V;
    constexpr int K = kRsK, NV = RsVec<T>::n;
    constexpr int64_t CB = 32 * K * (4 + (UNIT ? 0 : (int64_t)sizeof(T)));
    extern __shared__ __align__(16) unsigned char rs_smem[];
    T *xs = reinterpret_cast<T *>(rs_smem);  // x[wb .. wb + W)
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (int i = (blockIdx.x * kRsWarps + wib) * 32 + lane; i < rs.nempty;
         i += gridDim.x * kRsWarps * 32)
        y[__ldg(&rs.empty[i])] = T(0);
    const int G = gridDim.x, b = blockIdx.x;
    const int64_t wb = __ldg(&rs.wbase[b]);
    for (int i = threadIdx.x; i < rs.W; i += kRsWarps * 32)
        xs[i] = wb + i < rs.n ? __ldg(x + wb + i) : T(0);
    __syncthreads();
    const int sb0 = (int)((int64_t)b * rs.nseg / G);
    const int sb1 = (int)((int64_t)(b + 1) * rs.nseg / G);
    int s = sb0 + wib;
    if (s >= sb1) return;
    const int M = rs.M, nch = rs.nch, nord = rs.nord;
    const uint64_t pol = dev::policy_evict_first();
    uint4 nw[K / 4];
    V nv[K / NV];
    auto load = [&](int c) {
        const uint4 *gw = reinterpret_cast<const uint4 *>(rs.chunks + (int64_t)c * CB);
        const V *gv = reinterpret_cast<const V *>(rs.chunks + (int64_t)c * CB + 32 * K * 4);
#pragma unroll
        for (int q = 0; q < K / 4; ++q) nw[q] = ld_stream(gw + q * 32 + lane, pol);
        if (!UNIT) {
#pragma unroll
            for (int q = 0; q < K / NV; ++q) nv[q] = ld_stream(gv + q * 32 + lane, pol);
        }
    };
    auto rid = [&](int32_t o) { return rs.rowmap ? __ldg(&rs.rowmap[o]) : o; };
    int c = s * M;
    load(c);
    while (true) {
        // segment s: meta = {ordinal running before its first entry, its first
        // entry starts a row, head span, tail span}
        const int4 meta = __ldg(&rs.meta[s]);
        const int32_t first = meta.x;
        int32_t ord0 = meta.x;
        T carry = T(0);
        const int cend = min(nch, c + M);
        for (; c < cend; ++c) {
            uint32_t w[K];
            T v[K], xv[K];
#pragma unroll
            for (int q = 0; q < K / 4; ++q) {
                w[4 * q] = nw[q].x;
                w[4 * q + 1] = nw[q].y;
                w[4 * q + 2] = nw[q].z;
                w[4 * q + 3] = nw[q].w;
            }
            if (UNIT) {
#pragma unroll
                for (int j = 0; j < K; ++j) v[j] = T(1);
            } else {
#pragma unroll
                for (int q = 0; q < K / NV; ++q) unpack(nv[q], v + q * NV);
            }
            {  // the next chunk of this segment, or the first of the warp's next
                int cn = c + 1;
                if (cn >= cend) {
                    const int sn = s + kRsWarps;
                    cn = sn < sb1 ? sn * M : -1;
                }
                if (cn >= 0) load(cn);
            }
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const uint32_t col = w[j] & kRsColMask;
                xv[j] = (w[j] & kRsWin) ? xs[col - wb] : __ldg(x + col);
            }
            int cnt = 0;
#pragma unroll
            for (int j = 0; j < K; ++j) cnt += (int)(w[j] >> 31);
            int inc = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int t = __shfl_up_sync(kFull, inc, d);
                if (lane >= d) inc += t;
            }
            const int32_t ordS = ord0 + inc - cnt;  // the row this lane starts in
            int32_t ord = ordS;
            T run = T(0), head = T(0);
            bool seen = false;  // a row starts in this lane
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const bool f = (w[j] >> 31) != 0;
                if (f && seen) y[rid(ord)] = run;  // a row whole inside the lane
                head = (f && !seen) ? run : head;
                seen = seen || f;
                ord += f ? 1 : 0;
                run = fma(v[j], xv[j], f ? T(0) : run);
            }
            // rows across lanes: inclusive scan of run, reset at lanes that
            // hold a row start; lane 0 continues the previous chunk's row
            T sc = run;
            if (lane == 0 && !seen) sc += carry;
            bool r = seen;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const T su = __shfl_up_sync(kFull, sc, d);
                const bool ru = __shfl_up_sync(kFull, (int)r, d) != 0;
                if (lane >= d) {
                    if (!r) sc += su;
                    r = r || ru;
                }
            }
            T cin = __shfl_up_sync(kFull, sc, 1);
            if (lane == 0) cin = carry;
            if (seen) {  // the row this lane started in ends here
                const T val = cin + head;
                if (ordS == first && meta.z >= 0)
                    rs_arrive<T>(rs, y, meta.z, val, 2 * s);
                else if (!(ordS == first && meta.y) && ordS < nord)
                    y[rid(ordS)] = val;
            }
            carry = __shfl_sync(kFull, sc, 31);
            ord0 = __shfl_sync(kFull, ord, 31);
        }
        // the segment's last row: a span's part, or whole here
        if (lane == 0) {
            if (ord0 == first && meta.z >= 0)
                rs_arrive<T>(rs, y, meta.z, carry, 2 * s);
            else if (meta.w >= 0)
                rs_arrive<T>(rs, y, meta.w, carry, 2 * s + 1);
            else if (ord0 < nord && !(ord0 == first && meta.y))
                y[rid(ord0)] = carry;
        }
        s += kRsWarps;
        if (s >= sb1) break;
        c = s * M;
    }
}

// Several right-hand sides over the same stream: G lanes per entry, lane q
// of a group holding the V = 16 / sizeof(T) right-hand sides q*V .. q*V+V-1
// of its rows; P = 32 / G groups per warp, group p taking the 4G consecutive
// entries 4Gp .. 4Gp+4G-1 of each chunk (the entries lanes Gp .. Gp+G-1 take
// in the one-vector kernel).  A group walks its entries in steps of 4: the
// step's words and values are loaded by every lane of the group (one 16-byte
// access, broadcast), its four x rows gathered (one 16-byte load per lane
// and entry), then added along the rows in registers.  Row starts are
// counted per group and scanned over the groups; one segmented scan over the
// groups joins rows across groups.  No x window (the window holds single
// vectors).
constexpr int kRsMaxRhs = kRsSlotValues;  // right-hand sides per launch (slots hold this many)

// One matrix as the several-right-hand-side segment code reads it.
template <typename T>
struct RsMat {
    const uint8_t *chunks;
    const int32_t *rowmap;  // NULL: ordinals are rows
    const T *x;
    T *y;
    int64_t ldx, ldy;
    int32_t nrhs, nord;
    int32_t xvec, yvec;     // 16-byte loads of x rows / stores of y rows allowed
};

// The spans of one segmentation: per span {first segment, last segment,
// ordinal, -}, an arrival counter each (zero between launches), kRsMaxRhs
// values per slot and two slots per segment.
template <typename T>
struct RsSpans {
    const int4 *spans;
    int32_t *counters;
    T *part;
};

// The value gradient of a transposed stream (the fused adjoint): per stream
// entry e of row j (a column of A) gathering row i of G, gv[e] = sum over the
// right-hand sides of G[i, :] . xo[j, :] (written, or added when accum).
template <typename T>
struct RsGV {
    const T *xo;
    int64_t ldo;
    int32_t xovec;  // 16-byte loads of xo rows allowed
    int32_t accum;
    T *gv;
};

// Chunks [cb, ce) of matrix A as segment s, meta = {ordinal running before
// chunk cb, chunk cb starts a row, head span, tail span}.  Called by a whole
// warp.  GV: also the value gradient of every entry (gvp).
template <typename T, int G, bool UNIT, bool GV = false>
__device__ __forceinline__ void rs_mrhs_segment(const RsMat<T> &A, int cb, int ce, int4 meta,
                                                int s, const RsSpans<T> &S, int lane,
                                                uint64_t pol, const RsGV<T> *gvp = nullptr) {
    using VT = typename RsVec<T>::V;
    constexpr int V = RsVec<T>::n, P = 32 / G, NV = RsVec<T>::n;
    constexpr int64_t CB = 128 * (4 + (UNIT ? 0 : (int64_t)sizeof(T)));
    const int p = lane / G, q = lane % G, c0 = q * V;
    const unsigned gmask = (G == 32 ? kFull : ((1u << G) - 1u)) << (p * G);
    const int nrhs = A.nrhs, nord = A.nord;
    auto rid = [&](int32_t o) -> int64_t { return A.rowmap ? __ldg(&A.rowmap[o]) : o; };
    auto load_x = [&](uint32_t col, T *o) {
        const T *px = A.x + (int64_t)col * A.ldx + c0;
        if (A.xvec) {
            if (c0 < nrhs) unpack(__ldg(reinterpret_cast<const VT *>(px)), o);
            else
#pragma unroll
                for (int k = 0; k < V; ++k) o[k] = T(0);
        } else {
#pragma unroll
            for (int k = 0; k < V; ++k) o[k] = c0 + k < nrhs ? __ldg(px + k) : T(0);
        }
    };
    auto store_y = [&](int64_t row, const T *v) {
        T *py = A.y + row * A.ldy + c0;
        if (A.yvec && c0 + V <= nrhs) {
            VT t;
            T *tv = reinterpret_cast<T *>(&t);
#pragma unroll
            for (int k = 0; k < V; ++k) tv[k] = v[k];
            *reinterpret_cast<VT *>(py) = t;
        } else {
#pragma unroll
            for (int k = 0; k < V; ++k)
                if (c0 + k < nrhs) py[k] = v[k];
        }
    };
    // a row across segments: every lane of the group writes its columns of
    // the slot; lane 0 of the group takes the arrival; the last part's group
    // adds the slots in segment order and stores y
    auto arrive = [&](int span, const T *v, int slot) {
#pragma unroll
        for (int k = 0; k < V; ++k)
            if (c0 + k < nrhs) S.part[(int64_t)slot * kRsMaxRhs + c0 + k] = v[k];
        __threadfence();
        __syncwarp(gmask);
        int last = 0;
        const int4 sp = __ldg(&S.spans[span]);
        if (q == 0) {
            cuda::atomic_ref<int32_t, cuda::thread_scope_device> ctr(S.counters[span]);
            last = ctr.fetch_add(1, cuda::memory_order_acq_rel) + 1 == sp.y - sp.x + 1;
            if (last) ctr.store(0, cuda::memory_order_relaxed);
        }
        last = __shfl_sync(gmask, last, p * G);
        if (last) {
            __threadfence();
            T tot[V];
#pragma unroll
            for (int k = 0; k < V; ++k)
                tot[k] = c0 + k < nrhs
                             ? __ldcg(&S.part[(int64_t)(2 * sp.x + 1) * kRsMaxRhs + c0 + k])
                             : T(0);
            for (int w = sp.x + 1; w <= sp.y; ++w)
#pragma unroll
                for (int k = 0; k < V; ++k)
                    if (c0 + k < nrhs)
                        tot[k] += __ldcg(&S.part[(int64_t)(2 * w) * kRsMaxRhs + c0 + k]);
            store_y(rid(sp.z), tot);
        }
    };
    const int32_t first = meta.x;
    int32_t ord0 = meta.x;
    T carry[V];
#pragma unroll
    for (int k = 0; k < V; ++k) carry[k] = T(0);
    for (int c = cb; c < ce; ++c) {
        const uint4 *gw = reinterpret_cast<const uint4 *>(A.chunks + (int64_t)c * CB);
        const uint8_t *gv = A.chunks + (int64_t)c * CB + 4 * 128;
        // row starts of the group's entries: each lane counts one 4-entry
        // step, the group adds them
        int cnt;
        {
            const uint4 t = __ldg(gw + G * p + q);
            cnt = (int)((t.x >> 31) + (t.y >> 31) + (t.z >> 31) + (t.w >> 31));
#pragma unroll
            for (int d = 1; d < G; d <<= 1) cnt += __shfl_xor_sync(kFull, cnt, d);
        }
        int inc = cnt;  // inclusive scan over the groups
#pragma unroll
        for (int d = 1; d < P; d <<= 1) {
            const int t = __shfl_up_sync(kFull, inc, d * G);
            if (p >= d) inc += t;
        }
        const int32_t ordS = ord0 + inc - cnt;  // the row this group starts in
        int32_t ord = ordS;
        T run[V], head[V];
#pragma unroll
        for (int k = 0; k < V; ++k) run[k] = head[k] = T(0);
        bool seen = false;
#pragma unroll 1
        for (int i = 0; i < G; ++i) {
            const int ls = G * p + i;  // the one-vector lane whose 4 entries these are
            const uint4 t = __ldg(gw + ls);
            const uint32_t w[4] = {t.x, t.y, t.z, t.w};
            T v[4];
            if (UNIT) {
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = T(1);
            } else if (NV == 4) {
                unpack(ld_stream(reinterpret_cast<const VT *>(gv) + ls, pol), v);
            } else {
                unpack(ld_stream(reinterpret_cast<const VT *>(gv) + ls, pol), v);
                unpack(ld_stream(reinterpret_cast<const VT *>(gv) + 32 + ls, pol), v + 2);
            }
            T xv[4][V];
#pragma unroll
            for (int j = 0; j < 4; ++j) load_x(w[j] & kRsColMask, xv[j]);
            T xo[GV ? 4 : 1][V];
            if (GV) {  // the entries' own rows of xo (the padding row: zeros)
                int32_t o = ord;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    o += (int32_t)(w[j] >> 31);
                    const T *po = gvp->xo + (o < nord ? rid(o) : 0) * gvp->ldo + c0;
                    if (o < nord && c0 < nrhs && gvp->xovec) {
                        unpack(__ldg(reinterpret_cast<const VT *>(po)), xo[GV ? j : 0]);
                    } else {
#pragma unroll
                        for (int k = 0; k < V; ++k)
                            xo[GV ? j : 0][k] = o < nord && c0 + k < nrhs ? __ldg(po + k) : T(0);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool f = (w[j] >> 31) != 0;
                if (GV) {  // value gradient of this entry: the group's dot product
                    T dot = T(0);
#pragma unroll
                    for (int k = 0; k < V; ++k)
                        if (c0 + k < nrhs) dot = fma(xv[j][k], xo[GV ? j : 0][k], dot);
#pragma unroll
                    for (int d = 1; d < G; d <<= 1) dot += __shfl_xor_sync(kFull, dot, d);
                    if (q == 0) {
                        T *pg = gvp->gv + (int64_t)c * 128 + 4 * ls + j;
                        *pg = gvp->accum ? *pg + dot : dot;
                    }
                }
                if (f && seen) store_y(rid(ord), run);  // a row whole inside the group
#pragma unroll
                for (int k = 0; k < V; ++k) {
                    head[k] = (f && !seen) ? run[k] : head[k];
                    run[k] = fma(v[j], xv[j][k], f ? T(0) : run[k]);
                }
                seen = seen || f;
                ord += f ? 1 : 0;
            }
        }
        // rows across groups: inclusive scan over the groups, reset at groups
        // holding a row start; group 0 continues the previous chunk
        T sc[V];
#pragma unroll
        for (int k = 0; k < V; ++k) sc[k] = (p == 0 && !seen) ? run[k] + carry[k] : run[k];
        bool r = seen;
#pragma unroll
        for (int d = 1; d < P; d <<= 1) {
            const bool ru = __shfl_up_sync(kFull, (int)r, d * G) != 0;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                const T su = __shfl_up_sync(kFull, sc[k], d * G);
                if (p >= d && !r) sc[k] += su;
            }
            if (p >= d) r = r || ru;
        }
        T cin[V];
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const T t = __shfl_up_sync(kFull, sc[k], G);
            cin[k] = p == 0 ? carry[k] : t;
        }
        if (seen) {  // the row this group started in ends here
            T val[V];
#pragma unroll
            for (int k = 0; k < V; ++k) val[k] = cin[k] + head[k];
            if (ordS == first && meta.z >= 0)
                arrive(meta.z, val, 2 * s);
            else if (!(ordS == first && meta.y) && ordS < nord)
                store_y(rid(ordS), val);
        }
#pragma unroll
        for (int k = 0; k < V; ++k) carry[k] = __shfl_sync(kFull, sc[k], (P - 1) * G + q);
        ord0 = __shfl_sync(kFull, ord, (P - 1) * G);
    }
    // the segment's last row: a span's part, or whole here (group 0)
    if (p == 0) {
        if (ord0 == first && meta.z >= 0)
            arrive(meta.z, carry, 2 * s);
        else if (meta.w >= 0)
            arrive(meta.w, carry, 2 * s + 1);
        else if (ord0 < nord && !(ord0 == first && meta.y))
            store_y(rid(ord0), carry);
    }
    __syncwarp();
}

template <typename T, int G, bool UNIT>
__global__ void __launch_bounds__(kRsWarps * 32, 1)
    cb_rowseg_mrhs_kernel(const RowSegDev rs, const T *__restrict__ x, T *__restrict__ y,
                          int nrhs, int64_t ldx, int64_t ldy, int xvec, int yvec) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    {  // rows without entries
        const int64_t total = (int64_t)rs.nempty * nrhs;
        for (int64_t i = ((int64_t)blockIdx.x * kRsWarps + wib) * 32 + lane; i < total;
             i += (int64_t)gridDim.x * kRsWarps * 32)
            y[(int64_t)__ldg(&rs.empty[i / nrhs]) * ldy + i % nrhs] = T(0);
    }
    const int NB = gridDim.x, b = blockIdx.x;
    const int sb0 = (int)((int64_t)b * rs.nseg / NB);
    const int sb1 = (int)((int64_t)(b + 1) * rs.nseg / NB);
    const RsMat<T> A{rs.chunks, rs.rowmap, x, y, ldx, ldy, nrhs, rs.nord, xvec, yvec};
    const RsSpans<T> S{rs.spans, rs.counters, static_cast<T *>(rs.part)};
    const uint64_t pol = dev::policy_evict_first();
    for (int s = sb0 + wib; s < sb1; s += kRsWarps)
        rs_mrhs_segment<T, G, UNIT>(A, s * rs.M, min(rs.nch, s * rs.M + rs.M),
                                    __ldg(&rs.meta[s]), s, S, lane, pol);
}

// The fused adjoint on a transposed stream: A^T G into y and the value
// gradient of every entry (kRsGvWarps warps per CTA: the gradient's registers fit without
// spills; each CTA's warps stride over its share of the segments).
template <typename T, int G>
__global__ void __launch_bounds__(kRsGvWarps * 32, 1)
    cb_rowseg_gv_kernel(const RowSegDev rs, const T *__restrict__ x, T *__restrict__ y,
                        int nrhs, int64_t ldx, int64_t ldy, int xvec, int yvec,
                        const RsGV<T> gvp) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    {  // rows without entries
        const int64_t total = (int64_t)rs.nempty * nrhs;
        for (int64_t i = ((int64_t)blockIdx.x * kRsGvWarps + wib) * 32 + lane; i < total;
             i += (int64_t)gridDim.x * kRsGvWarps * 32)
            y[(int64_t)__ldg(&rs.empty[i / nrhs]) * ldy + i % nrhs] = T(0);
    }
    const int NB = gridDim.x, b = blockIdx.x;
    const int sb0 = (int)((int64_t)b * rs.nseg / NB);
    const int sb1 = (int)((int64_t)(b + 1) * rs.nseg / NB);
    const RsMat<T> A{rs.chunks, rs.rowmap, x, y, ldx, ldy, nrhs, rs.nord, xvec, yvec};
    const RsSpans<T> S{rs.spans, rs.counters, static_cast<T *>(rs.part)};
    const uint64_t pol = dev::policy_evict_first();
    for (int s = sb0 + wib; s < sb1; s += kRsGvWarps)
        rs_mrhs_segment<T, G, false, true>(A, s * rs.M, min(rs.nch, s * rs.M + rs.M),
                                           __ldg(&rs.meta[s]), s, S, lane, pol, &gvp);
}

// A batch over the streams (kRsBatchWarps warps per CTA: the kernel holds
// every lanes-per-entry variant, so it is given more registers per thread):
// warps take segments segs[0 .. nseg) ({matrix, first chunk, end chunk, -},
// with meta[] and the batch's own spans; queued by lanes per entry) from
// sched[0], choosing the segment code from the matrix's entry; the last warp
// out (sched[1]) resets both words for the next launch.
template <typename T>
__global__ void __launch_bounds__(kRsBatchWarps * 32, 1)
    cb_rowseg_batch_kernel(const RsBatchMat *__restrict__ mats, const int4 *__restrict__ segs,
                           const int4 *__restrict__ meta, int32_t nseg, uint32_t *sched,
                           const int2 *__restrict__ empty, int64_t nempty, const int4 *spans,
                           int32_t *counters, T *part) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (int64_t i = ((int64_t)blockIdx.x * kRsBatchWarps + wib) * 32 + lane; i < nempty;
         i += (int64_t)gridDim.x * kRsBatchWarps * 32) {  // rows without entries
        const int2 e = __ldg(&empty[i]);
        const RsBatchMat &m = mats[e.x];
        for (int k = 0; k < m.nrhs; ++k) static_cast<T *>(m.y)[(int64_t)e.y * m.ldy + k] = T(0);
    }
    const RsSpans<T> S{spans, counters, part};
    const uint64_t pol = dev::policy_evict_first();
    while (true) {
        int si = 0;
        if (lane == 0) si = (int)atomicAdd(&sched[0], 1u);
        si = __shfl_sync(kFull, si, 0);
        if (si >= nseg) break;
        const int4 sg = __ldg(&segs[si]);
        const RsBatchMat &m = mats[sg.x];
        const RsMat<T> A{m.chunks, m.rowmap, static_cast<const T *>(m.x), static_cast<T *>(m.y),
                         m.ldx, m.ldy, m.nrhs, m.nord, m.xvec, m.yvec};
        const int4 mt = __ldg(&meta[si]);
        constexpr int GMAX = sizeof(T) == 4 ? 4 : 8;
        switch (m.g * 2 + (m.unit ? 1 : 0)) {
            case 2: rs_mrhs_segment<T, 1, false>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            case 3: rs_mrhs_segment<T, 1, true>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            case 4: rs_mrhs_segment<T, 2, false>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            case 5: rs_mrhs_segment<T, 2, true>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            case 8: rs_mrhs_segment<T, 4, false>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            case 9: rs_mrhs_segment<T, 4, true>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            case 16: rs_mrhs_segment<T, GMAX, false>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            case 17: rs_mrhs_segment<T, GMAX, true>(A, sg.y, sg.z, mt, si, S, lane, pol); break;
            default: break;
        }
    }
    // the last warp out resets the scheduler words for the next launch
    if (lane == 0) {
        __threadfence();
        if (atomicAdd(&sched[1], 1u) == gridDim.x * kRsBatchWarps - 1) {
            atomicExch(&sched[0], 0u);
            atomicExch(&sched[1], 0u);
        }
    }
}

// Stream values refreshed from the tile payload: chunks[value of entry
// vpos[v]] = payload value v.
template <typename T>
__global__ void cb_rowseg_values_kernel(const RowSegDev rs, const uint8_t *__restrict__ payload,
                                        const uint64_t *__restrict__ val_off, int64_t nvals) {
    constexpr int64_t C = 32 * kRsK, NV = 16 / sizeof(T);
    constexpr int64_t CB = C * (4 + (int64_t)sizeof(T));
    uint8_t *chunks = const_cast<uint8_t *>(rs.chunks);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvals;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = __ldg(&rs.vpos[v]);
        if (e < 0) continue;  // a DENSE slot outside the valid rows and columns
        const int64_t c = e / C, i = e % C, l = i / kRsK, j = i % kRsK;
        const int64_t pos = (j / NV) * 32 * NV + l * NV + j % NV;
        *reinterpret_cast<T *>(chunks + c * CB + 4 * C + pos * (int64_t)sizeof(T)) =
            *reinterpret_cast<const T *>(payload + __ldg(&val_off[v]));
    }
}


// The balanced schedule (plans built with row_owned = 0): warps take whole
// groups (the reference's CTAs of waves_per_block blocks, balanced by its
// permutation), each lane a quad of 4 entries at a time; a run of one row
// inside the quad is summed in registers and added into y with an atomic
// (the reference's accumulate_output without CB_ROW_OWNED,
// cb-spmv-dcu.hpp:149-157).  y is zeroed before the launch.
constexpr int kBalWarps = 8;
template <typename T>
__global__ void __launch_bounds__(kBalWarps * 32)
    cb_balanced_kernel(const BalancedDev b, const T *__restrict__ x, T *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = (int64_t)gridDim.x * kBalWarps;
    for (int64_t g = (int64_t)blockIdx.x * kBalWarps + (threadIdx.x >> 5); g < b.ngroups;
         g += nw) {
        const int64_t q1 = __ldg(&b.gstart[g + 1]);
        for (int64_t q = __ldg(&b.gstart[g]) + lane; q < q1; q += 32) {
            const uint4 r4 = __ldg(&b.rows[q]), c4 = __ldg(&b.cols[q]);
            const uint32_t r[4] = {r4.x, r4.y, r4.z, r4.w}, c[4] = {c4.x, c4.y, c4.z, c4.w};
            T v[4];
            if (sizeof(T) == 4) {
                unpack(__ldg(reinterpret_cast<const float4 *>(b.vals) + q),
                       reinterpret_cast<float *>(v));
            } else {
                unpack(__ldg(reinterpret_cast<const double2 *>(b.vals) + 2 * q),
                       reinterpret_cast<double *>(v));
                unpack(__ldg(reinterpret_cast<const double2 *>(b.vals) + 2 * q + 1),
                       reinterpret_cast<double *>(v) + 2);
            }
            T xv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) xv[j] = r[j] != kBalSkip ? __ldg(x + c[j]) : T(0);
            uint32_t rr = r[0];
            T run = v[0] * xv[0];
#pragma unroll
            for (int j = 1; j < 4; ++j) {
                if (r[j] == rr) {
                    run = fma(v[j], xv[j], run);
                } else {
                    if (rr != kBalSkip) atomicAdd(&y[rr], run);
                    rr = r[j];
                    run = v[j] * xv[j];
                }
            }
            if (rr != kBalSkip) atomicAdd(&y[rr], run);
        }
    }
}

// Balanced stream values refreshed from the tile payload (skip entries 0).
template <typename T>
__global__ void cb_balanced_values_kernel(const BalancedDev b, const uint8_t *__restrict__ payload) {
    T *vals = static_cast<T *>(const_cast<void *>(b.vals));
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < 4 * b.nquads;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t off = __ldg(&b.eoff[e]);
        vals[e] = off >= 0 ? *reinterpret_cast<const T *>(payload + off) : T(0);
    }
}

}  // namespace

template <typename T, bool UNIT>
const void *rowseg_fn() {
    return reinterpret_cast<const void *>(cb_rowseg_kernel<T, UNIT>);
}

template <typename T, bool UNIT>
cudaError_t launch_rowseg_t(const DevLayout &d, const void *x, void *y, size_t smem,
                            cudaStream_t stream) {
    const void *fn = rowseg_fn<T, UNIT>();
    cudaError_t e = dev_enable_smem(fn, smem);
    if (e != cudaSuccess) return e;
    dev_resident_l1(fn, kRsWarps * 32, smem);  // sets the carveout
    // the grid the segments and windows were assigned for
    cb_rowseg_kernel<T, UNIT><<<(unsigned)d.rs.G, kRsWarps * 32, smem, stream>>>(
        d.rs, static_cast<const T *>(x), static_cast<T *>(y));
    return cudaSuccess;
}

int64_t rowseg_warps(int f32) {
    // the x window in shared memory; the carveout leaves the rest of the
    // unified L1/shared memory to the L1 (the other x gathers)
    const void *fn = f32 ? rowseg_fn<float, false>() : rowseg_fn<double, false>();
    if (dev_enable_smem(fn, (size_t)kRsWindowBytes) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (int64_t)dev_sms() * dev_resident_l1(fn, kRsWarps * 32, (size_t)kRsWindowBytes) *
           kRsWarps;
}

cudaError_t launch_rowseg(const DevLayout &d, const void *x, void *y, cudaStream_t stream) {
    if (!d.rs.chunks || d.rs.nseg <= 0 || d.rs.G <= 0 || !d.rs.wbase)
        return cudaErrorInvalidValue;
    const size_t smem = (size_t)d.rs.W * (d.f32 ? 4 : 8);
    const cudaError_t e =
        d.f32 ? (d.rs.unit ? launch_rowseg_t<float, true>(d, x, y, smem, stream)
                           : launch_rowseg_t<float, false>(d, x, y, smem, stream))
              : (d.rs.unit ? launch_rowseg_t<double, true>(d, x, y, smem, stream)
                           : launch_rowseg_t<double, false>(d, x, y, smem, stream));
    if (e != cudaSuccess) return e;
    note_launch();
    return cudaGetLastError();
}

template <typename T, int G, bool UNIT>
cudaError_t launch_mrhs_g(const DevLayout &d, const T *x, T *y, int r, int64_t ldx, int64_t ldy,
                          int xvec, int yvec, cudaStream_t stream) {
    const void *fn = reinterpret_cast<const void *>(cb_rowseg_mrhs_kernel<T, G, UNIT>);
    dev_resident_l1(fn, kRsWarps * 32, 0);  // sets the carveout: all L1
    cb_rowseg_mrhs_kernel<T, G, UNIT><<<(unsigned)d.rs.G, kRsWarps * 32, 0, stream>>>(
        d.rs, x, y, r, ldx, ldy, xvec, yvec);
    note_launch();
    return cudaGetLastError();
}

template <typename T, bool UNIT>
cudaError_t launch_mrhs_t(const DevLayout &d, const T *x, T *y, int nrhs, int64_t ldx,
                          int64_t ldy, cudaStream_t stream) {
    constexpr int V = 16 / sizeof(T);
    // slabs of at most kRsMaxRhs right-hand sides, one launch each
    for (int c = 0; c < nrhs; c += kRsMaxRhs) {
        const int r = std::min(kRsMaxRhs, nrhs - c);
        const int xvec = ldx % V == 0 && reinterpret_cast<uintptr_t>(x + c) % 16 == 0;
        const int yvec = ldy % V == 0 && reinterpret_cast<uintptr_t>(y + c) % 16 == 0;
        const int g = rs_lanes_per_entry(sizeof(T) == 4, r);
        cudaError_t e;
        switch (g) {
            case 1: e = launch_mrhs_g<T, 1, UNIT>(d, x + c, y + c, r, ldx, ldy, xvec, yvec, stream); break;
            case 2: e = launch_mrhs_g<T, 2, UNIT>(d, x + c, y + c, r, ldx, ldy, xvec, yvec, stream); break;
            case 4: e = launch_mrhs_g<T, 4, UNIT>(d, x + c, y + c, r, ldx, ldy, xvec, yvec, stream); break;
            default: e = launch_mrhs_g<T, (16 / sizeof(T) == 2 ? 8 : 4), UNIT>(
                         d, x + c, y + c, r, ldx, ldy, xvec, yvec, stream);
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_rowseg_mrhs(const DevLayout &d, const void *x, void *y, int nrhs,
                               int64_t ldx, int64_t ldy, cudaStream_t stream) {
    if (!d.rs.chunks || d.rs.nseg <= 0 || d.rs.G <= 0 || nrhs < 1) return cudaErrorInvalidValue;
    if (d.f32)
        return d.rs.unit ? launch_mrhs_t<float, true>(d, static_cast<const float *>(x),
                                                      static_cast<float *>(y), nrhs, ldx, ldy, stream)
                         : launch_mrhs_t<float, false>(d, static_cast<const float *>(x),
                                                       static_cast<float *>(y), nrhs, ldx, ldy, stream);
    return d.rs.unit ? launch_mrhs_t<double, true>(d, static_cast<const double *>(x),
                                                   static_cast<double *>(y), nrhs, ldx, ldy, stream)
                     : launch_mrhs_t<double, false>(d, static_cast<const double *>(x),
                                                    static_cast<double *>(y), nrhs, ldx, ldy, stream);
}

template <typename T, int G>
cudaError_t launch_gv_g(const DevLayout &d, const T *g, T *gx, int r, int64_t ldg,
                        int64_t ldgx, int xvec, int yvec, const RsGV<T> &gvp,
                        cudaStream_t stream) {
    const void *fn = reinterpret_cast<const void *>(cb_rowseg_gv_kernel<T, G>);
    dev_resident_l1(fn, kRsGvWarps * 32, 0);  // sets the carveout: all L1
    cb_rowseg_gv_kernel<T, G><<<(unsigned)d.rs.G, kRsGvWarps * 32, 0, stream>>>(
        d.rs, g, gx, r, ldg, ldgx, xvec, yvec, gvp);
    note_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_gv_t(const DevLayout &d, const T *g, T *gx, int nrhs, int64_t ldg,
                        int64_t ldgx, const T *x, int64_t ldx, T *gv, cudaStream_t stream) {
    constexpr int V = 16 / sizeof(T);
    for (int c = 0; c < nrhs; c += kRsMaxRhs) {  // slabs of 16: the gradient adds up
        const int r = std::min(kRsMaxRhs, nrhs - c);
        const int xvec = ldg % V == 0 && reinterpret_cast<uintptr_t>(g + c) % 16 == 0;
        const int yvec = ldgx % V == 0 && reinterpret_cast<uintptr_t>(gx + c) % 16 == 0;
        const RsGV<T> gvp{x + c, ldx,
                          (int32_t)(ldx % V == 0 && reinterpret_cast<uintptr_t>(x + c) % 16 == 0),
                          (int32_t)(c > 0), gv};
        const int gl = rs_lanes_per_entry(sizeof(T) == 4, r);
        cudaError_t e;
        switch (gl) {
            case 1: e = launch_gv_g<T, 1>(d, g + c, gx + c, r, ldg, ldgx, xvec, yvec, gvp, stream); break;
            case 2: e = launch_gv_g<T, 2>(d, g + c, gx + c, r, ldg, ldgx, xvec, yvec, gvp, stream); break;
            case 4: e = launch_gv_g<T, 4>(d, g + c, gx + c, r, ldg, ldgx, xvec, yvec, gvp, stream); break;
            default: e = launch_gv_g<T, (16 / sizeof(T) == 2 ? 8 : 4)>(
                         d, g + c, gx + c, r, ldg, ldgx, xvec, yvec, gvp, stream);
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_rowseg_adjoint(const DevLayout &d, const void *g, void *gx, int nrhs,
                                  int64_t ldg, int64_t ldgx, const void *x, int64_t ldx,
                                  void *gv, cudaStream_t stream) {
    if (!d.rs.chunks || d.rs.unit || d.rs.nseg <= 0 || d.rs.G <= 0 || nrhs < 1)
        return cudaErrorInvalidValue;
    if (d.f32)
        return launch_gv_t<float>(d, static_cast<const float *>(g), static_cast<float *>(gx),
                                  nrhs, ldg, ldgx, static_cast<const float *>(x), ldx,
                                  static_cast<float *>(gv), stream);
    return launch_gv_t<double>(d, static_cast<const double *>(g), static_cast<double *>(gx),
                               nrhs, ldg, ldgx, static_cast<const double *>(x), ldx,
                               static_cast<double *>(gv), stream);
}

cudaError_t launch_balanced(const DevLayout &d, const void *x, void *y, cudaStream_t stream) {
    if (!d.bal.rows) return cudaErrorInvalidValue;
    const size_t vsz = d.f32 ? 4 : 8;
    cudaError_t e = cudaMemsetAsync(y, 0, (size_t)d.m * vsz, stream);
    if (e != cudaSuccess) return e;
    const void *fn = d.f32 ? reinterpret_cast<const void *>(cb_balanced_kernel<float>)
                           : reinterpret_cast<const void *>(cb_balanced_kernel<double>);
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>((d.bal.ngroups + kBalWarps - 1) / kBalWarps,
                             (int64_t)dev_sms() * dev_resident(fn, kBalWarps * 32, 0)));
    if (d.f32)
        cb_balanced_kernel<float><<<(unsigned)grid, kBalWarps * 32, 0, stream>>>(
            d.bal, static_cast<const float *>(x), static_cast<float *>(y));
    else
        cb_balanced_kernel<double><<<(unsigned)grid, kBalWarps * 32, 0, stream>>>(
            d.bal, static_cast<const double *>(x), static_cast<double *>(y));
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_balanced_values(const DevLayout &d, cudaStream_t stream) {
    if (!d.bal.rows || !d.bal.eoff || d.bal.nquads <= 0) return cudaSuccess;
    const unsigned grid =
        (unsigned)std::min<int64_t>((4 * d.bal.nquads + 255) / 256, (int64_t)dev_sms() * 16);
    if (d.f32)
        cb_balanced_values_kernel<float><<<grid, 256, 0, stream>>>(d.bal, d.payload);
    else
        cb_balanced_values_kernel<double><<<grid, 256, 0, stream>>>(d.bal, d.payload);
    note_launch();
    return cudaGetLastError();
}

int rs_lanes_per_entry(int f32, int nrhs) {
    const int V = f32 ? 4 : 2, gmax = f32 ? 4 : 8;
    int g = 1;
    while (g * V < std::min(nrhs, kRsMaxRhs) && g < gmax) g *= 2;
    return g;
}

int64_t rowseg_batch_warps(int f32) {
    const void *fn = f32 ? reinterpret_cast<const void *>(cb_rowseg_batch_kernel<float>)
                         : reinterpret_cast<const void *>(cb_rowseg_batch_kernel<double>);
    return (int64_t)dev_sms() * dev_resident_l1(fn, kRsBatchWarps * 32, 0) * kRsBatchWarps;
}

cudaError_t launch_rowseg_batch(int f32, const RsBatchMat *mats, const int4 *segs,
                                const int4 *meta, int32_t nseg, uint32_t *sched, int64_t nwarps,
                                const int2 *empty, int64_t nempty, const int4 *spans,
                                int32_t *counters, void *part, cudaStream_t stream) {
    if (nwarps <= 0 || nwarps % kRsBatchWarps) return cudaErrorInvalidValue;
    const unsigned grid = (unsigned)(nwarps / kRsBatchWarps);
    if (f32)
        cb_rowseg_batch_kernel<float><<<grid, kRsBatchWarps * 32, 0, stream>>>(
            mats, segs, meta, nseg, sched, empty, nempty, spans, counters,
            static_cast<float *>(part));
    else
        cb_rowseg_batch_kernel<double><<<grid, kRsBatchWarps * 32, 0, stream>>>(
            mats, segs, meta, nseg, sched, empty, nempty, spans, counters,
            static_cast<double *>(part));
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_rowseg_values(const DevLayout &d, int64_t nvals, const uint64_t *val_off,
                                 cudaStream_t stream) {
    if (!d.rs.chunks || !d.rs.vpos || nvals <= 0) return cudaSuccess;
    const unsigned grid =
        (unsigned)std::min<int64_t>((nvals + 255) / 256, (int64_t)dev_sms() * 16);
    if (d.f32)
        cb_rowseg_values_kernel<float><<<grid, 256, 0, stream>>>(d.rs, d.payload, val_off, nvals);
    else
        cb_rowseg_values_kernel<double><<<grid, 256, 0, stream>>>(d.rs, d.payload, val_off,
                                                                  nvals);
    note_launch();
    return cudaGetLastError();
}

}  // namespace cb
