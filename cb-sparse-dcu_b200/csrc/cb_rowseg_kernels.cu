// Row-segment stream kernel (layout in cb_rowseg.hpp): y = A x for matrices
// whose stored entries are all in COO blocks.
//
// One CTA of kRsWarps warps per SM; warp w of CTA b takes the segments
// sb0 + w, sb0 + w + kRsWarps, ... of the CTA's share [sb0, sb1) of the
// segments (about one per warp).  Per chunk a lane
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
// order across lanes, fixed by the layout: results are bitwise reproducible.
// The reference adds each entry into its row with an atomic
// (cb-spmv-dcu.hpp:423-426); the sums here are the same rows' sums.
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
        const int64_t c = e / C, i = e % C, l = i / kRsK, j = i % kRsK;
        const int64_t pos = (j / NV) * 32 * NV + l * NV + j % NV;
        *reinterpret_cast<T *>(chunks + c * CB + 4 * C + pos * (int64_t)sizeof(T)) =
            *reinterpret_cast<const T *>(payload + __ldg(&val_off[v]));
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
