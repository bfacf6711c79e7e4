// Device helpers shared by the CB-SpMV kernels (cb_kernels.cu, cb_spmm.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace cb {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kColMask = (1u << 27) - 1;  // COO entry: row << 27 | column

__host__ __device__ constexpr uint32_t a16(uint32_t x) { return (x + 15u) & ~15u; }

// Adds K COO entries held by this lane -- slot u is the tile entry at position
// pos0 + stride * u, valid while below E -- into the lane's accumulators
// (row r at myacc[r * 32]).  A tile's COO entries are stored sorted by row, so
// the rows of a lane's slots never decrease: equal-row slots are summed in
// registers, each run of them adds to the accumulator once, and since
// different runs are different rows every load can be issued before any store.
template <typename T, int K>
__device__ __forceinline__ void add_entries(T *myacc, const uint32_t *w, const T *v,
                                            const T *xv, int pos0, int stride, int E) {
    uint32_t r[K];
    T s[K];
#pragma unroll
    for (int u = 0; u < K; ++u) r[u] = w[u] >> 27;
#pragma unroll
    for (int u = 0; u < K; ++u)
        s[u] = fma(v[u], xv[u], (u > 0 && r[u] == r[u > 0 ? u - 1 : 0]) ? s[u > 0 ? u - 1 : 0]
                                                                          : T(0));
    bool f[K];
#pragma unroll
    for (int u = 0; u < K; ++u) {
        const bool valid = pos0 + stride * u < E;
        const bool more = u + 1 < K && pos0 + stride * (u + 1) < E &&
                          r[u + 1 < K ? u + 1 : u] == r[u];
        f[u] = valid && !more;
    }
    T a[K];
#pragma unroll
    for (int u = 0; u < K; ++u) a[u] = f[u] ? myacc[r[u] * 32] : T(0);
#pragma unroll
    for (int u = 0; u < K; ++u)
        if (f[u]) myacc[r[u] * 32] = a[u] + s[u];
}

// Adds a tile's COO section into the warp's row accumulators acc[0, BS)
// (shared memory).  The section is stored in lane slices (coo_slice_pos in
// cb_layout.hpp): lane l holds the consecutive entries of positions
// 32 j + l < E, j = 0, 1, ... -- w[j] their index words (row << 27 | column),
// xv[j] their gathered x values, sval the staged values (unused when unit).
//   1. Each lane sums its slice along its rows in registers.  The slice's
//      first row (the head) may have begun in earlier lanes and its last (the
//      tail) may go on in later ones; rows that begin and end inside the slice
//      are complete and the lane adds them into acc itself.
//   2. A segmented shuffle scan over the lanes sums the tails of a row that
//      runs across several lanes; the lane where such a row ends adds the
//      row's total (a head that goes on from the previous lane takes that
//      lane's running sum).
// Every row of the tile is added into acc exactly once, by one lane, so the
// lanes never write the same accumulator and the order of the sums is fixed
// by the layout (bitwise reproducible results).  Ends with a __syncwarp.
template <typename T, int BS, int K>
__device__ __forceinline__ void slice_sums(T *__restrict__ acc, const uint32_t (&w)[K],
                                           const T (&xv)[K], const T *__restrict__ sval,
                                           int unit, int E, int lane) {
    constexpr uint32_t kNone = 63;  // row of an empty lane (after every real row)
    const bool have = lane < E;
    const uint32_t rh = have ? (w[0] >> 27) : kNone;  // head row
    uint32_t rc = rh;                                 // row of the running sum
    T run = have ? (unit ? T(1) : sval[lane]) * xv[0] : T(0);
    T head = T(0);
    bool split = false;  // the slice holds more than one row
    // branch-free: every step selects; only a row complete inside the slice
    // (a change of row after the first) updates acc, under a predicate
#pragma unroll
    for (int j = 1; j < K; ++j) {
        if (32 * j >= E) break;  // warp-uniform
        const int pos = 32 * j + lane;
        const bool valid = pos < E;
        const uint32_t r = valid ? (w[j] >> 27) : rc;
        const T p = valid ? (unit ? T(1) : sval[pos]) * xv[j] : T(0);
        const bool chg = r != rc;
        if (chg && split) acc[rc] += run;
        head = (chg && !split) ? run : head;
        split = split || chg;
        run = chg ? p : run + p;
        rc = r;
    }
    // rows across lanes: the running sum `run` of the tail row rc
    const uint32_t rt_prev = __shfl_up_sync(kFull, rc, 1);
    const uint32_t rh_next = __shfl_down_sync(kFull, rh, 1);
    const bool cont = lane > 0 && rh == rt_prev;  // my head goes on from the previous lane
    const uint32_t heads = __ballot_sync(kFull, !cont || split);
    const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
    const uint32_t longest = __reduce_max_sync(kFull, (uint32_t)(lane - start + 1));
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        if ((uint32_t)d >= longest) break;
        const T t = __shfl_up_sync(kFull, run, d);
        if (lane - d >= start) run += t;
    }
    const T prev = __shfl_up_sync(kFull, run, 1);
    if (split) acc[rh] += cont ? head + prev : head;
    if ((lane == 31 || rh_next != rc) && rc < (uint32_t)BS) acc[rc] += run;
    __syncwarp();
}

// Element (r, c) of a DENSE block payload: bs*bs values, or for a unit-valued
// plan a bs*bs-bit mask (bit r*bs + c) of the entries equal to 1.
template <typename T, int BS>
__device__ __forceinline__ T dense_at(const uint8_t *pb, int unit, int r, int c) {
    const int i = r * BS + c;
    if (unit) return T((pb[i >> 3] >> (i & 7)) & 1);
    return reinterpret_cast<const T *>(pb)[i];
}

// CSR and DENSE blocks of a tile, read from global memory, added into the
// lane-private accumulators (row r at myacc[r * 32]); used by the direct
// kernel (the streaming kernel keeps a lighter loop: this one's registers
// cost its COO path 3-5%).  bs = 16: each
// half-warp takes a block, one lane per row, so two blocks' dependent load
// chains (row pointers, then columns and values) are in flight at a time;
// bs = 32: a block at a time.  prefetch(jb2) brings the blocks of step jb2
// into L1, one 128-byte line per lane of a block's lanes, a step ahead of
// their reads.  bd: lane j holds the descriptor of block j (j < nxt); xt: the
// blocks' x columns, bs per block; base: the tile's payload.
template <typename T, int BS>
__device__ __forceinline__ void add_csr_dense(const uint8_t *base, const uint4 bd, int nxt,
                                              const T *xt, T *myacc, int unit, int lane) {
    auto prefetch = [&](int jb2) {
        const int j2 = jb2 + lane / BS;
        const int j2c = min(j2, nxt - 1);
        const uint32_t off2 = __shfl_sync(kFull, bd.x, j2c);
        const uint32_t mb2 = __shfl_sync(kFull, bd.y, j2c);
        if (j2 >= nxt) return;
        const uint32_t k2 = (mb2 >> 3) & 2047;
        constexpr uint32_t isz = BS == 16 ? 1u : 2u;
        const uint32_t bytes = (mb2 & 3) == 1
            ? a16((BS + 1 + k2) * isz) + (unit ? 0u : k2 * (uint32_t)sizeof(T))
            : (unit ? BS * BS / 8u : BS * BS * (uint32_t)sizeof(T));
        for (uint32_t b = (uint32_t)(lane % BS) * 128u; b < bytes; b += BS * 128u)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(base + off2 + b));
    };
    if (nxt) prefetch(0);
    if (BS == 16) {
        for (int jb = 0; jb < nxt; jb += 2) {
            prefetch(jb + 2);
            const int j = jb + (lane >> 4);
            const int jc = min(j, nxt - 1);
            const uint32_t off = __shfl_sync(kFull, bd.x, jc);
            const uint32_t mb = __shfl_sync(kFull, bd.y, jc);
            if (j < nxt) {
                const int k = (mb >> 3) & 2047;
                const uint8_t *pb = base + off;
                const T *xb = &xt[j * BS];
                const int row = lane & 15;
                T sum = T(0);
                if ((mb & 3) == 1) {
                    const uint8_t *rp = pb;
                    const uint8_t *ci = rp + BS + 1;
                    const T *vv = reinterpret_cast<const T *>(
                        pb + a16((uint32_t)(BS + 1 + k)));
                    const int kb = __ldg(&rp[row]), ke = __ldg(&rp[row + 1]);
#pragma unroll 4
                    for (int q = kb; q < ke; ++q)
                        sum += (unit ? T(1) : __ldg(&vv[q])) * xb[__ldg(&ci[q])];
                } else {
#pragma unroll
                    for (int c = 0; c < BS; ++c)
                        sum += dense_at<T, BS>(pb, unit, row, (c + row) & 15) *
                               xb[(c + row) & 15];
                }
                myacc[row * 32] += sum;
            }
        }
    }
    // bs = 32: a block at a time, one lane per row
    for (int jb = 0; BS == 32 && jb < nxt; ++jb) {
        prefetch(jb + 1);
        const uint32_t off = __shfl_sync(kFull, bd.x, jb);
        const uint32_t mb = __shfl_sync(kFull, bd.y, jb);
        const int k = (mb >> 3) & 2047;
        const uint8_t *pb = base + off;
        const T *xb = &xt[jb * BS];
        T sum = T(0);
        if ((mb & 3) == 1) {
            const uint16_t *rp = reinterpret_cast<const uint16_t *>(pb);
            const uint16_t *ci = rp + BS + 1;
            const T *vv = reinterpret_cast<const T *>(
                pb + a16((uint32_t)((BS + 1 + k) * sizeof(uint16_t))));
            const int kb = __ldg(&rp[lane]), ke = __ldg(&rp[lane + 1]);
#pragma unroll 4
            for (int q = kb; q < ke; ++q)
                sum += (unit ? T(1) : __ldg(&vv[q])) * xb[__ldg(&ci[q])];
        } else {
#pragma unroll 8
            for (int c = 0; c < BS; ++c) sum += dense_at<T, BS>(pb, unit, lane, c) * xb[c];
        }
        myacc[lane * 32] += sum;
    }
}

// ---- bulk asynchronous copies (TMA, no multicast) completing on mbarriers.
// Every wait is bounded: after kWaitLimit polls it sets *err and gives up.
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// orders this thread's (and, after a warp barrier, its warp's) generic
// shared-memory accesses before later async-proxy writes (bulk copies)
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// global -> this CTA's shared memory, completion counted on `bar`
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
// Waits for the phase `parity` of `bar` to complete, polling at most `limit`
// times; on give-up sets *err (the launch's error word: host-mapped memory the
// host reads without a copy, or device memory) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t *err,
                                          uint32_t limit = kWaitLimit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    *reinterpret_cast<volatile uint32_t *>(err) = 1u;
    __threadfence_system();
    return false;
}

}  // namespace dev
}  // namespace cb
