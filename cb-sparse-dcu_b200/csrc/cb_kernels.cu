// sm_100a kernels of the CB-SpMV.  The reference's `comp` and `gather` kernels
// (cb-spmv-dcu.hpp:159-1084) become two tile kernels over this library's own
// device layout, in which COO columns are resolved through the gather list at
// build time and CSR/DENSE blocks stage their bs gathered x values per block:
//   * cb_spmv_stream_kernel (COO-dominant matrices, one right-hand side):
//     per-warp bulk-async (TMA) double-buffered tiles, host-balanced
//     contiguous tile ranges, x gathers of the next tile in flight while the
//     current one is added up;
//   * cb_spmv_tile_kernel ("direct"; CSR/DENSE-heavy matrices, one
//     right-hand side): persistent warps take block-row units from a global
//     counter.
// Both add each COO entry's val * x[col] into its row (the reference's
// per-entry accumulate_output, cb-spmv-dcu.hpp:423-426) in a lane-private
// shared accumulator -- no atomics, a fixed order, bitwise reproducible -- and
// reduce the 32 copies of a row once per unit (direct) or once per run of a
// block row's tiles (streaming).  CSR blocks: the streaming kernel uses 32/bs
// lanes per row (the reference's LANES_PER_ROW, macros.h:84, re-derived for
// 32 lanes), the direct kernel one lane per row and a half-warp per block
// (bs = 16); DENSE blocks 2 lanes per row (streaming, bs = 16) or 1.  Several
// right-hand sides run in the staged kernel (cb_spmm.cu).  A block row split over
// several tiles (or warps) leaves partial sums; the last tile (or warp) to
// arrive on the row's counter adds them in a fixed order and stores y.  No
// tile waits on another (the reference spins on a row epoch,
// cb-spmv-dcu.hpp:238-282).  Also: value refresh and value-gradient kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "cb_device.cuh"
#include "cb_kernels.hpp"

namespace cb {
namespace {

// kernels this library has launched (all devices, all plans)
std::atomic<int64_t> g_kernel_launches{0};

using dev::a16;
using dev::add_csr_dense;
using dev::add_entries;
using dev::kColMask;
using dev::dense_at;
using dev::kFull;
constexpr int kWarps = 8;

__host__ __device__ constexpr int max_xt(int bs) { return bs == 16 ? 16 : 8; }

// Per-warp shared memory.  acc holds one private accumulator per lane and row:
// lane l's copy of row r is acc[r * 32 + l].  Entries accumulate without
// atomics and in a fixed order; a lane only ever touches its own column, so the
// updates of a warp hit 32 distinct banks (fp32) or 16 distinct bank pairs per
// half-warp (fp64) whatever the rows.
template <typename T, int BS>
struct WarpSmem {
    T xt[max_xt(BS) * BS];      // x tiles of the tile's CSR/DENSE blocks
    T acc[BS * 32];
};

template <typename T>
__device__ __forceinline__ T ldg(const T *p) {
    return __ldg(p);
}

// Sums the 32 lane-private copies of row r = lane % BS, clearing them for the
// next tile.  BS = 16: lanes 0-15 sum lanes 0-15's copies, lanes 16-31 the
// upper 16 and hand their half over by shuffle.  Lane r reads the copies in
// the rotated order l = r, r+1, ..., so the 16 (or 32) lanes of one step read
// distinct banks.  Result valid in lanes < BS.
template <typename T, int BS>
__device__ __forceinline__ T reduce_rows(T *acc, int lane) {
    T s = T(0);
    if (BS == 16) {
        const int r = lane & 15, l0 = lane & 16;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            T *p = &acc[r * 32 + l0 + ((q + r) & 15)];
            s += *p;
            *p = T(0);
        }
        s += __shfl_down_sync(kFull, s, 16);
    } else {
#pragma unroll 8
        for (int q = 0; q < 32; ++q) {
            T *p = &acc[lane * 32 + ((q + lane) & 31)];
            s += *p;
            *p = T(0);
        }
    }
    return s;
}

// One vector (x column stride ldx, y stride ldy).  Persistent warps take
// units from a global counter (sched[0]): unit u is tiles [ustart[u],
// ustart[u+1]) of one block row -- the whole row, or pieces of `unit_tiles`
// tiles starting at its first tile -- and add all of the unit's tiles into
// their lane-private accumulators before one reduction and store, so a row's
// tiles need no partial sums unless the row is longer than a unit.  The warp
// whose exit completes sched[1] == number of warps resets both for the next
// launch, so no launch waits on another and no host reset is needed.  kChunk
// COO entries per lane have their loads in flight together.
template <typename T, int BS, int kChunk>
__global__ void __launch_bounds__(kWarps * 32, 4)
    cb_spmv_tile_kernel(const uint4 *__restrict__ tiles, const uint4 *__restrict__ blocks,
                        const uint8_t *__restrict__ payload,
                        const int32_t *__restrict__ block_cols, int gather,
                        const T *__restrict__ x, T *__restrict__ y, int64_t m,
                        int64_t ldx, int64_t ldy, T *__restrict__ partials,
                        int32_t *__restrict__ counters, uint32_t *__restrict__ sched,
                        const uint32_t *__restrict__ ustart, int64_t nunits,
                        int unit_tiles, int unit) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    WarpSmem<T, BS> &S = reinterpret_cast<WarpSmem<T, BS> *>(smem_raw)[wib];
    T *myacc = &S.acc[lane];  // row r at myacc[r * 32]
    for (int t = lane; t < 32 * BS; t += 32) S.acc[t] = T(0);
    __syncwarp();

    auto grab = [&]() -> int64_t {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&sched[0], 1u);
        return (int64_t)__shfl_sync(kFull, t, 0);
    };
    int64_t cur = grab();  // the unit being processed
    while (cur < nunits) {
        const int64_t next = grab();
        const int64_t t0 = __ldg(&ustart[cur]), t1 = __ldg(&ustart[cur + 1]);
        uint4 ta = __ldg(&tiles[2 * t0]), tb = __ldg(&tiles[2 * t0 + 1]);
        for (int64_t tile = t0; tile < t1; ++tile) {
            uint4 na = ta, nb4 = tb;  // the next tile's descriptors, in flight
            if (tile + 1 < t1) {
                na = __ldg(&tiles[2 * tile + 2]);
                nb4 = __ldg(&tiles[2 * tile + 3]);
            }
            const int ncoo = (ta.z >> 8) & 0xff;
            const int nxt = (ta.z >> 16) & 0xff;
            const int E = (int)tb.x;
            const uint8_t *base = payload + (size_t)ta.w * 16;
            uint4 bd = make_uint4(0, 0, 0, 0);  // lane j: CSR/DENSE block j of the tile
            if (lane < nxt) bd = __ldg(&blocks[ta.x + ncoo + lane]);
            const uint32_t *cidx = reinterpret_cast<const uint32_t *>(base);
            const T *cval = reinterpret_cast<const T *>(base + a16(4u * E));

            // x tiles of CSR/DENSE blocks (through the gather list if any)
            for (int c0 = 0; c0 < nxt * BS; c0 += 32) {
                const int t = c0 + lane;
                const int jb = min(t / BS, nxt - 1);
                const uint32_t xb = __shfl_sync(kFull, bd.z, jb);
                const uint32_t mb = __shfl_sync(kFull, bd.y, jb);
                const int c = t % BS;
                const int valid = (mb >> 14) & 63;
                if (t < nxt * BS) {
                    T xv = T(0);
                    if (c < valid) {
                        const int64_t col = gather ? (int64_t)__ldg(&block_cols[xb + c])
                                                   : (int64_t)(xb + c);
                        xv = ldg(&x[col * ldx]);
                    }
                    S.xt[t] = xv;
                }
            }
            __syncwarp();

            // COO entries: each adds val * x[col] into its row (the
            // reference's per-entry accumulate_output, cb-spmv-dcu.hpp:
            // 423-426), here into the lane's private accumulator.
            for (int c0 = 0; c0 < E; c0 += 32 * kChunk) {
                uint32_t w[kChunk];
                T v[kChunk], xv[kChunk];
#pragma unroll
                for (int u = 0; u < kChunk; ++u) {
                    const int e = c0 + u * 32 + lane;
                    w[u] = 0;
                    v[u] = T(0);
                    if (e < E) {
                        w[u] = __ldg(&cidx[e]);
                        v[u] = unit ? T(1) : __ldg(&cval[e]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kChunk; ++u) {
                    const int e = c0 + u * 32 + lane;
                    xv[u] = e < E ? ldg(&x[(int64_t)(w[u] & kColMask) * ldx]) : T(0);
                }
#pragma unroll
                for (int u = 0; u < kChunk; ++u) {
                    const int e = c0 + u * 32 + lane;
                    if (e < E) myacc[(w[u] >> 27) * 32] += v[u] * xv[u];
                }
            }

            add_csr_dense<T, BS>(base, bd, nxt, S.xt, myacc, unit, lane);
            __syncwarp();  // xt is rewritten by the next tile
            if (tile + 1 < t1) {
                ta = na;
                tb = nb4;
            }
        }
        const T s = reduce_rows<T, BS>(S.acc, lane);
        __syncwarp();

        // output: the unit holds the whole block row -> y; else the unit's
        // sums go to the slot of its first tile, and the last unit to arrive
        // adds the row's units (starting at its first tile, then every
        // unit_tiles tiles) in order
        const int64_t row0 = (int64_t)ta.y * BS;
        const int64_t grow = row0 + lane;
        const int64_t ntl = t1 - t0;
        if (tb.y == 0xffffffffu || ntl == (int64_t)tb.w) {
            if (lane < BS && grow < m) y[grow * ldy] = s;
        } else {
            const int64_t first = t1 - 1 - (int64_t)(tb.y - tb.z);
            if (lane < BS) partials[(size_t)(tb.z + (t0 - first)) * BS + lane] = s;
            __threadfence();
            __syncwarp();
            int last = 0;
            if (lane == 0) {
                const int old = atomicAdd(&counters[ta.y], (int)ntl);
                last = old + (int)ntl == (int)tb.w;
            }
            last = __shfl_sync(kFull, last, 0);
            if (last) {
                __threadfence();
                if (lane < BS) {
                    T tot = T(0);
                    for (uint32_t t = 0; t < tb.w; t += (uint32_t)unit_tiles)
                        tot += __ldcg(&partials[(size_t)(tb.z + t) * BS + lane]);
                    if (grow < m) y[grow * ldy] = tot;
                }
                if (lane == 0) atomicExch(&counters[ta.y], 0);
            }
        }
        cur = next;
    }
    // this warp has made its last (failing) grab: count it out; the last warp
    // out resets the scheduler for the next launch
    if (lane == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(&sched[1], 1u);
        if (done == gridDim.x * kWarps - 1) {
            atomicExch(&sched[0], 0u);
            atomicExch(&sched[1], 0u);
        }
    }
}

// ============================================================================
// Streaming tile kernel (TMA-staged), for matrices whose entries are mostly
// in COO blocks (e.g. gathered power-law matrices).
//   * each warp double-buffers the COO sections of its tiles in shared memory
//     with cp.async.bulk (bulk async copies completing on an mbarrier; no
//     multicast), so the HBM stream runs a tile ahead of the compute;
//   * each warp owns a contiguous, cost-balanced range of tiles computed on
//     the host for the launch's grid (no shared counter: same-address atomics
//     on one counter cannot keep up with ~10^5 tiles per launch);
//   * a tile's COO entries are stored sorted by (row, column) and taken 32 at
//     a time, one per lane, so the rows of a step never decrease across the
//     lanes: the products of one row are a run of lanes, summed by a
//     segmented shuffle scan, and the run's last lane adds the sum into the
//     warp's single accumulator of that row (bs values in shared memory);
//   * consecutive tiles of one block row in a warp's range keep adding into
//     the same accumulators; only a block row that crosses a warp boundary
//     leaves one partial sum per warp, and the last of those warps to arrive
//     on the row's counter adds them in tile order (no tile waits on another).
// Every mbarrier wait is bounded (`limit` polls); on give-up the error word
// is set and the warp stops, after waiting (kWaitLimit polls at most) for
// its own copies in flight.  The per-block-row arrival counters return to
// zero by the end of every launch that completes.
// ============================================================================
using dev::bulk_g2s;
using dev::fence_mbar_init;
using dev::fence_proxy_async;
using dev::kWaitLimit;
using dev::mbar_arrive;
using dev::mbar_arrive_tx;
using dev::mbar_init;
using dev::mbar_wait;
using dev::policy_evict_first;
using dev::slice_sums;
constexpr int kStreamWarps = 4;  // warps per CTA
constexpr int kStreamSteps = 8;  // 32-entry steps: tiles hold <= 256 COO entries

// Per-warp shared memory: [acc | xt | mbar[2] | buf[2]].  acc: the warp's bs
// row accumulators; xt: x columns of a tile's CSR/DENSE blocks (only when the
// layout has such blocks, has_x); buf: one tile's COO section (`cap` bytes:
// indices, then values).
template <typename T, int BS>
struct StreamLayout {
    static constexpr uint32_t acc_bytes = a16(BS * sizeof(T));
    static constexpr uint32_t xt_bytes = max_xt(BS) * BS * sizeof(T);
    __host__ __device__ static uint32_t head(int has_x) {
        return acc_bytes + (has_x ? xt_bytes : 0u) + 16u;
    }
    __host__ __device__ static uint32_t bytes(uint32_t cap, int has_x) {
        return a16(head(has_x)) + 2 * cap;
    }
};

// CSR and DENSE blocks of a tile (read from global memory, their x columns
// staged in xts), added into the warp's row accumulators.  32 / bs lanes per
// row (the reference's LANES_PER_ROW, macros.h:84, re-derived for 32-lane
// warps): a CSR row's entries are split over them, a DENSE row's columns in
// halves (bs = 16); the lanes of a row meet by a shuffle and the first adds.
template <typename T, int BS>
__device__ __forceinline__ void stream_blocks(const uint4 ta, T *acc, T *xts,
                                              const uint4 *__restrict__ blocks,
                                              const uint8_t *__restrict__ payload,
                                              const int32_t *__restrict__ block_cols,
                                              int gather, int unit, const T *__restrict__ x,
                                              int lane) {
    const int ncoo = (ta.z >> 8) & 0xff;
    const int nxtb = (ta.z >> 16) & 0xff;
    const uint4 bd =
        lane < nxtb ? __ldg(&blocks[ta.x + ncoo + lane]) : make_uint4(0, 0, 0, 0);
    for (int t0 = 0; t0 < nxtb * BS; t0 += 32) {
        const int t = t0 + lane;
        const int jb = min(t / BS, nxtb - 1);
        const uint32_t xb = __shfl_sync(kFull, bd.z, jb);
        const uint32_t mb = __shfl_sync(kFull, bd.y, jb);
        const int c = t % BS;
        if (t < nxtb * BS) {
            T xv = T(0);
            if (c < (int)((mb >> 14) & 63)) {
                const int64_t col = gather ? (int64_t)__ldg(&block_cols[xb + c])
                                           : (int64_t)(xb + c);
                xv = ldg(&x[col]);
            }
            xts[t] = xv;
        }
    }
    __syncwarp();
    constexpr int L = 32 / BS;  // lanes per row
    const int row = lane / L, sub = lane % L;
    const uint8_t *gbase = payload + (size_t)ta.w * 16;
    for (int jb = 0; jb < nxtb; ++jb) {
        const uint32_t off = __shfl_sync(kFull, bd.x, jb);
        const uint32_t mb = __shfl_sync(kFull, bd.y, jb);
        const int k = (mb >> 3) & 2047;
        const uint8_t *pb = gbase + off;
        const T *xt = &xts[jb * BS];
        T sum = T(0);
        if ((mb & 3) == 1) {
            using IdxT = typename std::conditional<BS == 16, uint8_t, uint16_t>::type;
            const IdxT *rp = reinterpret_cast<const IdxT *>(pb);
            const IdxT *ci = rp + BS + 1;
            const T *vv = reinterpret_cast<const T *>(
                pb + a16((uint32_t)((BS + 1 + k) * sizeof(IdxT))));
            const int kb = __ldg(&rp[row]), ke = __ldg(&rp[row + 1]);
            for (int q = kb + sub; q < ke; q += L)
                sum += (unit ? T(1) : __ldg(&vv[q])) * xt[__ldg(&ci[q])];
        } else {
            constexpr int W = BS / L;  // columns per lane
#pragma unroll 8
            for (int c = 0; c < W; ++c)
                sum += dense_at<T, BS>(pb, unit, row, sub * W + c) * xt[sub * W + c];
        }
        if (L == 2) sum += __shfl_xor_sync(kFull, sum, 1);
        if (sub == 0) acc[row] += sum;
    }
    __syncwarp();  // xts is rewritten by the next tile
}

// Ends a run of consecutive tiles of one block row in this warp (the last
// tile `tg`, global index; `runlen` tiles): reads and clears the warp's row
// accumulators and stores the rows.  A run that holds the whole block row
// stores y.  Otherwise the row crosses a warp boundary: the run's sum goes to
// the slot of its first tile, and the last run to arrive on the row's counter
// adds the row's run sums in tile order and stores y.  Runs start at the
// row's first tile and at every warp boundary inside the row (wpart), so the
// order does not depend on which warp arrives last.
template <typename T, int BS>
__device__ __forceinline__ void store_run(const uint4 ta, const uint4 tb, int64_t tg,
                                          int64_t runlen, T *acc, T *__restrict__ y,
                                          int64_t m, T *__restrict__ partials,
                                          int32_t *__restrict__ counters,
                                          const uint32_t *__restrict__ wpart, int64_t gw,
                                          int lane) {
    __syncwarp();
    T sum = T(0);
    if (lane < BS) {
        sum = acc[lane];
        acc[lane] = T(0);
    }
    __syncwarp();
    const int64_t grow = (int64_t)ta.y * BS + lane;
    if (tb.y == 0xffffffffu || runlen == (int64_t)tb.w) {
        if (lane < BS && grow < m) y[grow] = sum;
        return;
    }
    const int64_t first = tg - (int64_t)(tb.y - tb.z);  // the row's first tile
    const int64_t run0 = tg - runlen + 1;
    if (lane < BS) partials[(size_t)(tb.z + (run0 - first)) * BS + lane] = sum;
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane == 0) {
        const int old = atomicAdd(&counters[ta.y], (int)runlen);
        last = old + (int)runlen == (int)tb.w;
    }
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    // warp k holds tiles [wpart[k], wpart[k+1]); find the warp holding `first`
    int64_t k = gw;
    while (k > 0 && (int64_t)__ldg(&wpart[k]) > first) --k;
    const int64_t end = first + (int64_t)tb.w;
    T tot = T(0);
    if (lane < BS) tot = __ldcg(&partials[(size_t)tb.z * BS + lane]);
    int64_t prev = first;
    for (int64_t b = __ldg(&wpart[k + 1]); b < end; b = __ldg(&wpart[++k + 1])) {
        if (b > prev) {
            if (lane < BS) tot += __ldcg(&partials[(size_t)(tb.z + (b - first)) * BS + lane]);
            prev = b;
        }
    }
    if (lane < BS && grow < m) y[grow] = tot;
    if (lane == 0) atomicExch(&counters[ta.y], 0);
}

// Warp w processes its tiles i = 0, 1, ... of wpart[w] .. wpart[w+1]: it
// waits for tile i's staged COO section, reads the section's indices and
// issues all of its x gathers (up to 8 per lane), adds the steps up as the
// gathers return (values read from the staged section), handles the tile's
// CSR/DENSE blocks, and then starts the bulk copy of tile i+2 into the buffer
// it has just finished with.  Tile i lives in buffer i % 2.  The descriptors
// of tiles i .. i+3 are held one word per lane (lanes 8s .. 8s+7 hold the
// tile in slot s = index % 4) and read by shuffles.
template <typename T, int BS>
__global__ void __launch_bounds__(kStreamWarps * 32, 8)
    cb_spmv_stream_kernel(const uint4 *__restrict__ tiles, int64_t ntiles,
                          const uint4 *__restrict__ blocks,
                          const uint8_t *__restrict__ payload,
                          const int32_t *__restrict__ block_cols, int gather,
                          const T *__restrict__ x, T *__restrict__ y, int64_t m,
                          T *__restrict__ partials, int32_t *__restrict__ counters,
                          uint32_t *__restrict__ err, const uint32_t *__restrict__ wpart,
                          uint32_t cap, int has_x, int unit, uint32_t limit) {
    using SL = StreamLayout<T, BS>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char *wbase = smem_raw + (size_t)wib * SL::bytes(cap, has_x);
    T *acc = reinterpret_cast<T *>(wbase);
    T *xts = reinterpret_cast<T *>(wbase + SL::acc_bytes);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(wbase + SL::head(has_x) - 16);
    unsigned char *const buf0 = wbase + a16(SL::head(has_x));  // buffer b at buf0 + b * cap
    constexpr uint32_t vsz = sizeof(T);

    if (lane < BS) acc[lane] = T(0);
    if (lane == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    __syncwarp();

    const int64_t gw = (int64_t)blockIdx.x * kStreamWarps + wib;
    const int64_t t0 = __ldg(&wpart[gw]);
    const int64_t nt = min((int64_t)__ldg(&wpart[gw + 1]), ntiles) - t0;  // my tiles
    if (nt <= 0) return;
    const uint32_t *tw = reinterpret_cast<const uint32_t *>(tiles) + 8 * t0;
    uint32_t ring = 0;
    auto fetch = [&](int64_t k) {  // descriptor of tile k into slot k % 4
        if (k < nt && (lane >> 3) == (int)(k & 3)) ring = __ldg(&tw[8 * k + (lane & 7)]);
    };
    auto field = [&](int64_t k, int f) -> uint32_t {
        return __shfl_sync(kFull, ring, (int)((k & 3) << 3) | f);
    };
    auto stage = [&](int64_t k, int bi) {  // tile k's COO section into buffer bi
        const uint32_t E = field(k, 4), p16 = field(k, 3);
        if (lane == 0) {
            const uint32_t bytes = a16(4u * E) + (unit ? 0u : a16(vsz * E));
            if (bytes == 0) {
                mbar_arrive(&mbar[bi]);
            } else {
                fence_proxy_async();  // the buffer's previous tile was read
                mbar_arrive_tx(&mbar[bi], bytes);
                bulk_g2s(buf0 + bi * cap, payload + (size_t)p16 * 16, bytes, &mbar[bi],
                         policy_evict_first());
            }
        }
    };
    uint32_t phase = 0u;     // bit b: parity to wait for on mbar[b]
    uint32_t inflight = 0u;  // bit b: a copy into buffer b is outstanding

    fetch(0);
    fetch(1);
    fetch(2);
    fetch(3);
    stage(0, 0);
    inflight |= 1u;
    if (nt > 1) {
        stage(1, 1);
        inflight |= 2u;
    }
    int64_t runlen = 0;  // tiles of the current block row added so far
    for (int64_t i = 0; i < nt; ++i) {
        const int bi = (int)(i & 1);
        // on give-up the copy into buffer bi may still be landing: leave it
        // marked in flight (same parity) for the drain below
        if (!mbar_wait(&mbar[bi], (phase >> bi) & 1u, err, limit)) break;
        phase ^= 1u << bi;
        inflight &= ~(1u << bi);
        const unsigned char *buf = buf0 + bi * cap;
        const int E = (int)field(i, 4);
        const uint32_t *sidx = reinterpret_cast<const uint32_t *>(buf);
        const T *sval = reinterpret_cast<const T *>(buf + a16(4u * E));
        uint32_t w[kStreamSteps];
        T xv[kStreamSteps];
#pragma unroll
        for (int j = 0; j < kStreamSteps; ++j) {
            const int pos = 32 * j + lane;
            w[j] = pos < E ? sidx[pos] : 0u;
        }
#pragma unroll
        for (int j = 0; j < kStreamSteps; ++j) {
            const int pos = 32 * j + lane;
            xv[j] = pos < E ? ldg(&x[w[j] & kColMask]) : T(0);
        }
        // COO entries: each adds val * x[col] into its row (the reference's
        // per-entry accumulate_output, cb-spmv-dcu.hpp:423-426), here summed
        // along the lane's slice first, then across lanes (slice_sums)
        slice_sums<T, BS, kStreamSteps>(acc, w, xv, sval, unit, E, lane);
        const uint4 ta = make_uint4(field(i, 0), field(i, 1), field(i, 2), field(i, 3));
        if ((ta.z >> 16) & 0xff)
            stream_blocks<T, BS>(ta, acc, xts, blocks, payload, block_cols, gather, unit, x,
                                 lane);
        __syncwarp();
        if (i + 2 < nt) {
            stage(i + 2, bi);
            inflight |= 1u << bi;
        }
        ++runlen;
        if (i + 1 >= nt || field(i + 1, 1) != ta.y) {  // the row's run in this warp ends here
            const uint4 tb = make_uint4(E, field(i, 5), field(i, 6), field(i, 7));
            store_run<T, BS>(ta, tb, t0 + i, runlen, acc, y, m, partials, counters, wpart, gw,
                             lane);
            runlen = 0;
        }
        fetch(i + 4);
    }
    // never leave with a bulk copy still writing this warp's buffers
    for (int q = 0; q < 2; ++q)
        if ((inflight >> q) & 1u) mbar_wait(&mbar[q], (phase >> q) & 1u, err, kWaitLimit);
    __syncwarp();
}

// Pattern reuse: LP lanes per column pattern (a power of two), G = 32 / LP
// patterns per warp at a time, grid-strided.  The lanes of a pattern sum x
// over its columns (two loads in flight per lane), meet by shuffles, and
// write the sum to every output row of the pattern.  Unit values only: the
// reference's pattern schedules (cb-spmv-dcu.hpp:626-674) read no values.
template <typename T, int LP>
__global__ void __launch_bounds__(256)
    cb_pattern_kernel(const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                      const int32_t *__restrict__ optr, const int32_t *__restrict__ orow,
                      int64_t npat, const T *__restrict__ x, T *__restrict__ y) {
    constexpr int G = 32 / LP;
    const int lane = threadIdx.x & 31, sub = lane % LP, g = lane / LP;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * G; base < npat; base += warps * G) {  // warp-uniform
        const int64_t p = base + g;
        T s0 = T(0), s1 = T(0);
        if (p < npat) {
            const int c1 = __ldg(&ptr[p + 1]);
            int i = __ldg(&ptr[p]) + sub;
            for (; i + LP < c1; i += 2 * LP) {
                s0 += ldg(&x[__ldg(&col[i])]);
                s1 += ldg(&x[__ldg(&col[i + LP])]);
            }
            if (i < c1) s0 += ldg(&x[__ldg(&col[i])]);
        }
        T s = s0 + s1;
#pragma unroll
        for (int o = LP / 2; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
        if (p < npat) {
            const int o1 = __ldg(&optr[p + 1]);
            for (int i = __ldg(&optr[p]) + sub; i < o1; i += LP) y[__ldg(&orow[i])] = s;
        }
    }
}

template <typename T>
__global__ void cb_set_values_kernel(int64_t nvals, const int64_t *__restrict__ ptr,
                                     const int32_t *__restrict__ src,
                                     const uint64_t *__restrict__ off,
                                     const T *__restrict__ in,
                                     uint8_t *__restrict__ payload) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvals) return;
    T s = T(0);
    for (int64_t z = ptr[v]; z < ptr[v + 1]; ++z) s += in[src[z]];
    *reinterpret_cast<T *>(payload + off[v]) = s;
}

// LP lanes per value slot (a power of two): lane `sub` of a slot takes the
// VEC-wide pieces sub, sub + LP, ... of the nrhs right-hand sides (one 16-byte
// vector load per piece when both rows are aligned to it, VEC = 1 otherwise),
// and the LP partial sums meet by shuffles.  With LP * VEC covering a 32-byte
// row, one warp instruction reads whole sectors of g and x.  Each thread
// carries U slots (a block step covers U runs of 256 / LP consecutive slots)
// so that U times as many g and x rows are in flight, and the grid holds only
// as many blocks as are resident at once, striding over the slots: the kernel
// is bound by the latency of its gathers and, with one short block per few
// slots, by block launches.
template <typename T, int VEC, int LP, int U>
__global__ void __launch_bounds__(256)
    cb_grad_vals_kernel(int64_t nvals, const int32_t *__restrict__ vrow,
                        const int32_t *__restrict__ vcol, const T *__restrict__ g,
                        int64_t ldg, const T *__restrict__ x, int64_t ldx, int nrhs,
                        T *__restrict__ out) {
    constexpr int VPB = 256 / LP;  // slots per block and step
    const int sub = (int)threadIdx.x % LP;
    for (int64_t step = blockIdx.x; step * VPB * U < nvals; step += gridDim.x) {
        const int64_t v0 = step * VPB * U + threadIdx.x / LP;
        int32_t r[U], c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t v = v0 + (int64_t)u * VPB;
            r[u] = v < nvals ? __ldg(&vrow[v]) : -1;
            c[u] = v < nvals ? __ldg(&vcol[v]) : -1;
            if (c[u] < 0) r[u] = -1;  // dense padding: gradient 0
        }
        T s[U];
#pragma unroll
        for (int u = 0; u < U; ++u) s[u] = T(0);
        for (int j = sub * VEC; j < nrhs; j += LP * VEC) {
            T a[U][VEC], b[U][VEC];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const T *gr = g + (int64_t)max(r[u], 0) * ldg + j;
                const T *xr = x + (int64_t)max(c[u], 0) * ldx + j;
                if (r[u] < 0) {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) a[u][q] = b[u][q] = T(0);
                } else if constexpr (VEC == 1) {
                    a[u][0] = __ldg(gr);
                    b[u][0] = __ldg(xr);
                } else if constexpr (sizeof(T) == 4) {
                    const float4 fa = __ldg(reinterpret_cast<const float4 *>(gr));
                    const float4 fb = __ldg(reinterpret_cast<const float4 *>(xr));
                    a[u][0] = fa.x, a[u][1] = fa.y, a[u][2] = fa.z, a[u][3] = fa.w;
                    b[u][0] = fb.x, b[u][1] = fb.y, b[u][2] = fb.z, b[u][3] = fb.w;
                } else {
                    const double2 da = __ldg(reinterpret_cast<const double2 *>(gr));
                    const double2 db = __ldg(reinterpret_cast<const double2 *>(xr));
                    a[u][0] = da.x, a[u][1] = da.y;
                    b[u][0] = db.x, b[u][1] = db.y;
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < VEC; ++q) s[u] = fma(a[u][q], b[u][q], s[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int o = LP / 2; o > 0; o >>= 1) s[u] += __shfl_xor_sync(kFull, s[u], o);
            const int64_t v = v0 + (int64_t)u * VPB;
            if (sub == 0 && v < nvals) out[v] = s[u];
        }
    }
}

template <typename T, int BS, int CH>
cudaError_t launch_chunk(const DevLayout &d, const void *x, void *y, int nrhs,
                         int64_t ldx, int64_t ldy, cudaStream_t stream) {
    const size_t smem = sizeof(WarpSmem<T, BS>) * kWarps;
    const void *fn = reinterpret_cast<const void *>(cb_spmv_tile_kernel<T, BS, CH>);
    cudaError_t e = dev_enable_smem(fn, smem);
    if (e != cudaSuccess) return e;
    if (nrhs != 1 || !d.dunit) return cudaErrorInvalidValue;
    int64_t grid = (d.ndunits + kWarps - 1) / kWarps;
    grid = std::min<int64_t>(grid, (int64_t)dev_sms() * dev_resident_l1(fn, kWarps * 32, smem));
    if (grid == 0) return cudaSuccess;
    cb_spmv_tile_kernel<T, BS, CH><<<(unsigned)grid, kWarps * 32, smem, stream>>>(
        static_cast<const uint4 *>(d.tiles), static_cast<const uint4 *>(d.blocks), d.payload,
        d.block_cols, d.gather, static_cast<const T *>(x), static_cast<T *>(y), d.m, ldx, ldy,
        static_cast<T *>(d.partials), d.counters, d.sched, d.dunit, d.ndunits, kDirectUnitTiles,
        d.unit);
    note_launch();
    return cudaGetLastError();
}

// COO entries per lane in flight in the direct kernel: 4 for both value
// types (measured fastest on CSR-heavy matrices; 6 and 8 also spill in
// FP64); CBSPMV_CHUNK=4|6|8 overrides it for tuning.
int chunk_choice() {
    static const int forced = [] {
        const char *e = std::getenv("CBSPMV_CHUNK");
        return e ? std::atoi(e) : 0;
    }();
    if (forced == 4 || forced == 6 || forced == 8) return forced;
    return 4;
}

template <typename T, int BS>
struct StreamConfig {
    uint32_t cap = 0;
    size_t smem = 0;
    int64_t warps = 0;  // warps one launch can keep resident
};

template <typename T, int BS>
cudaError_t stream_config(const DevLayout &d, StreamConfig<T, BS> &c) {
    using SL = StreamLayout<T, BS>;
    const uint32_t E = (uint32_t)d.max_entries;
    c.cap = std::max<uint32_t>(16, a16(4u * E) + (d.unit ? 0u : a16((uint32_t)sizeof(T) * E)));
    c.smem = (size_t)SL::bytes(c.cap, d.has_x) * kStreamWarps;
    const void *fn = reinterpret_cast<const void *>(cb_spmv_stream_kernel<T, BS>);
    cudaError_t e = dev_enable_smem(fn, c.smem);
    if (e != cudaSuccess) return e;
    const int resident = dev_resident_l1(fn, kStreamWarps * 32, c.smem);
    const int64_t need = (d.ntiles + kStreamWarps - 1) / kStreamWarps * kStreamWarps;
    c.warps = std::max<int64_t>(
        kStreamWarps, std::min<int64_t>((int64_t)dev_sms() * resident * kStreamWarps, need));
    return cudaSuccess;
}

template <typename T, int BS>
cudaError_t launch_stream(const DevLayout &d, const void *x, void *y, cudaStream_t stream) {
    StreamConfig<T, BS> c;
    cudaError_t e = stream_config(d, c);
    if (e != cudaSuccess) return e;
    if (d.ntiles == 0) return cudaSuccess;
    if (!d.wpart || d.nwarps % kStreamWarps || d.max_entries > 32 * kStreamSteps || !d.err)
        return cudaErrorInvalidValue;
    cb_spmv_stream_kernel<T, BS>
        <<<(unsigned)(d.nwarps / kStreamWarps), kStreamWarps * 32, c.smem, stream>>>(
            static_cast<const uint4 *>(d.tiles), d.ntiles,
            static_cast<const uint4 *>(d.blocks), d.payload, d.block_cols, d.gather,
            static_cast<const T *>(x), static_cast<T *>(y), d.m,
            static_cast<T *>(d.partials), d.counters, d.err, d.wpart, c.cap, d.has_x, d.unit,
            wait_polls());
    note_launch();
    return cudaGetLastError();
}

// Streaming kernel for COO-dominant matrices, the direct kernel otherwise
// (or as chosen by the plan's kernel option; 3 = the staged kernel).
// (single right-hand side; several go through the direct kernel)
bool use_stream(const DevLayout &d) {
    if (d.max_entries > 32 * kStreamSteps) return false;
    if (d.kernel == 1) return true;
    if (d.kernel >= 2) return false;
    if (d.small_direct) return false;
    return d.coo_share >= 0.5;
}

template <typename T, int LP>
cudaError_t launch_pattern_t(const DevLayout &d, const void *x, void *y, cudaStream_t st) {
    const void *fn = reinterpret_cast<const void *>(cb_pattern_kernel<T, LP>);
    const int64_t want = (d.npat * LP + 255) / 256;
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>(want, (int64_t)dev_sms() * dev_resident(fn, 256, 0)));
    cb_pattern_kernel<T, LP><<<(unsigned)grid, 256, 0, st>>>(
        d.pat_ptr, d.pat_col, d.pat_out_ptr, d.pat_out_rows, d.npat,
        static_cast<const T *>(x), static_cast<T *>(y));
    note_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_pattern_v(const DevLayout &d, const void *x, void *y, cudaStream_t st) {
    const double avg = d.npat ? (double)d.pat_cols / (double)d.npat : 0.0;
    if (avg <= 6) return launch_pattern_t<T, 4>(d, x, y, st);
    if (avg <= 12) return launch_pattern_t<T, 8>(d, x, y, st);
    if (avg <= 24) return launch_pattern_t<T, 16>(d, x, y, st);
    return launch_pattern_t<T, 32>(d, x, y, st);
}

// the pattern schedule: chosen (kernel 4) or automatic by the reference's
// rule, patterns fewer than half the rows (cb-spmv-dcu.hpp:1431-1433)
bool use_pattern(const DevLayout &d) {
    if (!d.npat || !d.unit) return false;
    return d.kernel == 4 || (d.kernel == 0 && d.pat_auto);
}

template <typename T, int BS>
cudaError_t launch_tiles(const DevLayout &d, const void *x, void *y, int nrhs,
                         int64_t ldx, int64_t ldy, cudaStream_t stream) {
    if (nrhs == 1 && ldx == 1 && ldy == 1 && use_pattern(d))
        return launch_pattern_v<T>(d, x, y, stream);
    // the row-segment stream: when chosen, and the automatic choice for
    // all-COO layouts except the reference's small-direct case
    const bool one = nrhs == 1 && ldx == 1 && ldy == 1;
    // the balanced schedule: plans built with row_owned = 0 (the reference's
    // non-row-owned mode), one right-hand side
    if (one && d.bal.rows && (d.kernel == 6 || d.kernel == 0))
        return launch_balanced(d, x, y, stream);
    if (d.rs.chunks && (d.kernel == 5 || (d.kernel == 0 && !d.small_direct &&
                                          !use_pattern(d) && (!one || d.rs.auto1))))
        return one ? launch_rowseg(d, x, y, stream)
                   : launch_rowseg_mrhs(d, x, y, nrhs, ldx, ldy, stream);
    if (nrhs == 1 && ldx == 1 && ldy == 1 && use_stream(d))
        return launch_stream<T, BS>(d, x, y, stream);
    if (nrhs > 1 || d.kernel == 3 || d.kernel == 4)
        return launch_spmm(d, x, y, nrhs, ldx, ldy, stream);
    switch (chunk_choice()) {
        case 4: return launch_chunk<T, BS, 4>(d, x, y, nrhs, ldx, ldy, stream);
        case 6: return launch_chunk<T, BS, 6>(d, x, y, nrhs, ldx, ldy, stream);
        default: return launch_chunk<T, BS, 8>(d, x, y, nrhs, ldx, ldy, stream);
    }
}

}  // namespace

std::vector<uint32_t> direct_units(const uint32_t *tile8, int64_t ntiles) {
    std::vector<uint32_t> us;
    int64_t row_start = 0;
    for (int64_t t = 0; t < ntiles; ++t) {
        const uint32_t *d = tile8 + 8 * t;
        const bool first = d[5] == 0xffffffffu || d[5] == d[6];  // slot == first slot
        if (first) row_start = t;
        if ((t - row_start) % kDirectUnitTiles == 0) us.push_back((uint32_t)t);
    }
    us.push_back((uint32_t)ntiles);
    return us;
}

int64_t kernel_launches() { return g_kernel_launches.load(); }
void note_launch() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {
std::mutex g_facts_mu;
std::map<int, int> g_sms;                                    // device -> SMs
std::map<std::pair<int, const void *>, size_t> g_smem;       // (device, kernel) -> enabled
std::map<std::tuple<int, const void *, int, size_t>, int> g_resident;
std::map<std::pair<int, const void *>, int> g_carve;        // carveout set + 1
std::atomic<uint32_t> g_wait_polls{0};                       // 0: kWaitLimit

int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}
}  // namespace

int dev_sms() {
    const int d = current_device();
    std::lock_guard<std::mutex> lock(g_facts_mu);
    auto it = g_sms.find(d);
    if (it != g_sms.end()) return it->second;
    int s = 0;
    cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, d);
    return g_sms[d] = std::max(1, s);
}

cudaError_t dev_enable_smem(const void *fn, size_t smem) {
    const int d = current_device();
    std::lock_guard<std::mutex> lock(g_facts_mu);
    size_t &have = g_smem[{d, fn}];
    if (smem <= have) return cudaSuccess;
    const cudaError_t e =
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) have = smem;
    return e;
}

int dev_resident(const void *fn, int threads, size_t smem) {
    const int d = current_device();
    std::lock_guard<std::mutex> lock(g_facts_mu);
    auto key = std::make_tuple(d, fn, threads, smem);
    auto it = g_resident.find(key);
    if (it != g_resident.end()) return it->second;
    int r = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        r = 1;
    }
    return g_resident[key] = std::max(1, r);
}

int dev_resident_l1(const void *fn, int threads, size_t smem) {
    // the occupancy query counts the carveout preference a previous launch
    // set for a smaller footprint, so take the register and thread limit
    // alone and the shared-memory limit from the largest carveout
    int r = dev_resident(fn, threads, 0);
    const int d = current_device();
    int maxs = 0, reserved = 0;
    cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerMultiprocessor, d);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, d);
    if (maxs <= (int)kL1Keep) return r;
    const size_t per = smem + (size_t)reserved;
    const size_t cap = (size_t)maxs - kL1Keep;
    r = std::min<int>(r, (int)((size_t)maxs / per));  // what fits at all
    r = std::max(1, std::min<int>(r, (int)(cap / std::max<size_t>(per, 1))));
    const int pct = (int)std::min<size_t>(100, (r * per * 100 + maxs - 1) / (size_t)maxs);
    std::lock_guard<std::mutex> lock(g_facts_mu);
    int &have = g_carve[{d, fn}];
    if (have != pct + 1 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct) ==
            cudaSuccess)
        have = pct + 1;
    cudaGetLastError();
    return r;
}

uint32_t wait_polls() {
    const uint32_t p = g_wait_polls.load(std::memory_order_relaxed);
    return p ? p - 1 : dev::kWaitLimit;
}

void set_wait_polls(int64_t polls) {
    g_wait_polls.store(polls < 0 ? 0u : (uint32_t)std::min<int64_t>(polls, dev::kWaitLimit) + 1u,
                       std::memory_order_relaxed);
}

size_t spmv_smem_bytes(int bs, int f32) {
    if (bs == 16)
        return kWarps * (f32 ? sizeof(WarpSmem<float, 16>) : sizeof(WarpSmem<double, 16>));
    return kWarps * (f32 ? sizeof(WarpSmem<float, 32>) : sizeof(WarpSmem<double, 32>));
}

template <typename T, int BS>
int64_t stream_warps_t(const DevLayout &d) {
    if (!use_stream(d)) return 0;
    StreamConfig<T, BS> c;
    if (stream_config(d, c) != cudaSuccess) return 0;
    return c.warps;
}

int64_t stream_warps(const DevLayout &d) {
    if (d.bs == 16) return d.f32 ? stream_warps_t<float, 16>(d) : stream_warps_t<double, 16>(d);
    return d.f32 ? stream_warps_t<float, 32>(d) : stream_warps_t<double, 32>(d);
}

cudaError_t launch_pattern(const DevLayout &d, const void *x, void *y, cudaStream_t stream) {
    if (!d.npat) return cudaErrorInvalidValue;
    return d.f32 ? launch_pattern_v<float>(d, x, y, stream)
                 : launch_pattern_v<double>(d, x, y, stream);
}

cudaError_t launch_spmv(const DevLayout &d, const void *x, void *y, int nrhs,
                        int64_t ldx, int64_t ldy, cudaStream_t stream) {
    if (d.bs == 16)
        return d.f32 ? launch_tiles<float, 16>(d, x, y, nrhs, ldx, ldy, stream)
                     : launch_tiles<double, 16>(d, x, y, nrhs, ldx, ldy, stream);
    return d.f32 ? launch_tiles<float, 32>(d, x, y, nrhs, ldx, ldy, stream)
                 : launch_tiles<double, 32>(d, x, y, nrhs, ldx, ldy, stream);
}

// ---- fixed scratch, for callers that may not allocate device memory -------
// A file-scope device array replaces the plan's own scratch (scheduler words,
// per-block-row arrival counters, split-row partial sums).  Every GPU that
// loads this library holds it until the process exits.
static __device__ __align__(256) unsigned char g_fixed_scratch[kFixedScratchBytes];

namespace {
// Device address of g_fixed_scratch on the current device, looked up once per
// device (the host-side symbol is not a device address).
cudaError_t fixed_scratch_ptr(void **ptr) {
    static std::mutex mu;
    static void *addr[64] = {};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_fixed_scratch);
        if (e != cudaSuccess) return e;
        addr[dev] = p;
    }
    *ptr = addr[dev];
    return cudaSuccess;
}
}  // namespace

size_t fixed_scratch_need(int64_t gb_m, int64_t slots, int nrhs, int bs, int f32) {
    const size_t words = 16 + 4 * (size_t)gb_m;  // 4 scheduler words, counters
    const size_t head = (words + 255) & ~size_t(255);
    return head + (size_t)slots * nrhs * bs * (f32 ? 4 : 8);
}

cudaError_t launch_spmv_fixed_scratch(const DevLayout &d, int64_t gb_m, int64_t slots,
                                      const void *x, void *y, int nrhs, int64_t ldx,
                                      int64_t ldy, cudaStream_t stream) {
    if (fixed_scratch_need(gb_m, slots, nrhs, d.bs, d.f32) > kFixedScratchBytes)
        return cudaErrorInvalidValue;
    void *base = nullptr;
    cudaError_t e = fixed_scratch_ptr(&base);
    if (e != cudaSuccess) return e;
    unsigned char *b = static_cast<unsigned char *>(base);
    const size_t words = 16 + 4 * (size_t)gb_m;
    // the scheduler words and arrival counters must start at zero
    e = cudaMemsetAsync(b, 0, words, stream);
    if (e != cudaSuccess) return e;
    DevLayout f = d;
    f.sched = reinterpret_cast<uint32_t *>(b);
    f.counters = reinterpret_cast<int32_t *>(b + 16);
    f.partials = b + ((words + 255) & ~size_t(255));
    return launch_spmv(f, x, y, nrhs, ldx, ldy, stream);
}

cudaError_t launch_set_values(int f32, int64_t nvals, const int64_t *vsrc_ptr,
                              const int32_t *vsrc, const uint64_t *val_off,
                              const void *in, uint8_t *payload,
                              cudaStream_t stream) {
    if (nvals == 0) return cudaSuccess;
    const unsigned grid = (unsigned)((nvals + 255) / 256);
    if (f32)
        cb_set_values_kernel<float><<<grid, 256, 0, stream>>>(
            nvals, vsrc_ptr, vsrc, val_off, static_cast<const float *>(in), payload);
    else
        cb_set_values_kernel<double><<<grid, 256, 0, stream>>>(
            nvals, vsrc_ptr, vsrc, val_off, static_cast<const double *>(in), payload);
    note_launch();
    return cudaGetLastError();
}

template <typename T, int V>
void grad_vals_go(int lp, int64_t nvals, const int32_t *vrow, const int32_t *vcol,
                  const void *g, int64_t ldg, const void *x, int64_t ldx, int nrhs,
                  void *gvals, cudaStream_t st) {
    constexpr int U = 4;
    const T *gp = static_cast<const T *>(g), *xp = static_cast<const T *>(x);
    T *op = static_cast<T *>(gvals);
    const int li = lp == 1 ? 0 : lp == 2 ? 1 : lp == 4 ? 2 : 3;
    void (*const kerns[4])(int64_t, const int32_t *, const int32_t *, const T *, int64_t,
                           const T *, int64_t, int, T *) = {
        cb_grad_vals_kernel<T, V, 1, U>, cb_grad_vals_kernel<T, V, 2, U>,
        cb_grad_vals_kernel<T, V, 4, U>, cb_grad_vals_kernel<T, V, 8, U>};
    auto kern = kerns[li];
    const int resident = dev_resident(reinterpret_cast<const void *>(kern), 256, 0);
    const int64_t per_block = 256 / lp * U;
    const int64_t grid = std::min<int64_t>((nvals + per_block - 1) / per_block,
                                           (int64_t)dev_sms() * resident);
    kern<<<(unsigned)grid, 256, 0, st>>>(nvals, vrow, vcol, gp, ldg, xp, ldx, nrhs, op);
}

cudaError_t launch_grad_vals(int f32, int64_t nvals, const int32_t *vrow,
                             const int32_t *vcol, const void *g, int64_t ldg,
                             const void *x, int64_t ldx, int nrhs, void *gvals,
                             cudaStream_t stream) {
    if (nvals == 0) return cudaSuccess;
    const int vec = f32 ? 4 : 2;
    const bool vok = nrhs % vec == 0 && ldg % vec == 0 && ldx % vec == 0 &&
                     reinterpret_cast<uintptr_t>(g) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(x) % 16 == 0;
    const int pieces = vok ? nrhs / vec : nrhs;
    int lp = 1;  // lanes per value slot
    while (lp < pieces && lp < 8) lp *= 2;
    if (f32) {
        (vok ? grad_vals_go<float, 4> : grad_vals_go<float, 1>)(lp, nvals, vrow, vcol, g, ldg,
                                                                x, ldx, nrhs, gvals, stream);
    } else {
        (vok ? grad_vals_go<double, 2> : grad_vals_go<double, 1>)(lp, nvals, vrow, vcol, g, ldg,
                                                                  x, ldx, nrhs, gvals, stream);
    }
    note_launch();
    return cudaGetLastError();
}

}  // namespace cb
