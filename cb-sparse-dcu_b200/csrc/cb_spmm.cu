// sm_100a multi-right-hand-side CB-SpMV: Y = A X with X (n x nrhs) and
// Y (m x nrhs) row-major (leading dimensions ldx, ldy), over the same tile
// layout as the single-vector kernels (cb_kernels.cu).
//
// A warp splits its lanes into G = 32 / R entry groups of R lanes, R the next
// power of two >= nrhs (at most 32; more right-hand sides take several
// passes).  Lane (g, j) handles right-hand side j of entries g, g + G, ...:
// each stored entry is read once per pass and the R values of an x row arrive
// in one coalesced load, where a loop over right-hand sides would read the
// tile nrhs times.  Accumulators are the single-vector kernels' lane-private
// columns (row r of lane l at acc[r * 32 + l]), so an output (row r, rhs j) is
// the sum of the G copies acc[r * 32 + g * R + j].  CSR and DENSE blocks stage
// their bs x rows (R values each) in shared memory one block at a time.
//
// Split block rows: each tile leaves its partial sums for the pass's
// right-hand sides in its slot; the last tile to arrive on the row's counter
// (tiles x passes arrivals) adds all slots in tile order and stores Y.  No
// tile waits on another.
//
// Two drivers: cb_spmm_tile_kernel (one matrix, tiles taken from a global
// counter) and cb_batch_kernel (many matrices in one launch, host-balanced
// contiguous ranges of the concatenated tile list per warp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "cb_device.cuh"
#include "cb_kernels.hpp"

namespace cb {
namespace {

using dev::a16;
using dev::add_entries;
using dev::kColMask;
using dev::kFull;

constexpr int kSpmmWarps = 8;

template <typename T, int BS, int R>
struct SpmmSmem {
    T acc[BS * 32];
    T xt[BS * R];  // x rows of the current CSR/DENSE block, R values each
};

// One tile, right-hand sides j0 .. j0 + R - 1.  `passes` = passes per tile
// (counts the arrivals on split rows).
template <typename T, int BS, int R, int KC>
__device__ __forceinline__ void spmm_tile(const MatView &M, const uint4 ta, const uint4 tb,
                                          int j0, int passes, T *acc, T *xt, int lane) {
    constexpr int G = 32 / R;
    const int es = lane / R, jr = lane % R;
    const int j = j0 + jr;
    const bool jok = j < M.nrhs;
    const T *__restrict__ x = static_cast<const T *>(M.x);
    T *__restrict__ y = static_cast<T *>(M.y);
    T *myacc = &acc[lane];
    const int ncoo = (ta.z >> 8) & 0xff;
    const int nxt = (ta.z >> 16) & 0xff;
    const int E = (int)tb.x;
    const uint8_t *base = M.payload + (size_t)ta.w * 16;
    const uint32_t *cidx = reinterpret_cast<const uint32_t *>(base);
    const T *cval = reinterpret_cast<const T *>(base + a16(4u * E));

    // COO entries: KC per lane in flight, the R lanes of a group share one
    for (int c0 = 0; c0 < E; c0 += G * KC) {
        uint32_t w[KC];
        T v[KC], xv[KC];
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            const int e = c0 + u * G + es;
            w[u] = 0u;
            v[u] = T(0);
            if (e < E) {
                w[u] = __ldg(&cidx[e]);
                v[u] = __ldg(&cval[e]);
            }
        }
#pragma unroll
        for (int u = 0; u < KC; ++u) {
            const int e = c0 + u * G + es;
            xv[u] = (e < E && jok) ? __ldg(&x[(int64_t)(w[u] & kColMask) * M.ldx + j]) : T(0);
        }
        add_entries<T, KC>(myacc, w, v, xv, c0 + es, G, E);
    }

    // CSR and DENSE blocks, one at a time
    uint4 bd = make_uint4(0, 0, 0, 0);  // lane q: CSR/DENSE block q of the tile
    if (lane < nxt) bd = __ldg(&M.blocks[ta.x + ncoo + lane]);
    for (int jb = 0; jb < nxt; ++jb) {
        const uint32_t off = __shfl_sync(kFull, bd.x, jb);
        const uint32_t mb = __shfl_sync(kFull, bd.y, jb);
        const uint32_t xb = __shfl_sync(kFull, bd.z, jb);
        const int valid = (mb >> 14) & 63;
        __syncwarp();  // the previous block is done with xt
        for (int idx = lane; idx < BS * R; idx += 32) {  // idx % R == jr
            const int c = idx / R;
            T xvv = T(0);
            if (c < valid && jok) {
                const int64_t col = M.gather ? (int64_t)__ldg(&M.block_cols[xb + c])
                                             : (int64_t)(xb + c);
                xvv = __ldg(&x[col * M.ldx + j]);
            }
            xt[idx] = xvv;
        }
        __syncwarp();
        const uint8_t *pb = base + off;
        const int k = (mb >> 3) & 2047;
        if ((mb & 3) == 1) {  // CSR
            using IdxT = typename std::conditional<BS == 16, uint8_t, uint16_t>::type;
            const IdxT *rp = reinterpret_cast<const IdxT *>(pb);
            const IdxT *ci = rp + BS + 1;
            const T *vv = reinterpret_cast<const T *>(
                pb + a16((uint32_t)((BS + 1 + k) * sizeof(IdxT))));
            if (G >= BS) {  // G / BS lanes per row
                constexpr int L = G >= BS ? G / BS : 1;
                const int row = es / L, sub = es % L;
                const int kb = __ldg(&rp[row]), ke = __ldg(&rp[row + 1]);
                T sum = T(0);
                for (int q = kb + sub; q < ke; q += L) sum += __ldg(&vv[q]) * xt[__ldg(&ci[q]) * R + jr];
                myacc[row * 32] += sum;
            } else {  // rows es, es + G, ...
                for (int row = es; row < BS; row += G) {
                    const int kb = __ldg(&rp[row]), ke = __ldg(&rp[row + 1]);
                    T sum = T(0);
                    for (int q = kb; q < ke; ++q) sum += __ldg(&vv[q]) * xt[__ldg(&ci[q]) * R + jr];
                    myacc[row * 32] += sum;
                }
            }
        } else {  // DENSE, row-major bs x bs
            const T *vv = reinterpret_cast<const T *>(pb);
            if (G >= BS) {
                constexpr int L = G >= BS ? G / BS : 1;
                constexpr int W = BS / L;  // columns per lane
                const int row = es / L, c0 = (es % L) * W;
                T sum = T(0);
#pragma unroll 8
                for (int c = 0; c < W; ++c)
                    sum += __ldg(&vv[row * BS + c0 + c]) * xt[(c0 + c) * R + jr];
                myacc[row * 32] += sum;
            } else {
                for (int row = es; row < BS; row += G) {
                    T sum = T(0);
#pragma unroll 8
                    for (int c = 0; c < BS; ++c) sum += __ldg(&vv[row * BS + c]) * xt[c * R + jr];
                    myacc[row * 32] += sum;
                }
            }
        }
    }
    __syncwarp();

    // outputs (row r, rhs jj): lanes take o = lane + 32 q; copy g of the sum
    // is read in the rotated order (t + r) % G so one step hits distinct banks
    constexpr int NO = BS * R;
    const int64_t row0 = (int64_t)ta.y * BS;
    const bool split = tb.y != 0xffffffffu;
#pragma unroll
    for (int q = 0; q < (NO + 31) / 32; ++q) {
        const int o = lane + 32 * q;
        if (o < NO) {
            const int r = o / R, jj = o % R;
            T s = T(0);
#pragma unroll 8
            for (int t = 0; t < G; ++t) {
                T *p = &acc[r * 32 + ((t + r) % G) * R + jj];
                s += *p;
                *p = T(0);
            }
            const int jo = j0 + jj;
            if (jo < M.nrhs) {
                if (!split) {
                    if (row0 + r < M.m) y[(row0 + r) * M.ldy + jo] = s;
                } else {
                    static_cast<T *>(M.partials)[((size_t)tb.y * M.nrhs + jo) * BS + r] = s;
                }
            }
        }
    }
    if (!split) return;
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane == 0) {
        const int old = atomicAdd(&M.counters[ta.y], 1);
        last = old == (int)tb.w * passes - 1;
    }
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    const T *part = static_cast<const T *>(M.partials);
    for (int o = lane; o < BS * M.nrhs; o += 32) {
        const int r = o % BS, jj = o / BS;
        T tot = T(0);
        for (uint32_t t = 0; t < tb.w; ++t)
            tot += __ldcg(&part[((size_t)(tb.z + t) * M.nrhs + jj) * BS + r]);
        if (row0 + r < M.m) y[(row0 + r) * M.ldy + jj] = tot;
    }
    if (lane == 0) atomicExch(&M.counters[ta.y], 0);
}

template <typename T, int BS, int R, int KC>
__device__ __forceinline__ void spmm_tile_all(const MatView &M, int64_t tile, T *acc, T *xt,
                                              int lane) {
    const uint4 ta = __ldg(&M.tiles[2 * tile]);
    const uint4 tb = __ldg(&M.tiles[2 * tile + 1]);
    const int passes = (M.nrhs + R - 1) / R;
    for (int j0 = 0; j0 < M.nrhs; j0 += R)
        spmm_tile<T, BS, R, KC>(M, ta, tb, j0, passes, acc, xt, lane);
}

// One matrix: persistent warps take tiles from a global counter (sched[0]);
// the warp whose exit completes sched[1] == number of warps resets both.
template <typename T, int BS, int R, int KC>
__global__ void __launch_bounds__(kSpmmWarps * 32, 2)
    cb_spmm_tile_kernel(const MatView M, uint32_t *__restrict__ sched) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    SpmmSmem<T, BS, R> &S = reinterpret_cast<SpmmSmem<T, BS, R> *>(smem_raw)[threadIdx.x >> 5];
    for (int t = lane; t < BS * 32; t += 32) S.acc[t] = T(0);
    __syncwarp();
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&sched[0], 1u);
        const int64_t tile = (int64_t)__shfl_sync(kFull, t, 0);
        if (tile >= M.ntiles) break;
        spmm_tile_all<T, BS, R, KC>(M, tile, S.acc, S.xt, lane);
    }
    if (lane == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(&sched[1], 1u);
        if (done == gridDim.x * kSpmmWarps - 1) {
            atomicExch(&sched[0], 0u);
            atomicExch(&sched[1], 0u);
        }
    }
}

__host__ __device__ constexpr int kc_for(int R, int vsz) { return R == 1 ? (vsz == 8 ? 6 : 8) : (R == 2 ? 6 : 8); }

// Many matrices in one launch: warp w takes tiles [wpart[w], wpart[w+1]) of
// the batch's concatenated tile list; matrix k owns tiles [toff[k],
// toff[k+1]) and runs with its own lanes per entry (mats[k].lanes).
template <typename T, int BS>
__global__ void __launch_bounds__(kSpmmWarps * 32, 2)
    cb_batch_kernel(const MatView *__restrict__ mats, int nmats,
                    const int64_t *__restrict__ toff, const int64_t *__restrict__ wpart) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    SpmmSmem<T, BS, 32> &S = reinterpret_cast<SpmmSmem<T, BS, 32> *>(smem_raw)[threadIdx.x >> 5];
    for (int t = lane; t < BS * 32; t += 32) S.acc[t] = T(0);
    __syncwarp();
    const int64_t gw = (int64_t)blockIdx.x * kSpmmWarps + (threadIdx.x >> 5);
    const int64_t g0 = __ldg(&wpart[gw]), g1 = __ldg(&wpart[gw + 1]);
    if (g0 >= g1) return;
    int l = 0, h = nmats;  // the last matrix k with toff[k] <= g0
    while (h - l > 1) {
        const int mid = (l + h) >> 1;
        if (__ldg(&toff[mid]) <= g0) l = mid; else h = mid;
    }
    int k = l;
    MatView M = mats[k];
    int64_t lo = __ldg(&toff[k]), hi = __ldg(&toff[k + 1]);
    for (int64_t g = g0; g < g1; ++g) {
        while (g >= hi) {
            ++k;
            M = mats[k];
            lo = hi;
            hi = __ldg(&toff[k + 1]);
        }
        const int64_t t = g - lo;
        switch (M.lanes) {
            case 1: spmm_tile_all<T, BS, 1, kc_for(1, sizeof(T))>(M, t, S.acc, S.xt, lane); break;
            case 2: spmm_tile_all<T, BS, 2, kc_for(2, sizeof(T))>(M, t, S.acc, S.xt, lane); break;
            case 4: spmm_tile_all<T, BS, 4, kc_for(4, sizeof(T))>(M, t, S.acc, S.xt, lane); break;
            case 8: spmm_tile_all<T, BS, 8, kc_for(8, sizeof(T))>(M, t, S.acc, S.xt, lane); break;
            case 16: spmm_tile_all<T, BS, 16, kc_for(16, sizeof(T))>(M, t, S.acc, S.xt, lane); break;
            default: spmm_tile_all<T, BS, 32, kc_for(32, sizeof(T))>(M, t, S.acc, S.xt, lane); break;
        }
    }
}


template <typename T, int BS, int R>
cudaError_t spmm_launch_r(const MatView &M, uint32_t *sched, cudaStream_t stream) {
    constexpr int KC = kc_for(R, sizeof(T));
    const size_t smem = sizeof(SpmmSmem<T, BS, R>) * kSpmmWarps;
    static int resident = 0, sms = 0;
    if (!resident) {
        cudaError_t e = cudaFuncSetAttribute(cb_spmm_tile_kernel<T, BS, R, KC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        int devid = 0;
        cudaGetDevice(&devid);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devid);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, cb_spmm_tile_kernel<T, BS, R, KC>,
                                                      kSpmmWarps * 32, smem);
        if (resident < 1) resident = 1;
    }
    int64_t grid = (M.ntiles + kSpmmWarps - 1) / kSpmmWarps;
    grid = std::min<int64_t>(grid, (int64_t)sms * resident);
    if (grid <= 0) return cudaSuccess;
    cb_spmm_tile_kernel<T, BS, R, KC><<<(unsigned)grid, kSpmmWarps * 32, smem, stream>>>(M, sched);
    note_launch();
    return cudaGetLastError();
}

template <typename T, int BS>
size_t batch_smem() {
    return sizeof(SpmmSmem<T, BS, 32>) * kSpmmWarps;
}

template <typename T, int BS>
cudaError_t batch_configure() {
    static bool done = false;
    if (done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(cb_batch_kernel<T, BS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)batch_smem<T, BS>());
    if (e == cudaSuccess) done = true;
    return e;
}

template <typename T, int BS>
cudaError_t batch_launch_t(const MatView *mats, int nmats, const int64_t *toff,
                           const int64_t *wpart, int64_t nwarps, cudaStream_t stream) {
    cudaError_t e = batch_configure<T, BS>();
    if (e != cudaSuccess) return e;
    if (nwarps <= 0 || nwarps % kSpmmWarps) return cudaErrorInvalidValue;
    cb_batch_kernel<T, BS><<<(unsigned)(nwarps / kSpmmWarps), kSpmmWarps * 32,
                             batch_smem<T, BS>(), stream>>>(mats, nmats, toff, wpart);
    note_launch();
    return cudaGetLastError();
}

template <typename T, int BS>
int64_t batch_warps_t() {
    if (batch_configure<T, BS>() != cudaSuccess) return 0;
    int devid = 0, sms = 0, resident = 0;
    cudaGetDevice(&devid);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devid);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, cb_batch_kernel<T, BS>,
                                                  kSpmmWarps * 32, batch_smem<T, BS>());
    return (int64_t)std::max(1, resident) * sms * kSpmmWarps;
}

template <typename T, int BS, typename F>
auto by_r(int R, F f) {
    switch (R) {
        case 1: return f(std::integral_constant<int, 1>());
        case 2: return f(std::integral_constant<int, 2>());
        case 4: return f(std::integral_constant<int, 4>());
        case 8: return f(std::integral_constant<int, 8>());
        case 16: return f(std::integral_constant<int, 16>());
        default: return f(std::integral_constant<int, 32>());
    }
}

template <typename F>
auto by_type(int bs, int f32, F f) {
    if (bs == 16)
        return f32 ? f(float(), std::integral_constant<int, 16>())
                   : f(double(), std::integral_constant<int, 16>());
    return f32 ? f(float(), std::integral_constant<int, 32>())
               : f(double(), std::integral_constant<int, 32>());
}

}  // namespace

int spmm_lanes(int nrhs) {
    int R = 1;
    while (R < nrhs && R < 32) R *= 2;
    return R;
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
    M.lanes = spmm_lanes(nrhs);
    return M;
}

cudaError_t launch_spmm(const DevLayout &d, const void *x, void *y, int nrhs, int64_t ldx,
                        int64_t ldy, int lanes, cudaStream_t stream) {
    if (d.ntiles == 0) return cudaSuccess;
    const MatView M = mat_view(d, x, y, nrhs, ldx, ldy);
    const int R = lanes > 0 ? lanes : spmm_lanes(nrhs);
    return by_type(d.bs, d.f32, [&](auto t, auto bs) {
        using T = decltype(t);
        return by_r<T, bs()>(R, [&](auto r) { return spmm_launch_r<T, bs(), r()>(M, d.sched, stream); });
    });
}

int64_t batch_warps(int bs, int f32) {
    return by_type(bs, f32, [&](auto t, auto b) {
        using T = decltype(t);
        return batch_warps_t<T, b()>();
    });
}

cudaError_t launch_batch(int bs, int f32, const MatView *mats, int nmats, const int64_t *toff,
                         const int64_t *wpart, int64_t nwarps, cudaStream_t stream) {
    return by_type(bs, f32, [&](auto t, auto b) {
        using T = decltype(t);
        return batch_launch_t<T, b()>(mats, nmats, toff, wpart, nwarps, stream);
    });
}

int64_t batch_tile_cost(const uint32_t *tile8, const uint32_t *blocks4, int nrhs) {
    const int R = spmm_lanes(nrhs);
    const int64_t passes = (nrhs + R - 1) / R;
    const uint32_t counts = tile8[2];
    const uint32_t nb = counts & 0xff, ncoo = (counts >> 8) & 0xff;
    double work = (double)tile8[4];  // COO entries
    for (uint32_t q = ncoo; q < nb; ++q)
        work += 1.5 * (double)((blocks4[4 * (tile8[0] + q) + 1] >> 3) & 2047);
    // ~100 instruction slots per tile pass, ~15 per 32 lane-entries
    return (int64_t)(passes * (100.0 + 15.0 * work * R / 32.0));
}

}  // namespace cb
