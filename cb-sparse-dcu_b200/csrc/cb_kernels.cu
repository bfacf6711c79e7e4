// sm_100a kernels of the CB-SpMV: the tile kernel (the reference's `comp` and
// `gather` kernels, cb-spmv-dcu.hpp:159-1084, folded into one: the layout
// resolves COO columns at build time and stages gathered x columns per
// CSR/DENSE block), plus value refresh and value-gradient kernels.
//
// Mapping (32-lane warps, one warp per tile, 8 warps per CTA):
//   phase 1  products of all COO entries of the tile, lane-strided with
//            independent loads (idx, value, x[col]) -> shared memory; x tiles
//            of the CSR/DENSE blocks (bs values each, through the gather list
//            when the matrix was gathered) -> shared memory.
//   phase 2  per COO block: a segmented scan over its row runs (entries are
//            sorted by row inside a block, coo2block.h:219-227), two blocks of
//            <= 16 entries per warp, 32-entry passes otherwise; the number of
//            scan steps is the block's log2(longest run), stored in its
//            descriptor.  CSR: 32/bs lanes per row (the reference's
//            LANES_PER_ROW, macros.h:84, re-derived for 32 lanes).  DENSE:
//            2 lanes per row for bs=16, 1 for bs=32.  Run tails add into two
//            per-warp row accumulators (one per half-warp), never colliding.
//   phase 3  the tile's bs row sums go to y, or for a block row split over
//            several tiles to a partial slot; the last tile to arrive on the
//            row's counter adds all partials in tile order and stores y.  No
//            tile waits on another (the reference spins on a row epoch,
//            cb-spmv-dcu.hpp:238-282).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <type_traits>

#include "cb_kernels.hpp"

namespace cb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 8;
constexpr uint32_t kColMask = (1u << 27) - 1;

__host__ __device__ constexpr int max_xt(int bs) { return bs == 16 ? 16 : 8; }
__host__ __device__ constexpr uint32_t a16(uint32_t x) { return (x + 15u) & ~15u; }

// Per-warp shared memory.  acc holds one private row accumulator per lane
// (lane l owns acc[l * (BS + 1) + r]; the +1 pad spreads a column over the
// banks), so entries accumulate without atomics and in a fixed order.
template <typename T, int BS>
struct WarpSmem {
    T xt[max_xt(BS) * BS];      // x tiles of the tile's CSR/DENSE blocks
    T acc[32 * (BS + 1)];
};

template <typename T>
__device__ __forceinline__ T ldg(const T *p) {
    return __ldg(p);
}

// Sums the 32 lane-private accumulators of row r = lane % BS, clearing them
// for the next tile.  Lanes >= BS (BS = 16) sum the upper 16 lanes' copies and
// hand their half over by shuffle.  Result valid in lanes < BS.
template <typename T, int BS>
__device__ __forceinline__ T reduce_rows(T *acc, int lane) {
    T s = T(0);
    if (BS == 16) {
        const int r = lane & 15, l0 = (lane >> 4) * 16;
#pragma unroll
        for (int l = 0; l < 16; ++l) {
            T *p = &acc[(l0 + l) * (BS + 1) + r];
            s += *p;
            *p = T(0);
        }
        s += __shfl_down_sync(kFull, s, 16);
    } else {
#pragma unroll 8
        for (int l = 0; l < 32; ++l) {
            T *p = &acc[l * (BS + 1) + lane];
            s += *p;
            *p = T(0);
        }
    }
    return s;
}

// Persistent warps fetch tiles from a global counter (sched[0]); the warp
// whose exit completes sched[1] == number of warps resets both for the next
// launch, so no launch waits on another and no host reset is needed.
// kChunk COO entries per lane have their loads in flight together; nrhs
// right-hand sides are handled one after another (x column j at
// x[col * ldx + j]).
template <typename T, int BS, int kChunk>
__global__ void __launch_bounds__(kWarps * 32, 4)
    cb_spmv_tile_kernel(const uint4 *__restrict__ tiles, int64_t ntiles,
                        const uint4 *__restrict__ blocks,
                        const uint8_t *__restrict__ payload,
                        const int32_t *__restrict__ block_cols, int gather,
                        const T *__restrict__ x, T *__restrict__ y, int64_t m,
                        int nrhs, int64_t ldx, int64_t ldy,
                        T *__restrict__ partials, int32_t *__restrict__ counters,
                        uint32_t *__restrict__ sched) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    WarpSmem<T, BS> &S = reinterpret_cast<WarpSmem<T, BS> *>(smem_raw)[wib];
    T *myacc = &S.acc[lane * (BS + 1)];
    for (int t = lane; t < 32 * (BS + 1); t += 32) S.acc[t] = T(0);
    __syncwarp();

    auto grab = [&]() -> int64_t {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&sched[0], 1u);
        return (int64_t)__shfl_sync(kFull, t, 0);
    };
    int64_t tile = grab();
    uint4 na = make_uint4(0, 0, 0, 0), nb4 = na;
    if (tile < ntiles) {
        na = __ldg(&tiles[2 * tile]);
        nb4 = __ldg(&tiles[2 * tile + 1]);
    }
    while (tile < ntiles) {
        const uint4 ta = na;   // begin, row, counts, pay16
        const uint4 tb = nb4;  // E, slot, first, ntiles
        const int64_t next = grab();
        if (next < ntiles) {
            na = __ldg(&tiles[2 * next]);
            nb4 = __ldg(&tiles[2 * next + 1]);
        }
        const int nb = ta.z & 0xff;
        const int ncoo = (ta.z >> 8) & 0xff;
        const int nxt = (ta.z >> 16) & 0xff;
        const int E = (int)tb.x;
        const uint8_t *base = payload + (size_t)ta.w * 16;
        uint4 bd = make_uint4(0, 0, 0, 0);
        if (lane < nb) bd = __ldg(&blocks[ta.x + lane]);
        const uint32_t *cidx = reinterpret_cast<const uint32_t *>(base);
        const T *cval = reinterpret_cast<const T *>(base + a16(4u * E));
        const int64_t row0 = (int64_t)ta.y * BS;

        for (int j = 0; j < nrhs; ++j) {
            const T *xj = x + j;
            // x tiles of CSR/DENSE blocks (through the gather list if any)
            for (int t0 = 0; t0 < nxt * BS; t0 += 32) {
                const int t = t0 + lane;
                const int jb = min(t / BS, nxt - 1);
                const uint32_t xb = __shfl_sync(kFull, bd.z, ncoo + jb);
                const uint32_t mb = __shfl_sync(kFull, bd.y, ncoo + jb);
                const int c = t % BS;
                const int valid = (mb >> 14) & 63;
                if (t < nxt * BS) {
                    T xv = T(0);
                    if (c < valid) {
                        const int64_t col = gather ? (int64_t)__ldg(&block_cols[xb + c])
                                                   : (int64_t)(xb + c);
                        xv = ldg(&xj[col * ldx]);
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
                        v[u] = __ldg(&cval[e]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kChunk; ++u) {
                    const int e = c0 + u * 32 + lane;
                    xv[u] = e < E ? ldg(&xj[(int64_t)(w[u] & kColMask) * ldx]) : T(0);
                }
#pragma unroll
                for (int u = 0; u < kChunk; ++u) {
                    const int e = c0 + u * 32 + lane;
                    if (e < E) myacc[w[u] >> 27] += v[u] * xv[u];
                }
            }

            // CSR and DENSE blocks
            for (int jb = 0; jb < nxt; ++jb) {
                const uint32_t off = __shfl_sync(kFull, bd.x, ncoo + jb);
                const uint32_t mb = __shfl_sync(kFull, bd.y, ncoo + jb);
                const int k = (mb >> 3) & 2047;
                const uint8_t *pb = base + off;
                const T *xt = &S.xt[jb * BS];
                if ((mb & 3) == 1) {
                    using IdxT = typename std::conditional<BS == 16, uint8_t, uint16_t>::type;
                    const IdxT *rp = reinterpret_cast<const IdxT *>(pb);
                    const IdxT *ci = rp + BS + 1;
                    const T *vv = reinterpret_cast<const T *>(
                        pb + a16((uint32_t)((BS + 1 + k) * sizeof(IdxT))));
                    constexpr int L = 32 / BS;
                    const int row = lane / L, sub = lane % L;
                    const int kb = __ldg(&rp[row]), ke = __ldg(&rp[row + 1]);
                    T sum = T(0);
                    for (int q = kb + sub; q < ke; q += L)
                        sum += __ldg(&vv[q]) * xt[__ldg(&ci[q])];
                    myacc[row] += sum;
                } else {
                    const T *vv = reinterpret_cast<const T *>(pb);
                    T sum = T(0);
                    if (BS == 16) {
                        const int row = lane >> 1, c0 = (lane & 1) * 8;
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            sum += __ldg(&vv[row * 16 + c0 + c]) * xt[c0 + c];
                        myacc[row] += sum;
                    } else {
#pragma unroll 8
                        for (int c = 0; c < BS; ++c)
                            sum += __ldg(&vv[lane * BS + c]) * xt[c];
                        myacc[lane] += sum;
                    }
                }
            }
            __syncwarp();
            const T s = reduce_rows<T, BS>(S.acc, lane);
            __syncwarp();

            // output: whole block row -> y; split row -> partial slot, and the
            // last tile to arrive adds the row's partials in tile order
            const int64_t grow = row0 + lane;
            if (tb.y == 0xffffffffu) {
                if (lane < BS && grow < m) y[grow * ldy + j] = s;
            } else {
                T *part = partials + ((size_t)tb.y * nrhs + j) * BS;
                if (lane < BS) part[lane] = s;
                __threadfence();
                __syncwarp();
                int last = 0;
                if (lane == 0) {
                    const int old = atomicAdd(&counters[ta.y], 1);
                    last = old == (int)(tb.w * nrhs) - 1;
                }
                last = __shfl_sync(kFull, last, 0);
                if (last) {
                    __threadfence();
                    if (lane < BS) {
                        for (int jj = 0; jj < nrhs; ++jj) {
                            T tot = T(0);
                            for (uint32_t t = 0; t < tb.w; ++t)
                                tot += __ldcg(&partials[((size_t)(tb.z + t) * nrhs + jj) * BS + lane]);
                            if (grow < m) y[grow * ldy + jj] = tot;
                        }
                    }
                    if (lane == 0) atomicExch(&counters[ta.y], 0);
                }
            }
        }
        tile = next;
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

template <typename T>
__global__ void cb_grad_vals_kernel(int64_t nvals, const int32_t *__restrict__ vrow,
                                    const int32_t *__restrict__ vcol,
                                    const T *__restrict__ g, int64_t ldg,
                                    const T *__restrict__ x, int64_t ldx, int nrhs,
                                    T *__restrict__ out) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvals) return;
    const int32_t r = vrow[v], c = vcol[v];
    T s = T(0);
    if (r >= 0 && c >= 0)
        for (int j = 0; j < nrhs; ++j)
            s += __ldg(&g[(int64_t)r * ldg + j]) * __ldg(&x[(int64_t)c * ldx + j]);
    out[v] = s;
}

template <typename T, int BS, int CH>
cudaError_t launch_chunk(const DevLayout &d, const void *x, void *y, int nrhs,
                         int64_t ldx, int64_t ldy, cudaStream_t stream) {
    const size_t smem = sizeof(WarpSmem<T, BS>) * kWarps;
    static int resident = 0;  // CTAs per SM, per instantiation
    static int sms = 0;
    if (!resident) {
        cudaError_t e = cudaFuncSetAttribute(cb_spmv_tile_kernel<T, BS, CH>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, cb_spmv_tile_kernel<T, BS, CH>,
                                                      kWarps * 32, smem);
        if (resident < 1) resident = 1;
    }
    int64_t grid = (d.ntiles + kWarps - 1) / kWarps;
    grid = std::min<int64_t>(grid, (int64_t)sms * resident);
    if (grid == 0) return cudaSuccess;
    cb_spmv_tile_kernel<T, BS, CH><<<(unsigned)grid, kWarps * 32, smem, stream>>>(
        static_cast<const uint4 *>(d.tiles), d.ntiles,
        static_cast<const uint4 *>(d.blocks), d.payload, d.block_cols, d.gather,
        static_cast<const T *>(x), static_cast<T *>(y), d.m, nrhs, ldx, ldy,
        static_cast<T *>(d.partials), d.counters, d.sched);
    return cudaGetLastError();
}

int chunk_choice(int vsz) {
    static int forced = -1;
    if (forced < 0) {
        const char *e = std::getenv("CBSPMV_CHUNK");
        forced = e ? std::atoi(e) : 0;
    }
    if (forced == 4 || forced == 6 || forced == 8) return forced;
    return vsz == 8 ? 6 : 8;
}

template <typename T, int BS>
cudaError_t launch_tiles(const DevLayout &d, const void *x, void *y, int nrhs,
                         int64_t ldx, int64_t ldy, cudaStream_t stream) {
    switch (chunk_choice(sizeof(T))) {
        case 4: return launch_chunk<T, BS, 4>(d, x, y, nrhs, ldx, ldy, stream);
        case 6: return launch_chunk<T, BS, 6>(d, x, y, nrhs, ldx, ldy, stream);
        default: return launch_chunk<T, BS, 8>(d, x, y, nrhs, ldx, ldy, stream);
    }
}

}  // namespace

size_t spmv_smem_bytes(int bs, int f32) {
    if (bs == 16)
        return kWarps * (f32 ? sizeof(WarpSmem<float, 16>) : sizeof(WarpSmem<double, 16>));
    return kWarps * (f32 ? sizeof(WarpSmem<float, 32>) : sizeof(WarpSmem<double, 32>));
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
    return cudaGetLastError();
}

cudaError_t launch_grad_vals(int f32, int64_t nvals, const int32_t *vrow,
                             const int32_t *vcol, const void *g, int64_t ldg,
                             const void *x, int64_t ldx, int nrhs, void *gvals,
                             cudaStream_t stream) {
    if (nvals == 0) return cudaSuccess;
    const unsigned grid = (unsigned)((nvals + 255) / 256);
    if (f32)
        cb_grad_vals_kernel<float><<<grid, 256, 0, stream>>>(
            nvals, vrow, vcol, static_cast<const float *>(g), ldg,
            static_cast<const float *>(x), ldx, nrhs, static_cast<float *>(gvals));
    else
        cb_grad_vals_kernel<double><<<grid, 256, 0, stream>>>(
            nvals, vrow, vcol, static_cast<const double *>(g), ldg,
            static_cast<const double *>(x), ldx, nrhs, static_cast<double *>(gvals));
    return cudaGetLastError();
}

}  // namespace cb
