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

}  // namespace dev
}  // namespace cb
