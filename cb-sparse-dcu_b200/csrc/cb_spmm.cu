// sm_100a multi-right-hand-side CB-SpMV and batches: Y = A X with X (n x nrhs)
// and Y (m x nrhs) row-major (leading dimensions ldx, ldy), over the same tile
// layout as the single-vector kernels (cb_kernels.cu); a batch runs many such
// products, of any sizes and right-hand-side counts, in ONE launch.
//
// cb_mslice_kernel: persistent warps take units of consecutive tiles (of one
// matrix, or of a batch's concatenated tile list) from a counter, one unit
// ahead, and double-buffer whole tile payloads -- COO section, CSR and DENSE
// payloads -- in shared memory with bulk asynchronous copies (TMA, no
// multicast): the next tile is in flight while one is computed from shared
// memory.  Tile payloads are capped in size by the packer so two fit per warp.
//
// A tile is computed in passes of NV right-hand sides (NV = 4 FP32 / 2 FP64,
// or 1 for a single vector), each lane gathering NV consecutive values of an
// x row (one vector load where the layout allows it).  COO sections are
// stored in lane slices of consecutive entries (coo_slice_pos, cb_layout.hpp):
// each lane sums its slice along its rows in registers, and one segmented
// shuffle scan per pass joins the rows that run across lanes, so every row of
// the tile is added into the warp's accumulators exactly once per pass, by
// one lane.  CSR and DENSE blocks: one lane per row (a half-warp per 16 x 16
// block, two blocks at a time), their x rows staged in shared memory.  The
// accumulators hold up to kRA right-hand sides of the block row being summed
// (one copy per warp); consecutive tiles of one block row inside a warp's
// range keep adding into them.  More right-hand sides are summed kRA at a
// time, every tile then being a run of its own.
//
// Block rows split over several tiles: a row whose tiles all lie in one
// warp's run is stored directly; otherwise each run leaves its sums in the
// slot of its first tile and the last run to arrive on the row's counter adds
// them in tile order.  No tile waits on another.  Every mbarrier wait is
// bounded; on give-up the error word is set and the warp stops after draining
// its own copies.
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
using dev::bulk_g2s;
using dev::dense_at;
using dev::fence_mbar_init;
using dev::fence_proxy_async;
using dev::kColMask;
using dev::kFull;
using dev::kWaitLimit;
using dev::mbar_arrive;
using dev::mbar_arrive_tx;
using dev::mbar_init;
using dev::mbar_wait;
using dev::policy_evict_first;

constexpr int kMsWarps = 4;  // warps per CTA
constexpr int kRA = 16;      // right-hand sides the accumulators hold
constexpr int kSub = 4;      // slice entries per lane in registers at a time

template <typename T>
struct VecOf {
    static constexpr int V = sizeof(T) == 4 ? 4 : 2;
};

// Per-warp shared memory: [acc | xt | xo | mbar[2] | buf[2]].  acc: BS rows x kRA
// right-hand sides (row r, column c at acc[r * kRA + c]); xt: the x rows of
// the CSR/DENSE blocks of one step (RL * V values for every block column of
// BPS blocks, at most 4 V); buf: one tile payload (`cap` bytes).
template <typename T, int BS>
struct MsLayout {
    static constexpr int V = VecOf<T>::V;
    static constexpr uint32_t acc_bytes = BS * kRA * sizeof(T);
    static constexpr uint32_t xt_bytes = BS * 4 * V * sizeof(T);
    static constexpr uint32_t xo_bytes = BS * 4 * V * sizeof(T);
    static constexpr uint32_t head = a16(acc_bytes + xt_bytes + xo_bytes + 16);
    __host__ __device__ static uint32_t bytes(uint32_t cap) { return head + 2 * cap; }
};

// NV consecutive values at p: one vector load when vec (aligned), else nv
// scalar loads (the rest 0).
template <typename T, int NV>
__device__ __forceinline__ void ldg_row(const T *p, bool vec, int nv, T (&o)[NV]) {
    if constexpr (NV == 4 && sizeof(T) == 4) {
        if (vec) {
            const float4 f = __ldg(reinterpret_cast<const float4 *>(p));
            o[0] = f.x, o[1] = f.y, o[2] = f.z, o[3] = f.w;
            return;
        }
    } else if constexpr (NV == 2 && sizeof(T) == 8) {
        if (vec) {
            const double2 f = __ldg(reinterpret_cast<const double2 *>(p));
            o[0] = f.x, o[1] = f.y;
            return;
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = v < nv ? __ldg(p + v) : T(0);
}

// The lanes of a warp form G = 32 / RL groups of RL lanes; a group works on
// one entry (or one block row) at a time, its lanes on NV consecutive
// right-hand sides each, so one x row is read by RL lanes side by side (RL
// pieces of NV values).
//
// One pass of a tile's COO section over right-hand sides c0 + [0, RL * NV)
// (accumulator columns ca + ...).  The section is stored in 32 lane slices
// of consecutive entries (coo_slice_pos, cb_layout.hpp); group g takes the
// RL slices g RL, ..., g RL + RL - 1 in turn -- slot q = t Kt + j is entry j
// of slice g RL + t, at position 32 j + g RL + t (none when not below E) --
// so its entries are one run of the sorted section.  Each lane sums along
// the rows in registers, kSub slots at a time (a slot with no entry carries
// the row on and adds 0); a row that begins and ends inside the group's
// range is added into acc by the group itself, and one segmented shuffle
// scan over the groups joins the rows that run across groups: the scheme of
// the single-vector streaming kernel (slice_sums, cb_device.cuh).  Each row
// of the tile is added by exactly one group, so no two lanes write one
// accumulator.
template <typename T, int BS, int RL, int NV, bool GV>
__device__ __forceinline__ void coo_pass(const MatView &M, const uint4 ta,
                                         const unsigned char *buf, int E, int c0, int ca,
                                         T *__restrict__ acc, const T *__restrict__ xo,
                                         int lane) {
    constexpr uint32_t kNone = 63;  // row of a group with no entry (after every real row)
    constexpr int G = 32 / RL;
    const int g = lane / RL, sub = lane % RL;
    const uint32_t *sidx = reinterpret_cast<const uint32_t *>(buf);
    const T *sval = reinterpret_cast<const T *>(buf + a16(4u * E));
    const int cl = c0 + sub * NV;                    // this lane's first right-hand side
    const int nv = max(0, min(NV, M.nrhs - cl));     // of them real
    const int cal = ca + sub * NV;                   // its first accumulator column
    const T *__restrict__ xr = static_cast<const T *>(M.x) + cl;
    const bool vec = M.xvec != 0;
    const int Kt = (E + 31) >> 5;
    const int nslots = RL * Kt;
    uint32_t rh = kNone, rc = kNone;  // head row, row of the running sum
    bool split = false;               // the group's range holds more than one row
    T run[NV], head[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) run[v] = head[v] = T(0);
    int t = 0, j = 0;  // slot being loaded: slice g RL + t, entry j
    for (int q0 = 0; q0 < nslots; q0 += kSub) {
        int pos[kSub];
        uint32_t w[kSub];
        T a[kSub], xv[kSub][NV];
#pragma unroll
        for (int u = 0; u < kSub; ++u) {
            pos[u] = t < RL ? 32 * j + g * RL + t : E;
            if (++j == Kt) {
                j = 0;
                ++t;
            }
            w[u] = pos[u] < E ? sidx[pos[u]] : 0u;
            a[u] = pos[u] < E ? (M.unit ? T(1) : sval[pos[u]]) : T(0);
        }
#pragma unroll
        for (int u = 0; u < kSub; ++u) {
            if (pos[u] < E && nv > 0) {
                ldg_row<T, NV>(xr + (size_t)(w[u] & kColMask) * (size_t)M.ldx, vec, nv, xv[u]);
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) xv[u][v] = T(0);
            }
        }
        if (GV) {  // value gradient: x row . own row, summed over the group's lanes
            T *gv = static_cast<T *>(M.gv) +
                    ((size_t)ta.w * 16 + a16(4u * E)) / sizeof(T);
#pragma unroll
            for (int u = 0; u < kSub; ++u) {
                const int r = pos[u] < E ? (int)(w[u] >> 27) : 0;
                T d = T(0);
#pragma unroll
                for (int v = 0; v < NV; ++v) d = fma(xv[u][v], xo[r * RL * NV + sub * NV + v], d);
#pragma unroll
                for (int o = RL / 2; o > 0; o >>= 1) d += __shfl_xor_sync(kFull, d, o);
                if (sub == 0 && pos[u] < E) gv[pos[u]] = c0 == 0 ? d : gv[pos[u]] + d;
            }
        }
#pragma unroll
        for (int u = 0; u < kSub; ++u) {
            if (q0 + u >= nslots) break;  // warp-uniform
            const uint32_t r = pos[u] < E ? (w[u] >> 27) : rc;
            if (q0 + u == 0) {  // the group's first slot
                rh = rc = r;
#pragma unroll
                for (int v = 0; v < NV; ++v) run[v] = a[u] * xv[u][v];
                continue;
            }
            const bool chg = r != rc;
            if (chg && split) {  // a row complete inside the group's range
#pragma unroll
                for (int v = 0; v < NV; ++v)
                    if (v < nv) acc[rc * kRA + cal + v] += run[v];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                head[v] = (chg && !split) ? run[v] : head[v];
                const T p = a[u] * xv[u][v];
                run[v] = chg ? p : run[v] + p;
            }
            split = split || chg;
            rc = r;
        }
    }
    // rows across groups: `run` holds the sum of the tail row rc
    const uint32_t rt_prev = __shfl_up_sync(kFull, rc, RL);
    const uint32_t rh_next = __shfl_down_sync(kFull, rh, RL);
    const bool cont = g > 0 && rh == rt_prev;  // my head goes on from the previous group
    const uint32_t heads = __ballot_sync(kFull, !cont || split);
    const int start = (31 - __clz(heads & (0xffffffffu >> (31 - lane)))) / RL;  // head group
    const uint32_t longest = __reduce_max_sync(kFull, (uint32_t)(g - start + 1));
#pragma unroll
    for (int d = 1; d < G; d <<= 1) {
        if ((uint32_t)d >= longest) break;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const T tt = __shfl_up_sync(kFull, run[v], d * RL);
            if (g - d >= start) run[v] += tt;
        }
    }
    T prev[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) prev[v] = __shfl_up_sync(kFull, run[v], RL);
    if (split) {
#pragma unroll
        for (int v = 0; v < NV; ++v)
            if (v < nv) acc[rh * kRA + cal + v] += cont ? head[v] + prev[v] : head[v];
    }
    if ((g == G - 1 || rh_next != rc) && rc < (uint32_t)BS) {
#pragma unroll
        for (int v = 0; v < NV; ++v)
            if (v < nv) acc[rc * kRA + cal + v] += run[v];
    }
    __syncwarp();
}

// One pass of a tile's CSR and DENSE blocks over right-hand sides c0 +
// [0, RL * NV): P = 32 / RL row slots; a step covers BPS = max(1, P / BS)
// blocks (their x rows staged in xt, column c of block q at
// xt[(q * BS + c) * RL * NV]), each row slot summing rows p, p + P, ... of
// its block (DENSE columns in a rotated order, so the slots of a step read
// distinct banks); with two blocks per step the second block's slots hand
// their sums to the first by a shuffle, so each row is added by one group.
template <typename T, int BS, int RL, int NV, bool GV>
__device__ __forceinline__ void blk_pass(const MatView &M, const uint4 ta,
                                         const unsigned char *buf, int c0, int ca,
                                         T *__restrict__ acc, T *__restrict__ xt,
                                         const T *__restrict__ xo, int lane) {
    constexpr int P = 32 / RL;
    constexpr int BPS = P >= BS ? P / BS : 1;  // blocks per step (1 or 2)
    constexpr int RW = RL * NV;                // x values per column
    using IdxT = typename std::conditional<BS == 16, uint8_t, uint16_t>::type;
    const int ncoo = (ta.z >> 8) & 0xff, nxt = (ta.z >> 16) & 0xff;
    const int p = lane / RL, sub = lane % RL;
    const int cl = c0 + sub * NV;
    const int nv = max(0, min(NV, M.nrhs - cl));
    const int cal = ca + sub * NV;
    const bool vec = M.xvec != 0;
    const uint4 bd =
        lane < nxt ? __ldg(&M.blocks[ta.x + ncoo + lane]) : make_uint4(0, 0, 0, 0);
    const int q = BPS > 1 ? p / BS : 0;           // block of this slot in the step
    const int prow = BPS > 1 ? p % BS : p;        // first row of this slot
    for (int jb = 0; jb < nxt; jb += BPS) {
        // stage the x rows: item i = (block qq, column c, piece s)
        for (int i = lane; i < BPS * BS * RL; i += 32) {
            const int s = i % RL, c = (i / RL) % BS, qq = i / (RL * BS);
            const int jj = min(jb + qq, nxt - 1);
            const uint32_t mb = __shfl_sync(kFull, bd.y, jj);
            const uint32_t xbase = __shfl_sync(kFull, bd.z, jj);
            const int cs = c0 + s * NV;
            const int ns = max(0, min(NV, M.nrhs - cs));
            T xv[NV];
            if (jb + qq < nxt && c < (int)((mb >> 14) & 63) && ns > 0) {
                const int64_t col = M.gather ? (int64_t)__ldg(&M.block_cols[xbase + c])
                                             : (int64_t)(xbase + c);
                ldg_row<T, NV>(static_cast<const T *>(M.x) + (size_t)col * (size_t)M.ldx + cs,
                               vec, ns, xv);
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) xv[v] = T(0);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) xt[(qq * BS + c) * RW + s * NV + v] = xv[v];
        }
        __syncwarp();
        const int j = jb + q;
        const int jc = min(j, nxt - 1);
        const uint32_t off = __shfl_sync(kFull, bd.x, jc);
        const uint32_t mb = __shfl_sync(kFull, bd.y, jc);
        const unsigned char *pb = buf + off;
        const T *xq = xt + q * BS * RW + sub * NV;
        // value gradient: the lanes of one row slot sum their pieces
        const unsigned gmask = (RL == 1 ? 1u : ((1u << RL) - 1u)) << (p * RL);
        T *gvb = GV ? static_cast<T *>(M.gv) + ((size_t)ta.w * 16 + off) / sizeof(T) : nullptr;
#pragma unroll 1
        for (int row = prow; row < BS; row += (BPS > 1 ? BS : P)) {
            T sum[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) sum[v] = T(0);
            if (j < nxt) {
                if ((mb & 3) == 1) {  // CSR
                    const int k = (mb >> 3) & 2047;
                    const IdxT *rp = reinterpret_cast<const IdxT *>(pb);
                    const IdxT *ci = rp + BS + 1;
                    const T *vv = reinterpret_cast<const T *>(
                        pb + a16((uint32_t)((BS + 1 + k) * sizeof(IdxT))));
                    const int vo = (int)(a16((uint32_t)((BS + 1 + k) * sizeof(IdxT))) / sizeof(T));
                    for (int e = rp[row]; e < (int)rp[row + 1]; ++e) {
                        const T av = M.unit ? T(1) : vv[e];
                        const int c = ci[e];
#pragma unroll
                        for (int v = 0; v < NV; ++v) sum[v] = fma(av, xq[c * RW + v], sum[v]);
                        if (GV) {
                            T d = T(0);
#pragma unroll
                            for (int v = 0; v < NV; ++v)
                                d = fma(xq[c * RW + v], xo[row * RW + sub * NV + v], d);
#pragma unroll
                            for (int o = RL / 2; o > 0; o >>= 1) d += __shfl_xor_sync(gmask, d, o);
                            if (sub == 0) gvb[vo + e] = c0 == 0 ? d : gvb[vo + e] + d;
                        }
                    }
                } else {  // DENSE, row-major BS x BS
#pragma unroll 4
                    for (int c = 0; c < BS; ++c) {
                        const int cc = (c + row) & (BS - 1);
                        const T av = dense_at<T, BS>(pb, M.unit, row, cc);
#pragma unroll
                        for (int v = 0; v < NV; ++v) sum[v] = fma(av, xq[cc * RW + v], sum[v]);
                        if (GV) {
                            T d = T(0);
#pragma unroll
                            for (int v = 0; v < NV; ++v)
                                d = fma(xq[cc * RW + v], xo[row * RW + sub * NV + v], d);
#pragma unroll
                            for (int o = RL / 2; o > 0; o >>= 1) d += __shfl_xor_sync(gmask, d, o);
                            if (sub == 0) {
                                T *gp = gvb + row * BS + cc;
                                *gp = c0 == 0 ? d : *gp + d;
                            }
                        }
                    }
                }
            }
            if (BPS > 1) {
#pragma unroll
                for (int v = 0; v < NV; ++v) sum[v] += __shfl_down_sync(kFull, sum[v], BS * RL);
            }
            if (q == 0) {
#pragma unroll
                for (int v = 0; v < NV; ++v)
                    if (v < nv) acc[row * kRA + cal + v] += sum[v];
            }
        }
        __syncwarp();
    }
}

// Value-gradient passes: the block row's own vectors for right-hand sides
// c0 + [0, RL * NV) into xo (row r, piece s at xo[r * RL * NV + s * NV]).
template <typename T, int BS, int RL, int NV>
__device__ __forceinline__ void stage_xo(const MatView &M, const uint4 ta, int c0, T *xo,
                                         int lane) {
    const bool vec = M.xvec != 0;
    __syncwarp();  // the previous pass is done with xo
    for (int i = lane; i < BS * RL; i += 32) {
        const int r = i / RL, sp = i % RL;
        const int64_t row = (int64_t)ta.y * BS + r;
        const int cs = c0 + sp * NV;
        const int ns = max(0, min(NV, M.nrhs - cs));
        T v[NV];
        if (row < M.m && ns > 0) {
            ldg_row<T, NV>(static_cast<const T *>(M.xo) + (size_t)row * (size_t)M.ldo + cs,
                           vec && M.ldo % NV == 0, ns, v);
        } else {
#pragma unroll
            for (int k = 0; k < NV; ++k) v[k] = T(0);
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) xo[i * NV + k] = v[k];
    }
    __syncwarp();
}

// Adds a staged tile into the accumulators for right-hand sides [cg0, cg1)
// (accumulator column c - cg0), RL * NV at a time; with M.gv, also the value
// gradient of every stored value of the tile.
template <typename T, int BS, int RL, int NV, bool GV>
__device__ __forceinline__ void tile_group(const MatView &M, const uint4 ta, const uint4 tb,
                                           const unsigned char *buf, int cg0, int cg1, T *acc,
                                           T *xt, T *xo, int lane) {
    const int E = (int)tb.x;
    const int nxt = (ta.z >> 16) & 0xff;
    for (int c0 = cg0; c0 < cg1; c0 += RL * NV) {
        if (GV) stage_xo<T, BS, RL, NV>(M, ta, c0, xo, lane);
        if (E > 0) coo_pass<T, BS, RL, NV, GV>(M, ta, buf, E, c0, c0 - cg0, acc, xo, lane);
        if (nxt) blk_pass<T, BS, RL, NV, GV>(M, ta, buf, c0, c0 - cg0, acc, xt, xo, lane);
    }
}

// Lanes per entry for R right-hand sides: the fewest (1, 2 or 4) whose
// RL * V values cover min(R, kRA), or 4 (more passes).  Three lane splits
// keep the kernel's code small enough for the instruction cache.
template <typename T>
__device__ __forceinline__ int lanes_for(int R) {
    constexpr int V = VecOf<T>::V;
    const int need = (min(R, kRA) + V - 1) / V;
    return need <= 1 ? 1 : need <= 2 ? 2 : 4;
}

// A tile for right-hand sides [cg0, cg1) with the lane split for R.
template <typename T, int BS, bool GV>
__device__ __forceinline__ void tile_any(const MatView &M, const uint4 ta, const uint4 tb,
                                         const unsigned char *buf, int cg0, int cg1, T *acc,
                                         T *xt, T *xo, int lane) {
    constexpr int V = VecOf<T>::V;
    switch (M.rl ? M.rl : lanes_for<T>(M.nrhs)) {
        case 1: return tile_group<T, BS, 1, V, GV>(M, ta, tb, buf, cg0, cg1, acc, xt, xo, lane);
        case 2: return tile_group<T, BS, 2, V, GV>(M, ta, tb, buf, cg0, cg1, acc, xt, xo, lane);
        default:
            return tile_group<T, BS, 4, V, GV>(M, ta, tb, buf, cg0, cg1, acc, xt, xo, lane);
    }
}

// Ends a run of `runlen` consecutive tiles of one block row (the last one
// tile g of the launch's tile list, descriptors ta/tb) for right-hand sides
// [cg0, cg0 + ncol): reads and clears those accumulator columns and stores Y,
// or, for a row whose tiles are not all in this run, leaves the run's sums in
// the slot of its first tile; the last run to arrive on the row's counter
// adds the row's runs in tile order (all right-hand sides).  groups: the
// number of column groups a tile is summed in; with one group, runs start at
// the row's first tile and at every scheduling unit start inside the row
// (ustart[0 .. nunits)), so the order does not depend on which warp ran
// which unit; with several, every tile is a run.
template <typename T, int BS>
__device__ __forceinline__ void ms_flush(const MatView &M, const uint4 ta, const uint4 tb,
                                         int64_t g, int64_t runlen, int cg0, int ncol,
                                         int groups, T *acc,
                                         const int64_t *__restrict__ ustart, int64_t nunits,
                                         int lane) {
    T *__restrict__ y = static_cast<T *>(M.y);
    T *part = static_cast<T *>(M.partials);
    const int64_t row0 = (int64_t)ta.y * BS;
    const bool whole = tb.y == 0xffffffffu || (groups == 1 && runlen == (int64_t)tb.w);
    const int64_t first = g - (int64_t)(tb.y - tb.z);  // the row's first tile
    const int64_t run0 = g - runlen + 1;
    __syncwarp();
    for (int o = lane; o < BS * ncol; o += 32) {
        const int r = o % BS, c = o / BS;
        const T s = acc[r * kRA + c];
        acc[r * kRA + c] = T(0);
        if (whole) {
            if (row0 + r < M.m) y[(row0 + r) * M.ldy + cg0 + c] = s;
        } else {
            const int64_t slot = (int64_t)tb.z + (run0 - first);
            part[((size_t)slot * M.nrhs + cg0 + c) * BS + r] = s;
        }
    }
    __syncwarp();
    if (whole) return;
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane == 0) {
        const int add = (int)runlen;
        const int old = atomicAdd(&M.counters[ta.y], add);
        last = old + add == (int)tb.w * groups;
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
        const int r = o % BS, c = o / BS;
        T tot = __ldcg(&part[((size_t)tb.z * M.nrhs + c) * BS + r]);
        if (groups > 1) {
            for (uint32_t t = 1; t < tb.w; ++t)
                tot += __ldcg(&part[((size_t)(tb.z + t) * M.nrhs + c) * BS + r]);
        } else {
            for (int64_t u = u0; u < nunits; ++u) {
                const int64_t b = __ldg(&ustart[u]);
                if (b >= end) break;
                tot += __ldcg(&part[((size_t)(tb.z + (b - first)) * M.nrhs + c) * BS + r]);
            }
        }
        if (row0 + r < M.m) y[(row0 + r) * M.ldy + c] = tot;
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

// Single matrix: mats == nullptr and `single` is the matrix (tiles
// [0, single.ntiles)).  Batch: mats[k] owns tiles [toff[k], toff[k+1]) of the
// launch's tile list, each with its own right-hand-side count.
// Tiles come in units -- unit u is [ustart[u], ustart[u+1]).  dynamic = 0:
// warp w runs unit w (host cost-balanced ranges, one per warp).  dynamic = 1:
// units of at least two tiles but the last, boundaries at block-row starts
// where the host could place them, taken from a counter (sched[0]) one unit
// ahead, in the queue order uorder (the costliest first; NULL: unit order);
// the warp whose exit completes sched[1] == number of warps resets both for
// the next launch.
template <typename T, int BS, bool GV>
__global__ void __launch_bounds__(kMsWarps * 32, 4)
    cb_mslice_kernel(const MatView single, const MatView *__restrict__ mats, int nmats,
                     const int64_t *__restrict__ toff, const int64_t *__restrict__ ustart,
                     const int32_t *__restrict__ uorder, int64_t nunits, int dynamic,
                     uint32_t cap, uint32_t *__restrict__ sched, uint32_t *__restrict__ err,
                     uint32_t limit) {
    using SL = MsLayout<T, BS>;
    constexpr int V = SL::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char *wbase = smem_raw + (size_t)wib * SL::bytes(cap);
    T *acc = reinterpret_cast<T *>(wbase);
    T *xt = reinterpret_cast<T *>(wbase + SL::acc_bytes);
    T *xo = reinterpret_cast<T *>(wbase + SL::acc_bytes + SL::xt_bytes);
    uint64_t *mbar =
        reinterpret_cast<uint64_t *>(wbase + SL::acc_bytes + SL::xt_bytes + SL::xo_bytes);
    unsigned char *const buf0 = wbase + SL::head;
    const uint64_t pol = policy_evict_first();

    for (int t = lane; t < BS * kRA; t += 32) acc[t] = T(0);
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
            if (ub < nunits && uorder) ub = __ldg(&uorder[ub]);  // queue order
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
            const int R = M.nrhs;
            if (R <= kRA) {  // one column group: runs across the block row's tiles
                tile_any<T, BS, GV>(M, ta, tb, buf, 0, R, acc, xt, xo, lane);
                ++runlen;
                if (!cont) {
                    ms_flush<T, BS>(M, ta, tb, g, runlen, 0, R, 1, acc, ustart, nunits, lane);
                    runlen = 0;
                }
            } else {  // kRA right-hand sides at a time, each tile a run
                const int groups = (R + kRA - 1) / kRA;
                for (int cg0 = 0; cg0 < R; cg0 += kRA) {
                    const int cg1 = min(R, cg0 + kRA);
                    tile_any<T, BS, GV>(M, ta, tb, buf, cg0, cg1, acc, xt, xo, lane);
                    ms_flush<T, BS>(M, ta, tb, g, 1, cg0, cg1 - cg0, groups, acc, ustart, nunits,
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

template <typename T, int BS, bool GV>
cudaError_t ms_configure(uint32_t cap, size_t *smem) {
    *smem = (size_t)MsLayout<T, BS>::bytes(cap) * kMsWarps;
    return dev_enable_smem(reinterpret_cast<const void *>(cb_mslice_kernel<T, BS, GV>), *smem);
}

template <typename T, int BS, bool GV = false>
int64_t ms_warps_t(uint32_t cap) {
    size_t smem = 0;
    if (ms_configure<T, BS, GV>(cap, &smem) != cudaSuccess) return 0;
    const int resident = dev_resident_l1(
        reinterpret_cast<const void *>(cb_mslice_kernel<T, BS, GV>), kMsWarps * 32, smem);
    return (int64_t)resident * dev_sms() * kMsWarps;
}

template <typename T, int BS, bool GV>
cudaError_t ms_launch_t(const MatView &single, const MatView *mats, int nmats,
                        const int64_t *toff, const int64_t *ustart, const int32_t *uorder,
                        int64_t nunits, int dynamic, uint32_t cap, uint32_t *sched,
                        uint32_t *err, cudaStream_t stream) {
    size_t smem = 0;
    cudaError_t e = ms_configure<T, BS, GV>(cap, &smem);
    if (e != cudaSuccess) return e;
    if (cap % 16 || !sched || !err) return cudaErrorInvalidValue;
    if (nunits <= 0) return cudaSuccess;
    // dynamic: resident warps (or fewer); static: one warp per unit.  The
    // resident count also sets the kernel's carveout for this buffer size.
    const int64_t resident_warps = ms_warps_t<T, BS, GV>(cap);
    const int64_t w = dynamic ? std::min<int64_t>(resident_warps, nunits) : nunits;
    const int64_t ctas = (w + kMsWarps - 1) / kMsWarps;
    cb_mslice_kernel<T, BS, GV><<<(unsigned)ctas, kMsWarps * 32, smem, stream>>>(
        single, mats, nmats, toff, ustart, uorder, nunits, dynamic, cap, sched, err,
        wait_polls());
    note_launch();
    return cudaGetLastError();
}

// Calls f(T(), BS) for the run-time value type and block size.
template <typename F>
auto by_type(int bs, int f32, F f) {
    if (bs == 16)
        return f32 ? f(float(), std::integral_constant<int, 16>())
                   : f(double(), std::integral_constant<int, 16>());
    return f32 ? f(float(), std::integral_constant<int, 32>())
               : f(double(), std::integral_constant<int, 32>());
}

}  // namespace

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
    M.rl = d.rl;
    // vector x loads of V values (4 FP32 / 2 FP64): rows aligned to V values
    // and every V-group a lane reads inside its row (ldx a multiple of V, the
    // last group within ldx)
    const int V = d.f32 ? 4 : 2;
    const size_t vsz = d.f32 ? 4 : 8;
    const int64_t vcols = (nrhs + V - 1) / V * V;
    M.xvec = reinterpret_cast<uintptr_t>(x) % (V * vsz) == 0 && ldx % V == 0 && vcols <= ldx;
    return M;
}

int64_t ms_warps(int bs, int f32, uint32_t cap) {
    return by_type(bs, f32, [&](auto t, auto b) {
        using T = decltype(t);
        return ms_warps_t<T, b()>(cap);
    });
}

int64_t ms_tile_cost(const uint32_t *tile8, const uint32_t *blocks4) {
    const uint32_t counts = tile8[2];
    const uint32_t nb = counts & 0xff, ncoo = (counts >> 8) & 0xff;
    int64_t work = 64 + tile8[4];  // per-tile overhead + COO entries
    for (uint32_t q = ncoo; q < nb; ++q) work += (blocks4[4 * (tile8[0] + q) + 1] >> 3) & 2047;
    return work;
}

int64_t ms_tile_cost_rhs(const uint32_t *tile8, const uint32_t *blocks4, int nrhs, int f32) {
    const int V = f32 ? 4 : 2;
    return ms_tile_cost(tile8, blocks4) * (int64_t)((nrhs + V - 1) / V);
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
                        int64_t ldy, cudaStream_t stream, void *gv, const void *xo,
                        int64_t ldo) {
    if (d.ntiles == 0) return cudaSuccess;
    if (!d.ustart) return cudaErrorInvalidValue;
    MatView M = mat_view(d, x, y, nrhs, ldx, ldy);
    if (gv) {
        if (!xo || d.unit) return cudaErrorInvalidValue;
        M.gv = gv;
        M.xo = xo;
        M.ldo = ldo;
        // own-row vector loads need the same alignment as x's
        const size_t vsz = d.f32 ? 4 : 8;
        const int V = d.f32 ? 4 : 2;
        if (reinterpret_cast<uintptr_t>(xo) % (V * vsz) != 0) M.xvec = 0;
    }
    return by_type(d.bs, d.f32, [&](auto t, auto b) {
        using T = decltype(t);
        return M.gv ? ms_launch_t<T, b(), true>(M, nullptr, 1, nullptr, d.ustart, nullptr,
                                                d.nunits, 0, d.mcap, d.sched, d.err, stream)
                    : ms_launch_t<T, b(), false>(M, nullptr, 1, nullptr, d.ustart, nullptr,
                                                 d.nunits, 0, d.mcap, d.sched, d.err, stream);
    });
}

cudaError_t launch_batch(int bs, int f32, const MatView *mats, int nmats, const int64_t *toff,
                         const int64_t *ustart, const int32_t *uorder, int64_t nunits,
                         uint32_t cap, uint32_t *sched, uint32_t *err, cudaStream_t stream) {
    return by_type(bs, f32, [&](auto t, auto b) {
        using T = decltype(t);
        return ms_launch_t<T, b(), false>(MatView(), mats, nmats, toff, ustart, uorder, nunits,
                                          1, cap, sched, err, stream);
    });
}

}  // namespace cb
