// Tiled MLS step for B200: particles binned by cell tile, P2G accumulated by
// warps over runs of same-cell particles, and a grid update that only visits
// the node blocks P2G touched.
//
// Tiles are T^D cells (3D: 4^3, 2D: 8^2). Every `sort_period` steps (counted
// in absolute steps) a sort moves the particle state into the order
// (tile, cell in tile, particle id), which depends on the state alone
// (k_sort_count, k_sort_scan, k_sort_bucket, k_tile_sort). P2G (k_p2g_warp)
// groups consecutive slots whose particles share their current cell; inside
// a group the contributions are summed in FP32 in slot order, and every
// cross-group sum is an int64 fixed-point atomic. Grid sums are therefore
// bit-identical run to run, and a checkpoint that carries the slot order
// resumes bit-identically.
#pragma once

#include "mpm_kernels.cuh"

namespace mpm {

template <int D> struct TileGeom;
// T: cells per tile edge (also nodes per node-block edge); BN: nodes per block.
template <> struct TileGeom<3> { static constexpr int T = 4, BN = T * T * T; };
template <> struct TileGeom<2> { static constexpr int T = 8, BN = T * T; };

struct TileInfo {
    int tiles[3];      // cell tiles per axis
    int n_tiles;
    int nblk[3];       // node blocks per axis (nodes / T, rounded up)
    int n_blocks;
    int* key;          // per slot: tile of the particle at the last sort
    int* tile_count;   // per tile
    int* tile_cursor;  // per tile
    int* tile_start;   // per tile (exclusive scan of tile_count)
    int* mark;         // per node block: touched by this step's P2G
    int* mark_list;    // touched node blocks
    int* n_marked;     // device scalar
    int* perm;         // sort scratch: slot order by tile (source slots)
    int* tile_list;    // non-empty tiles of the last sort
    int* n_tile_list;  // device scalar
    int* p2g_next;     // device scalar: next P2G chunk to hand out (zeroed before each P2G)
    int* tile_len;     // per entry of tile_list: particles of that tile at the last sort
    int* fused_next;   // device scalar: next tile of the fused transfer (zeroed before each launch)
    unsigned long long* skey;  // global sort scratch (tiles above SortGeom<D>::SMEM particles)
    int* sval;
};

// The sort cell of a coordinate: floor(x + SHIFT) clamped to the grid, i.e.
// base + 1 of the stencil (the cell for the cubic stencil, the nearest node
// for the quadratic), so that particles sharing a stencil sort together.
template <int S> __device__ __forceinline__ int cell_clamped(float x, int ext) {
    if constexpr (Stencil<S>::SHIFT != 0.f) x += Stencil<S>::SHIFT;
    const int c = int(fminf(fmaxf(x, 0.f), float(ext) - 0.5f));
    return c < 0 ? 0 : (c >= ext ? ext - 1 : c);
}

template <int D, int S> __device__ __forceinline__ int tile_of_slot(const Particles& P, const StepConsts& C,
                                                                   const TileInfo& TI, int i) {
    constexpr int T = TileGeom<D>::T;
    const int ext[3] = {C.W, C.H, C.Dp};
    int t = 0;
#pragma unroll
    for (int k = D - 1; k >= 0; --k) t = t * TI.tiles[k] + cell_clamped<S>(P.x[k * P.n + i], ext[k]) / T;
    return t;
}

// ---------------------------------------------------------------------------
// Largest |v_k| over all particle velocity components (non-negative floats
// order as their bit patterns; NaN is skipped), for the auto sort period.
__global__ void __launch_bounds__(256) k_max_abs(const float* __restrict__ v, long long count,
                                                 unsigned* __restrict__ out) {
    float m = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(v[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(out, __float_as_uint(m));
}

// ---------------------------------------------------------------------------
// Counting sort by tile.

template <int D, int S = 4>
__global__ void __launch_bounds__(256) k_sort_count(Particles P, StepConsts C, TileInfo TI) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int t = tile_of_slot<D, S>(P, C, TI, i);
    TI.key[i] = t;
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, t);
    const int lane = threadIdx.x & 31;
    if (lane == __ffs(peers) - 1) atomicAdd(&TI.tile_count[t], __popc(peers));
}

// Single-CTA exclusive scans of the tile counts and of the non-empty tiles;
// writes each tile's first slot and the list of non-empty tiles, and clears
// the cursors for the bucket pass. Rounds of 1024 consecutive tiles (coalesced
// loads, eight rounds' loads issued together), each a warp-shuffle scan plus a
// scan of the 32 warp totals.
__global__ void __launch_bounds__(1024) k_sort_scan(TileInfo TI) {
    constexpr int R = 8;
    __shared__ int s_wc[32], s_wn[32], s_tc, s_tn, s_base, s_lbase;
    const int nt = TI.n_tiles, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) { s_base = 0; s_lbase = 0; }
    __syncthreads();
    for (int r0 = 0; r0 < nt; r0 += 1024 * R) {
        int cv[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int idx = r0 + q * 1024 + tid;
            cv[q] = idx < nt ? TI.tile_count[idx] : 0;
        }
#pragma unroll 1
        for (int q = 0; q < R && r0 + q * 1024 < nt; ++q) {
            const int idx = r0 + q * 1024 + tid;
            const int c = cv[q], ne = c > 0;
            int ic = c, in = ne;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, ic, off), v = __shfl_up_sync(0xffffffffu, in, off);
                if (lane >= off) { ic += u; in += v; }
            }
            if (lane == 31) { s_wc[warp] = ic; s_wn[warp] = in; }
            __syncthreads();
            if (warp == 0) {
                const int wc = s_wc[lane], wn = s_wn[lane];
                int jc = wc, jn = wn;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, jc, off), v = __shfl_up_sync(0xffffffffu, jn, off);
                    if (lane >= off) { jc += u; jn += v; }
                }
                s_wc[lane] = jc - wc;  // exclusive warp offsets
                s_wn[lane] = jn - wn;
                if (lane == 31) { s_tc = jc; s_tn = jn; }
            }
            __syncthreads();
            if (idx < nt) {
                TI.tile_start[idx] = s_base + s_wc[warp] + ic - c;
                TI.tile_cursor[idx] = 0;
                if (ne) TI.tile_list[s_lbase + s_wn[warp] + in - 1] = idx;  // non-empty tiles in tile order
            }
            __syncthreads();
            if (tid == 0) { s_base += s_tc; s_lbase += s_tn; }
            __syncthreads();
        }
    }
    if (tid == 0) *TI.n_tile_list = s_lbase;
}

struct SortBuffers {
    float *x, *v, *B, *Fe, *Jp, *A, *mass, *vol;
    int* id;
};

// Bucket the source slots by tile (order inside a tile is fixed by k_tile_sort).
__global__ void __launch_bounds__(256) k_sort_bucket(int n, TileInfo TI) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int t = TI.key[i];
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, t);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&TI.tile_cursor[t], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    TI.perm[TI.tile_start[t] + base + __popc(peers & ((1u << lane) - 1))] = i;
}

// Ascending bitonic sort of m (key, value) pairs, any m: the network of the
// next power of two with every index >= m standing for +infinity (all merges
// ascend, so such indices are never compared with a smaller key).
template <typename K, typename V>
__device__ void bitonic_sort_padded(K* key, V* val, int m) {
    int np = 1;
    while (np < m) np <<= 1;
    for (int k = 2; k <= np; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < np; i += blockDim.x) {
                const int l = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
                if (l > i && l < m) {
                    if (key[l] < key[i]) {
                        const K tk = key[i]; key[i] = key[l]; key[l] = tk;
                        const V tv = val[i]; val[i] = val[l]; val[l] = tv;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Particles per tile sorted in shared memory (12 B each) and CTAs per SM of
// the sort: 3D tiles (4^3 cells) rarely hold more than ~1000 particles, so a
// 24 KB buffer lets eight sorting CTAs share an SM; 2D tiles (8^2 cells) hold
// more and keep the 48 KB buffer.
template <int D> struct SortGeom;
template <> struct SortGeom<3> { static constexpr int SMEM = 2048, CTAS_PER_SM = 8; };
template <> struct SortGeom<2> { static constexpr int SMEM = 4032, CTAS_PER_SM = 4; };
constexpr int kTileCells = 64;   // cells per tile: 4^3 in 3D, 8^2 in 2D
constexpr int kCellSortMax = 64;  // counting sort when no cell of the tile holds more particles than this

// One CTA per non-empty tile: order the tile's particles by (cell in tile,
// particle id) -- a function of the state alone -- and gather their state into
// the destination buffers in that order. Tiles of up to SMEM / 2 particles
// whose cells hold at most kCellSortMax each take a counting sort by
// cell and a rank sort by id inside each cell (every item counts the smaller
// ids of its cell, all threads at once);
// larger tiles a bitonic network (in shared memory up to SMEM, else in
// global scratch). The result is the same order either way.
template <int D, int S = 4>
__global__ void __launch_bounds__(256) k_tile_sort(Particles P, const int* __restrict__ id_src, SortBuffers dst,
                                                   StepConsts C, TileInfo TI) {
    static_assert(TileGeom<D>::BN == kTileCells, "a tile has 64 cells");
    constexpr int T = TileGeom<D>::T;
    constexpr int kSortSmem = SortGeom<D>::SMEM, kCountSortMax = kSortSmem / 2;
    __shared__ unsigned long long s_key[kSortSmem];
    __shared__ int s_val[kSortSmem];
    __shared__ int s_cnt[kTileCells], s_off[kTileCells];
    __shared__ int s_big;
    const int n = P.n, ext[3] = {C.W, C.H, C.Dp};
    const int ntl = *TI.n_tile_list;
    for (int e = blockIdx.x; e < ntl; e += gridDim.x) {
        const int t = TI.tile_list[e];
        const int start = TI.tile_start[t];
        const int m = TI.tile_count[t];
        const bool in_smem = m <= kSortSmem;
        const bool counting = m <= kCountSortMax;
        unsigned long long* key = in_smem ? s_key : TI.skey + start;
        int* val = in_smem ? s_val : TI.sval + start;
        if (threadIdx.x < kTileCells) s_cnt[threadIdx.x] = 0;
        if (threadIdx.x == 0) s_big = 0;
        __syncthreads();
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            const int src = TI.perm[start + j];
            int cl = 0;
#pragma unroll
            for (int k = D - 1; k >= 0; --k) cl = cl * T + cell_clamped<S>(P.x[k * n + src], ext[k]) % T;
            key[j] = ((unsigned long long)cl << 32) | (unsigned)id_src[src];
            val[j] = src;
            if (counting) atomicAdd(&s_cnt[cl], 1);
        }
        __syncthreads();
        if (counting) {
            // exclusive scan of the 64 cell counts (one warp, two cells per lane)
            if (threadIdx.x < 32) {
                const int c0 = s_cnt[2 * threadIdx.x], c1 = s_cnt[2 * threadIdx.x + 1];
                int incl = c0 + c1;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, incl, o);
                    if ((int)threadIdx.x >= o) incl += u;
                }
                const int ex = incl - c0 - c1;
                s_off[2 * threadIdx.x] = ex;
                s_off[2 * threadIdx.x + 1] = ex + c0;
                if (max(c0, c1) > kCellSortMax) s_big = 1;
            }
            __syncthreads();
        }
        if (counting && !s_big) {
            // scatter by cell into the second half, then order each cell by id
            unsigned long long* key2 = s_key + kCountSortMax;
            int* val2 = s_val + kCountSortMax;
            if (threadIdx.x < kTileCells) s_cnt[threadIdx.x] = s_off[threadIdx.x];  // cursors
            __syncthreads();
            for (int j = threadIdx.x; j < m; j += blockDim.x) {
                const int p = atomicAdd(&s_cnt[(int)(key[j] >> 32)], 1);
                key2[p] = key[j];
                val2[p] = val[j];
            }
            __syncthreads();
            // each item's place in its cell = the number of smaller keys there
            // (keys are unique: cell and particle id), written back to the first half
            for (int j = threadIdx.x; j < m; j += blockDim.x) {
                const unsigned long long kj = key2[j];
                const int c = (int)(kj >> 32), lo = s_off[c], hi = s_cnt[c];
                int rank = 0;
                for (int q = lo; q < hi; ++q) rank += key2[q] < kj;
                key[lo + rank] = kj;
                val[lo + rank] = val2[j];
            }
            __syncthreads();
        } else {
            bitonic_sort_padded(key, val, m);
        }
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            const int src = val[j], s = start + j;
#pragma unroll
            for (int k = 0; k < D; ++k) { dst.x[k * n + s] = P.x[k * n + src]; dst.v[k * n + s] = P.v[k * n + src]; }
#pragma unroll
            for (int k = 0; k < D * D; ++k) {
                dst.B[k * n + s] = P.B[k * n + src];
                dst.Fe[k * n + s] = P.Fe[k * n + src];
                if (dst.A) dst.A[k * n + s] = P.A[k * n + src];
            }
            dst.Jp[s] = P.Jp[src];
            dst.id[s] = id_src[src];
            if (P.mass) dst.mass[s] = P.mass[src];
            if (P.vol) dst.vol[s] = P.vol[src];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            TI.tile_len[e] = m;
            TI.tile_count[t] = 0;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Node-block marking (which blocks of T^D nodes received mass this step).

__device__ __forceinline__ void mark_block(const TileInfo& TI, int b) {
    if (atomicExch(&TI.mark[b], 1) == 0) TI.mark_list[atomicAdd(TI.n_marked, 1)] = b;
}

// ---------------------------------------------------------------------------
// Grid update over the node blocks P2G marked (reads and clears the int64 sums).
template <int D, int FORM>
__global__ void __launch_bounds__(256) k_grid_marked(StepConsts C, TileInfo TI, unsigned long long* __restrict__ acc,
                                                     float4* __restrict__ gv, unsigned* __restrict__ status) {
    using G = TileGeom<D>;
    const int nb = *TI.n_marked;
    const long long total = (long long)nb * G::BN;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
         w += (long long)gridDim.x * blockDim.x) {
        const int blk = TI.mark_list[w / G::BN];
        const int loc = int(w % G::BN);
        int b[3] = {0, 0, 0}, l[3] = {0, 0, 0}, rb = blk, rl = loc;
#pragma unroll
        for (int k = 0; k < D; ++k) { b[k] = rb % TI.nblk[k]; rb /= TI.nblk[k]; l[k] = rl % G::T; rl /= G::T; }
        const int gx = b[0] * G::T + l[0], gy = b[1] * G::T + l[1], gz = D == 3 ? b[2] * G::T + l[2] : 0;
        if (loc == 0) TI.mark[blk] = 0;
        if (gx >= C.nx || gy >= C.ny || gz >= C.nz) continue;
        grid_node_at<D, FORM>(C, acc, gv, status, ((long long)gz * C.ny + gy) * C.nx + gx, gx, gy, gz);
    }
}

// The int64 sums of the marked node blocks to / from a packed array
// [block][channel][node of block] (checkpoints of the fused transfer, which
// keep the next step's grid sums). Unpacking also marks the blocks.
template <int D>
__global__ void __launch_bounds__(256) k_pack_marked(StepConsts C, TileInfo TI, int nch, int nb,
                                                     const unsigned long long* __restrict__ acc,
                                                     unsigned long long* __restrict__ out) {
    using G = TileGeom<D>;
    const long long total = (long long)nb * G::BN;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
        const int blk = TI.mark_list[w / G::BN], loc = int(w % G::BN);
        int b[3] = {0, 0, 0}, l[3] = {0, 0, 0}, rb = blk, rl = loc;
#pragma unroll
        for (int k = 0; k < D; ++k) { b[k] = rb % TI.nblk[k]; rb /= TI.nblk[k]; l[k] = rl % G::T; rl /= G::T; }
        const int gx = b[0] * G::T + l[0], gy = b[1] * G::T + l[1], gz = D == 3 ? b[2] * G::T + l[2] : 0;
        const bool in = gx < C.nx && gy < C.ny && gz < C.nz;
        const long long id = ((long long)gz * C.ny + gy) * C.nx + gx;
        for (int c = 0; c < nch; ++c) out[((w / G::BN) * nch + c) * G::BN + loc] = in ? acc[c * C.nodes + id] : 0ull;
    }
}

template <int D>
__global__ void __launch_bounds__(256) k_unpack_marked(StepConsts C, TileInfo TI, int nch, int nb,
                                                       const int* __restrict__ blocks,
                                                       const unsigned long long* __restrict__ in,
                                                       unsigned long long* __restrict__ acc) {
    using G = TileGeom<D>;
    const long long total = (long long)nb * G::BN;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
        const int blk = blocks[w / G::BN], loc = int(w % G::BN);
        if (loc == 0) {
            TI.mark[blk] = 1;
            TI.mark_list[w / G::BN] = blk;
        }
        int b[3] = {0, 0, 0}, l[3] = {0, 0, 0}, rb = blk, rl = loc;
#pragma unroll
        for (int k = 0; k < D; ++k) { b[k] = rb % TI.nblk[k]; rb /= TI.nblk[k]; l[k] = rl % G::T; rl /= G::T; }
        const int gx = b[0] * G::T + l[0], gy = b[1] * G::T + l[1], gz = D == 3 ? b[2] * G::T + l[2] : 0;
        if (gx >= C.nx || gy >= C.ny || gz >= C.nz) continue;
        const long long id = ((long long)gz * C.ny + gy) * C.nx + gx;
        for (int c = 0; c < nch; ++c) acc[c * C.nodes + id] = in[((w / G::BN) * nch + c) * G::BN + loc];
    }
}

}  // namespace mpm

namespace mpm {

// ---------------------------------------------------------------------------
// Warp-chunk P2G (MLS). The sorted slot array is cut into fixed chunks of
// WarpGeom<D, S>::CHUNK slots; each warp takes one chunk at a time, with no
// CTA-wide synchronisation. In the chunk, maximal runs of consecutive slots
// whose particles share their current stencil are grouped; SPLIT threads per
// run [3D: one per (x-offset, share of the y-offsets); 2D: one per x-offset]
// accumulate the run's S^D nodes x (1 + D) channels in FP32 registers, in slot
// order, and add them as int64 fixed point to the global sums. S is the
// stencil width: 4 (cubic) or 3 (quadratic; unused payload entries are 0). The grouping is a function of the slot order (the
// deterministic sort order, kept between sorts), so the sums are bit-identical
// run to run; particles that drifted to another cell since the last sort just
// form shorter runs.
//
// Payload per particle (float4-aligned, conflict-free for 8 distinct
// particles per load):
//   3D (36): wx[4] | wy[4] | wz[4] | yd[4] | zd[4] | m s0 s1 s2 | A00 A10 A20 A01 | A11 A21 A02 A12 | A22 pad pad pad
//            with yd[b] = wy[b] (b - 1 - fy), zd[c] = wz[c] (c - 1 - fz) and
//            s_r = m v_r - fx A_r0 (f = x - cell: the particle's offset in its cell)
//   2D (20): wx[4] | wy[4] | fx fy m mv0 | mv1 A00 A01 A10 | A11 pad pad pad
template <int D, int S = 4> struct WarpGeom;
#ifndef MPM_P2G_CHUNK3
#define MPM_P2G_CHUNK3 48
#endif
#ifndef MPM_P2G_SPLIT3
#define MPM_P2G_SPLIT3 8
#endif
// 3D: SPLIT threads per run, each holding 16 * 4 / SPLIT nodes (x-offset a,
// and 16 / SPLIT of the y-offsets) x 4 channels.
template <> struct WarpGeom<3, 4> { static constexpr int CHUNK = MPM_P2G_CHUNK3, SPLIT = MPM_P2G_SPLIT3, PS = 36; };
// 2D: MPM_P2G_SPLIT2 threads per run (1: all 16 nodes; 4: one node column each)
#ifndef MPM_P2G_SPLIT2
#define MPM_P2G_SPLIT2 4
#endif
#ifndef MPM_P2G_CHUNK2
#define MPM_P2G_CHUNK2 64
#endif
template <> struct WarpGeom<2, 4> { static constexpr int CHUNK = MPM_P2G_CHUNK2, SPLIT = MPM_P2G_SPLIT2, PS = 20; };
// quadratic: MPM_P2G_SPLIT3Q threads per run in 3D (3: one per x-offset, 9
// nodes each; 9: one per (x, y)-offset, 3 nodes each)
#ifndef MPM_P2G_CHUNK3Q
#define MPM_P2G_CHUNK3Q 48
#endif
#ifndef MPM_P2G_SPLIT3Q
#define MPM_P2G_SPLIT3Q 3
#endif
template <> struct WarpGeom<3, 3> { static constexpr int CHUNK = MPM_P2G_CHUNK3Q, SPLIT = MPM_P2G_SPLIT3Q, PS = 36; };
template <> struct WarpGeom<2, 3> {
    static constexpr int CHUNK = MPM_P2G_CHUNK2, SPLIT = MPM_P2G_SPLIT2 == 1 ? 1 : 3, PS = 20;
};
constexpr int kP2GWarps = 8;

// A particle's stencil as one word: base + 9 (>= 0) per axis in KEY_BITS-bit
// fields, so that runs compare one word and decode with shifts.
template <int D> struct StencilKey {
    static constexpr int BITS = D == 3 ? 21 : 32;
    static constexpr unsigned long long MASK = (1ull << BITS) - 1;
};
constexpr unsigned long long kNoStencil = ~0ull;

// Chunk hand-out of k_p2g_warp: a global counter (3D cubic) or round-robin.
template <int D, int S> struct P2GDynamic { static constexpr bool value = D == 3 && S == 4; };

template <int D, int S = 4> struct P2GWarpSmem {
    using W = WarpGeom<D, S>;
    float4 pay[kP2GWarps][W::CHUNK * W::PS / 4];
    unsigned long long key[kP2GWarps][W::CHUNK];  // stencil key (kNoStencil: nothing to scatter)
    int run[kP2GWarps][W::CHUNK + 1];
};

__device__ __forceinline__ void mark_block_once(const TileInfo& TI, int b) {
    if (TI.mark[b] == 0) mark_block(TI, b);
}

// int64 fixed-point add of a unit's sums; the range is checked once per unit.
__device__ __forceinline__ void red_fixed(unsigned long long* p, float v, float scale) {
    // an explicit global reduction (no return value): p always points into the
    // grid sums, and spelling it out keeps the compiler from falling back to a
    // generic atomic with a return where it cannot prove the address space
    const unsigned long long g = (unsigned long long)__cvta_generic_to_global(p);
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(g), "l"((unsigned long long)__float2ll_rn(v * scale)));
}

#ifndef MPM_P2G_MIN_BLOCKS
#define MPM_P2G_MIN_BLOCKS 3
#endif
#ifndef MPM_P2G_MIN_BLOCKS_2D
#define MPM_P2G_MIN_BLOCKS_2D 2
#endif
template <int D, int S = 4>
__global__ void __launch_bounds__(kP2GWarps * 32, D == 3 ? MPM_P2G_MIN_BLOCKS : MPM_P2G_MIN_BLOCKS_2D) k_p2g_warp(Particles P, StepConsts C, TileInfo TI,
                                                              unsigned long long* __restrict__ acc,
                                                              unsigned* __restrict__ status) {
    using W = WarpGeom<D, S>;
    using St = Stencil<S>;
    constexpr int T = TileGeom<D>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P2GWarpSmem<D, S>& SM = *reinterpret_cast<P2GWarpSmem<D, S>*>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float4* pay = SM.pay[wid];
    float* payf = reinterpret_cast<float*>(pay);
    unsigned long long* key = SM.key[wid];
    int* run = SM.run[wid];
    const int n = P.n;
    const int nchunks = (n + W::CHUNK - 1) / W::CHUNK;
    // 3D cubic: chunks are handed out one at a time from a counter, so that no
    // warp is left with a tail of chunks while others idle (-3% P2G; the sums
    // depend only on each chunk's contents, not on which warp takes it). The
    // other geometries measured faster with a fixed round-robin.
    constexpr bool kDynamic = P2GDynamic<D, S>::value;
    int chunk = blockIdx.x * kP2GWarps + wid;
    if constexpr (kDynamic) {
        if (lane == 0) chunk = atomicAdd(TI.p2g_next, 1);
        chunk = __shfl_sync(0xffffffffu, chunk, 0);
    }
    while (chunk < nchunks) {
        const int s0 = chunk * W::CHUNK;
        const int cnt = min(W::CHUNK, n - s0);
        for (int j = lane; j < cnt; j += 32) {
            const int i = s0 + j;
            const float mass = P.mass ? P.mass[i] : P.mass_u;
            const float vol = P.vol ? P.vol[i] : P.vol_u;
            if (vol == 0.f) { key[j] = kNoStencil; continue; }  // p2g.glsl:42
            float* q = payf + j * W::PS;
            unsigned long long k3 = 0;
            float f[3], mv[3];
#pragma unroll
            for (int k = D - 1; k >= 0; --k) {
                const int extk = k == 0 ? C.W : (k == 1 ? C.H : C.Dp);
                const float x = P.x[k * n + i];
                const int base = St::base(x, extk);
                float wt[S];
                St::weights(x, base, wt);
#pragma unroll
                for (int o = 0; o < 4; ++o) q[4 * k + o] = o < S ? wt[o] : 0.f;
                f[k] = x - float(base + 1);
                mv[k] = mass * P.v[k * n + i];
                k3 |= (unsigned long long)(base + 9) << (StencilKey<D>::BITS * k);  // base + 9 >= 0
            }
            if constexpr (D == 3) {
                float A[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) A[k] = P.A[k * n + i];
#pragma unroll
                for (int o = 0; o < 4; ++o) {
                    q[12 + o] = q[4 + o] * (float(o - 1) - f[1]);
                    q[16 + o] = q[8 + o] * (float(o - 1) - f[2]);
                }
                reinterpret_cast<float4*>(q)[5] =
                    make_float4(mass, mv[0] - f[0] * A[0], mv[1] - f[0] * A[3], mv[2] - f[0] * A[6]);
                reinterpret_cast<float4*>(q)[6] = make_float4(A[0], A[3], A[6], A[1]);
                reinterpret_cast<float4*>(q)[7] = make_float4(A[4], A[7], A[2], A[5]);
                reinterpret_cast<float4*>(q)[8] = make_float4(A[8], 0.f, 0.f, 0.f);
            } else {
                reinterpret_cast<float4*>(q)[2] = make_float4(f[0], f[1], mass, mv[0]);
                reinterpret_cast<float4*>(q)[3] = make_float4(mv[1], P.A[i], P.A[n + i], P.A[2 * n + i]);
                reinterpret_cast<float4*>(q)[4] = make_float4(P.A[3 * n + i], 0.f, 0.f, 0.f);
            }
            key[j] = k3;
        }
        __syncwarp();
        int nruns = 0;
        for (int j0 = 0; j0 < cnt; j0 += 32) {
            const int j = j0 + lane;
            const bool start = j < cnt && (j == 0 || key[j] != key[j - 1]);
            const unsigned b = __ballot_sync(0xffffffffu, start);
            if (start) run[nruns + __popc(b & ((1u << lane) - 1))] = j;
            nruns += __popc(b);
        }
        if (lane == 0) run[nruns] = cnt;
        __syncwarp();
        for (int u = lane; u < nruns * W::SPLIT; u += 32) {
            const int r = u / W::SPLIT, a = u % W::SPLIT;
            const int j0 = run[r], j1 = run[r + 1];
            const unsigned long long kk = key[j0];
            if (kk == kNoStencil) continue;
            int cell[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < D; ++k)  // stored base + 9; cell = base + 1
                cell[k] = int((kk >> (StencilKey<D>::BITS * k)) & StencilKey<D>::MASK) - 8;
            if constexpr (D == 3) {
                constexpr int NB = S * S / W::SPLIT;  // y-offsets per thread
                constexpr int NN = NB * S;            // nodes per thread
                const int ax = a % S, by0 = (a / S) * NB;
                float am[NN], a0[NN], a1[NN], a2[NN];
#pragma unroll
                for (int k = 0; k < NN; ++k) { am[k] = 0.f; a0[k] = 0.f; a1[k] = 0.f; a2[k] = 0.f; }
                const float da = float(ax - 1);
                for (int j = j0; j < j1; ++j) {
                    const float4* pp = pay + j * (W::PS / 4);
                    const float alpha = payf[j * W::PS + ax];
                    const float4 wy = pp[1], wz = pp[2], yd = pp[3], zd = pp[4], ms = pp[5], q6 = pp[6], q7 = pp[7];
                    const float a22 = payf[j * W::PS + 32];
                    // A = (q6.x q6.w q7.z | q6.y q7.x q7.w | q6.z q7.y a22)
                    const float ad = alpha * da;
                    const float e0 = alpha * ms.y + ad * q6.x;
                    const float e1 = alpha * ms.z + ad * q6.y;
                    const float e2 = alpha * ms.w + ad * q6.z;
                    const float f0 = alpha * q6.w, f1 = alpha * q7.x, f2 = alpha * q7.y;
                    const float g0 = alpha * q7.z, g1 = alpha * q7.w, g2 = alpha * a22;
                    const float ma = ms.x * alpha;
                    const float Z[4] = {wz.x, wz.y, wz.z, wz.w};
                    const float Zd[4] = {zd.x, zd.y, zd.z, zd.w};
                    const float Yv[4] = {wy.x, wy.y, wy.z, wy.w};
                    const float Ydv[4] = {yd.x, yd.y, yd.z, yd.w};
#pragma unroll
                    for (int bb = 0; bb < NB; ++bb) {
                        const int b = by0 + bb;
                        const float Y = NB == S ? Yv[bb] : (b == 0 ? wy.x : b == 1 ? wy.y : b == 2 ? wy.z : wy.w);
                        const float Yd = NB == S ? Ydv[bb] : (b == 0 ? yd.x : b == 1 ? yd.y : b == 2 ? yd.z : yd.w);
                        const float h0 = e0 * Y + f0 * Yd, h1 = e1 * Y + f1 * Yd, h2 = e2 * Y + f2 * Yd;
                        const float k0 = g0 * Y, k1 = g1 * Y, k2 = g2 * Y, mY = ma * Y;
#pragma unroll
                        for (int cc = 0; cc < S; ++cc) {
                            const int idx = bb * S + cc;
                            am[idx] += mY * Z[cc];
                            a0[idx] += h0 * Z[cc] + k0 * Zd[cc];
                            a1[idx] += h1 * Z[cc] + k1 * Zd[cc];
                            a2[idx] += h2 * Z[cc] + k2 * Zd[cc];
                        }
                    }
                }
                float mx_m = 0.f, mx_p = 0.f;
#pragma unroll
                for (int k = 0; k < NN; ++k) {
                    mx_m = fmaxf(mx_m, fabsf(am[k]));
                    mx_p = fmaxf(mx_p, fmaxf(fabsf(a0[k]), fmaxf(fabsf(a1[k]), fabsf(a2[k]))));
                }
                if (!(mx_m * C.sm < kFixedLimit && mx_p * C.sp < kFixedLimit))
                    raise_flag(status, (mx_m != mx_m || mx_p != mx_p) ? 1u : 2u);
                const int gx = cell[0] - 1 + ax;
                const bool inside = gx >= 0 && gx <= C.W && cell[1] >= 1 && cell[1] + (S - 2) <= C.H &&
                                    cell[2] >= 1 && cell[2] + (S - 2) <= C.Dp;
                if (inside) {
                    const long long g0 = ((long long)(cell[2] - 1) * C.ny + (cell[1] - 1 + by0)) * C.nx + gx;
                    const long long sy = C.nx, sz = (long long)C.nx * C.ny;
#pragma unroll
                    for (int bb = 0; bb < NB; ++bb)
#pragma unroll
                        for (int cc = 0; cc < S; ++cc) {
                            const int idx = bb * S + cc;
                            unsigned long long* p0 = acc + (g0 + bb * sy + cc * sz);
                            red_fixed(p0, am[idx], C.sm);
                            red_fixed(p0 + C.nodes, a0[idx], C.sp);
                            red_fixed(p0 + 2 * C.nodes, a1[idx], C.sp);
                            red_fixed(p0 + 3 * C.nodes, a2[idx], C.sp);
                        }
                } else {
                    bool outside = false;
                    for (int bb = 0; bb < NB; ++bb)
                        for (int cc = 0; cc < S; ++cc) {
                            const int gy = cell[1] - 1 + by0 + bb, gz = cell[2] - 1 + cc;
                            if (gx < 0 || gx > C.W || gy < 0 || gy > C.H || gz < 0 || gz > C.Dp) { outside = true; continue; }
                            const int idx = bb * S + cc;
                            unsigned long long* p0 = acc + (((long long)gz * C.ny + gy) * C.nx + gx);
                            red_fixed(p0, am[idx], C.sm);
                            red_fixed(p0 + C.nodes, a0[idx], C.sp);
                            red_fixed(p0 + 2 * C.nodes, a1[idx], C.sp);
                            red_fixed(p0 + 3 * C.nodes, a2[idx], C.sp);
                        }
                    if (outside) raise_flag(status, 4u);
                }
                if (gx >= 0 && gx <= C.W) {
                    // node blocks holding the thread's in-grid nodes (empty range: none)
                    const int y0 = max(0, cell[1] - 1 + by0), y1 = min(C.H, cell[1] - 2 + by0 + NB);
                    const int z0 = max(0, cell[2] - 1), z1 = min(C.Dp, cell[2] + (S - 2));
                    if (y0 <= y1 && z0 <= z1)
                        for (int bz = z0 / T; bz <= z1 / T; ++bz)
                            for (int by = y0 / T; by <= y1 / T; ++by)
                                mark_block_once(TI, (bz * TI.nblk[1] + by) * TI.nblk[0] + gx / T);
                }
            } else {
                // 2D: SPLIT threads per run, each holding NA = S / SPLIT x-offsets
                // (all S y-offsets) x 3 channels
                constexpr int NA = S / W::SPLIT;
                const int gx0 = cell[0] - 1 + a * NA;  // first node column of this thread
                float am[NA * S], a0[NA * S], a1[NA * S];
#pragma unroll
                for (int k = 0; k < NA * S; ++k) { am[k] = 0.f; a0[k] = 0.f; a1[k] = 0.f; }
                for (int j = j0; j < j1; ++j) {
                    const float4* pp = pay + j * (W::PS / 4);
                    const float4 wx = pp[0], wy = pp[1], p2 = pp[2], p3 = pp[3], p4 = pp[4];
                    // f = (p2.x, p2.y), m = p2.z, mv = (p2.w, p3.x), A = (p3.y p3.z | p3.w p4.x)
                    const float Xv[4] = {wx.x, wx.y, wx.z, wx.w};
                    const float Y[4] = {wy.x, wy.y, wy.z, wy.w};
                    float Yd[4];
#pragma unroll
                    for (int b = 0; b < S; ++b) Yd[b] = Y[b] * (float(b - 1) - p2.y);
#pragma unroll
                    for (int i = 0; i < NA; ++i) {
                        const int aa = a * NA + i;
                        const float X = NA == S ? Xv[i] : payf[j * W::PS + aa];
                        const float Xd = X * (float(aa - 1) - p2.x);
                        const float e0 = p2.w * X + p3.y * Xd, e1 = p3.x * X + p3.w * Xd;
                        const float f0 = p3.z * X, f1 = p4.x * X, mX = p2.z * X;
#pragma unroll
                        for (int b = 0; b < S; ++b) {
                            const int idx = i * S + b;
                            am[idx] += mX * Y[b];
                            a0[idx] += e0 * Y[b] + f0 * Yd[b];
                            a1[idx] += e1 * Y[b] + f1 * Yd[b];
                        }
                    }
                }
                float mx_m = 0.f, mx_p = 0.f;
#pragma unroll
                for (int k = 0; k < NA * S; ++k) {
                    mx_m = fmaxf(mx_m, fabsf(am[k]));
                    mx_p = fmaxf(mx_p, fmaxf(fabsf(a0[k]), fabsf(a1[k])));
                }
                if (!(mx_m * C.sm < kFixedLimit && mx_p * C.sp < kFixedLimit))
                    raise_flag(status, (mx_m != mx_m || mx_p != mx_p) ? 1u : 2u);
                const bool inside = gx0 >= 0 && gx0 + (NA - 1) <= C.W && cell[1] >= 1 && cell[1] + (S - 2) <= C.H;
                if (inside) {
                    const long long g0 = (long long)(cell[1] - 1) * C.nx + gx0;
#pragma unroll
                    for (int i = 0; i < NA; ++i)
#pragma unroll
                        for (int b = 0; b < S; ++b) {
                            const int idx = i * S + b;
                            unsigned long long* p0 = acc + (g0 + i + (long long)b * C.nx);
                            red_fixed(p0, am[idx], C.sm);
                            red_fixed(p0 + C.nodes, a0[idx], C.sp);
                            red_fixed(p0 + 2 * C.nodes, a1[idx], C.sp);
                        }
                } else {
                    bool outside = false;
                    for (int i = 0; i < NA; ++i)
                        for (int b = 0; b < S; ++b) {
                            const int gx = gx0 + i, gy = cell[1] - 1 + b;
                            if (gx < 0 || gx > C.W || gy < 0 || gy > C.H) { outside = true; continue; }
                            const int idx = i * S + b;
                            unsigned long long* p0 = acc + ((long long)gy * C.nx + gx);
                            red_fixed(p0, am[idx], C.sm);
                            red_fixed(p0 + C.nodes, a0[idx], C.sp);
                            red_fixed(p0 + 2 * C.nodes, a1[idx], C.sp);
                        }
                    if (outside) raise_flag(status, 4u);
                }
                const int x0 = max(0, gx0), x1 = min(C.W, gx0 + (NA - 1));
                const int y0 = max(0, cell[1] - 1), y1 = min(C.H, cell[1] + (S - 2));
                if (x0 <= x1 && y0 <= y1)
                    for (int by = y0 / T; by <= y1 / T; ++by)
                        for (int bx = x0 / T; bx <= x1 / T; ++bx) mark_block_once(TI, by * TI.nblk[0] + bx);
            }
        }
        __syncwarp();
        if constexpr (kDynamic) {
            if (lane == 0) chunk = atomicAdd(TI.p2g_next, 1);
            chunk = __shfl_sync(0xffffffffu, chunk, 0);
        } else {
            chunk += gridDim.x * kP2GWarps;
        }
    }
}

}  // namespace mpm
