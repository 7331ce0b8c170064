// Batched 2D scenes: many independent MLS scenes of uneven size in one
// persistent launch per cluster size.
//
// Each scene runs on a thread-block cluster of 1, 2, 4 or 8 CTAs that holds the
// scene's whole grid in distributed shared memory: node rows are cut into
// bands, one per CTA, three int64 fixed-point accumulators per node (mass,
// momentum x, momentum y; 24 bytes, so a 257 x 257 grid fits in 8 CTAs). A
// step is
//   P2G   each CTA scatters its particles into the owning CTAs' shared memory
//         (red.shared::cluster.add.u64)
//   grid  each CTA turns its own band into velocities (vf, vc) in place
//   G2P   each CTA gathers its particles' stencils from the owning CTAs
//         (ld.shared::cluster), updates them and the return map, and writes
//         the next step's affine matrix
// with a cluster barrier between phases. No grid touches HBM and no global
// atomics are issued; particle state streams through HBM once per phase.
//
// Every sort_period steps a multi-CTA cluster counting-sorts its scene's
// particles by cell row into the second particle buffer and re-cuts the bands
// so that each CTA holds about n / cl particles and the rows they touch
// (within its shared-memory capacity): most scatter and gather traffic then
// stays in the CTA's own shared memory. The per-particle arithmetic is that
// of the single-scene kernels (the same device functions) and the int64 sums
// are exact, so a scene's result depends neither on its cluster size, nor on
// the particle order, nor on the other scenes of the batch.
//
// Clusters are persistent: each takes scenes from an atomic queue (most
// expensive first) and runs all requested steps of one scene before taking
// the next.
#pragma once

#include <cooperative_groups.h>

#include "mpm_kernels.cuh"

namespace mpm {

namespace cg = cooperative_groups;

constexpr int kBatchMaxCluster = 8;
constexpr int kBatchAccs = 3;         // mass, momentum x, momentum y
constexpr int kBatchMaxRows = 512;    // node rows of one scene

struct BatchScene {
    StepConsts C;
    long long p0;  // first particle slot of the scene
    int n;         // particles
    int cl;        // CTAs of the scene's cluster
    int rows;      // most node rows one CTA can hold (shared-memory capacity / nx)
    int pad;
};

// Per-scene state that persists between launches.
struct BatchSceneState {
    int parity;                      // which particle buffer holds the scene
    int step;                        // steps taken since creation (or the last state upload)
    int sorted;                      // the bands below are valid
    int pad;
    int cut[kBatchMaxCluster + 1];   // band b holds node rows [cut[b], cut[b+1])
    int off[kBatchMaxCluster + 1];   // and particles [p0 + off[b], p0 + off[b+1])
};

struct BatchBuffers {
    float* x;
    float* v;
    float* B;
    float* Fe;
    float* Jp;
    float* A;  // P2G affine matrix of the next step (written by G2P)
    float* mass;
    float* vol;
    int* id;   // creation index of the particle within its scene
};

struct BatchParticles {
    BatchBuffers buf[2];
    long long N;  // component stride of the SoA arrays
};

struct BatchRun {
    const BatchScene* scenes;
    BatchSceneState* state;
    const int* order;            // this class's scenes, most expensive first
    int count;                   // scenes in this class
    int cap;                     // nodes per accumulator array in each CTA
    int* queue;                  // next work item; zero before the launch
    int* needs_affine;           // per scene: derive A from (B, F_E, J_p) first
    unsigned* status;            // per scene: MPM_FLAG_* bits
    unsigned long long* stamps;  // per scene: steps + 1 device timestamps (ns), or null
    int steps;
    int sort_period;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Address of the same shared-memory offset in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_map(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

// Each shared::cluster access carries a "memory" clobber so that the compiler
// keeps it on its side of the cluster barriers (which order the phases).
__device__ __forceinline__ void cluster_red_add(uint32_t addr, long long v) {
    if (v != 0)
        asm volatile("red.relaxed.cluster.shared::cluster.add.u64 [%0], %1;" ::"r"(addr), "l"((unsigned long long)v)
                     : "memory");
}

__device__ __forceinline__ void cluster_red_add_u32(uint32_t addr, unsigned v) {
    asm volatile("red.relaxed.cluster.shared::cluster.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned cluster_atom_add_u32(uint32_t addr, unsigned v) {
    unsigned old;
    asm volatile("atom.relaxed.cluster.shared::cluster.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(addr), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ unsigned cluster_ld_u32(uint32_t addr) {
    unsigned r;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(r) : "r"(addr) : "memory");
    return r;
}

__device__ __forceinline__ float2 cluster_ld_f2(uint32_t addr) {
    float2 r;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(r.x), "=f"(r.y) : "r"(addr) : "memory");
    return r;
}

__device__ __forceinline__ unsigned long long device_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long pack_f2(float lo, float hi) {
    return (unsigned long long)__float_as_uint(lo) | ((unsigned long long)__float_as_uint(hi) << 32);
}

// Node row -> (owning CTA, offset of the row in that CTA's arrays).
struct BatchRowMap {
    const unsigned char* owner;
    const int* base;  // (row - first row of the band) * nx
};

// P2G of particles [lo, hi) of one scene (MLS, src/gpu/shaders/2d/p2g.glsl:29-92):
//   m_i += w m_p,  p_i += w (m_p v_p + A_p (x_i - x_p)),  int64 fixed point.
template <int THREADS>
__device__ __forceinline__ void batch_p2g(const BatchBuffers& P, long long N, const StepConsts& C, long long lo,
                                          long long hi, const BatchRowMap& M, uint32_t g0, int cap,
                                          unsigned* status) {
    for (long long i = lo + threadIdx.x; i < hi; i += THREADS) {
        const float vol = P.vol[i];
        if (vol == 0.f) continue;
        const float x[2] = {P.x[i], P.x[N + i]};
        const float mass = P.mass[i];
        const float mv[2] = {mass * P.v[i], mass * P.v[N + i]};
        float A[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) A[k] = P.A[k * N + i];
        const int ext[2] = {C.W, C.H};
        int base[2];
        float wk[2][4], off[2][4];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            base[k] = stencil_base(x[k], ext[k]);
            Stencil<4>::weights(x[k], base[k], wk[k]);
#pragma unroll
            for (int o = 0; o < 4; ++o) off[k][o] = float(base[k] + o) - x[k];
        }
        bool outside = false;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int iy = base[1] + b;
            if (iy < 0 || iy > C.H) { outside = true; continue; }
            const uint32_t row = cluster_map(g0, M.owner[iy]) + 8u * (uint32_t)M.base[iy];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int ix = base[0] + a;
                if (ix < 0 || ix > C.W) { outside = true; continue; }
                const float w = wk[0][a] * wk[1][b];
                const float d[2] = {off[0][a], off[1][b]};
                const uint32_t at = row + 8u * (uint32_t)ix;
                cluster_red_add(at, to_fixed(w * mass, C.sm, status));
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    float s = mv[r];
#pragma unroll
                    for (int k = 0; k < 2; ++k) s += A[r * 2 + k] * d[k];
                    cluster_red_add(at + 8u * (uint32_t)((1 + r) * cap), to_fixed(w * s, C.sp, status));
                }
            }
        }
        if (outside) raise_flag(status, 4u);
    }
}

// G2P + APIC + return map of particles [lo, hi) (src/gpu/shaders/2d/g2p.glsl:
// 21-93), the arithmetic of k_g2p_simple, then the next step's affine matrix.
template <int THREADS>
__device__ __forceinline__ void batch_g2p(const BatchBuffers& P, long long N, const StepConsts& C, long long lo,
                                          long long hi, const BatchRowMap& M, uint32_t g0, int cap,
                                          unsigned* status) {
    for (long long i = lo + threadIdx.x; i < hi; i += THREADS) {
        const float x[2] = {P.x[i], P.x[N + i]};
        // the rest of the particle's state, loaded before the gather so that
        // its latency overlaps the stencil reads
        float Fe[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) Fe[k] = P.Fe[k * N + i];
        float Jp = P.Jp[i];
        const float mass = P.mass[i], vol = P.vol[i];
        const int ext[2] = {C.W, C.H};
        int base[2];
        float wk[2][4], off[2][4];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            base[k] = stencil_base(x[k], ext[k]);
            Stencil<4>::weights(x[k], base[k], wk[k]);
#pragma unroll
            for (int o = 0; o < 4; ++o) off[k][o] = float(base[k] + o) - x[k];
        }
        uint32_t row[4];
        bool row_in[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int iy = base[1] + b;
            row_in[b] = iy >= 0 && iy <= C.H;
            const int r = row_in[b] ? iy : 0;
            row[b] = cluster_map(g0, M.owner[r]) + 8u * (uint32_t)M.base[r];
        }
        float nv[2] = {0.f, 0.f}, nxp[2] = {0.f, 0.f}, nB[4] = {0.f, 0.f, 0.f, 0.f};
        float wsum = 0.f;
        bool clipped = false;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int ix = base[0] + a;
            if (ix < 0 || ix > C.W) { clipped = true; continue; }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (!row_in[b]) { clipped = true; continue; }
                const uint32_t at = row[b] + 8u * (uint32_t)ix;
                const float2 gf = cluster_ld_f2(at);
                const float2 gc = cluster_ld_f2(at + 8u * (uint32_t)cap);
                const float vf[2] = {gf.x, gf.y}, vc[2] = {gc.x, gc.y};
                const float w = wk[0][a] * wk[1][b];
                const float d[2] = {off[0][a], off[1][b]};
                wsum += w;
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    nv[r] += vf[r] * w;
#pragma unroll
                    for (int k = 0; k < 2; ++k) nB[r * 2 + k] += w * (vf[r] * d[k]);
                    nxp[r] += (d[r] + C.dt * vc[r]) * w;
                }
            }
        }
        bool finite = true;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const float xn = (clipped ? x[k] * wsum : x[k]) + nxp[k];
            P.v[k * N + i] = nv[k];
            P.x[k * N + i] = xn;
            finite = finite && isfinite(xn);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) P.B[k * N + i] = nB[k];
        float L[4], Fh[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) L[k] = ((k % 3) == 0 ? 1.f : 0.f) + C.dt * (3.f * nB[k]);
        matmul<2>(L, Fe, Fh);
        plasticity<2, kMLS>(C, Fh, Fe, Jp, status);
        float Anext[4];
        mls_affine<2>(C, nB, Fe, Jp, mass, vol, Anext);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            P.Fe[k * N + i] = Fe[k];
            P.A[k * N + i] = Anext[k];
        }
        P.Jp[i] = Jp;
        if (!finite || !isfinite(Jp)) raise_flag(status, 1u);
    }
}

__device__ __forceinline__ int cell_row(float y, int H) { return min(max(int(fmaxf(y, 0.f)), 0), H); }

// Counting sort of one scene's particles by cell row, from buffer `src` to
// `dst`, and new bands: cut rows balance the particle count per CTA subject to
// at most `max_rows` rows per CTA. Runs on every CTA of the cluster; the
// scratch is CTA 0's first accumulator array (all-zero on entry and on exit).
// s_cut / s_off (shared, every CTA) receive the bands.
template <int THREADS>
__device__ void batch_sort(const BatchParticles& P, int src, const BatchScene& S, int max_rows, unsigned rank,
                           unsigned cl, long long lo, long long hi, unsigned long long* a0, int* s_cut, int* s_off,
                           cg::cluster_group& cluster) {
    const int tid = threadIdx.x;
    const int ny = S.C.ny;
    unsigned* hist = reinterpret_cast<unsigned*>(a0);  // rows counts, then row cursors (CTA 0)
    const uint32_t hist0 = cluster_map(smem_addr(hist), 0);
    const BatchBuffers& F = P.buf[src];
    const BatchBuffers& T = P.buf[src ^ 1];
    const long long N = P.N;
    for (long long i = lo + tid; i < hi; i += THREADS)
        cluster_red_add_u32(hist0 + 4u * (uint32_t)cell_row(F.x[N + i], S.C.H), 1u);
    cluster.sync();
    if (rank == 0) {
        // exclusive prefix over rows (one warp), then the cuts (one thread)
        if (tid < 32) {
            const int per = (ny + 31) / 32, r0 = tid * per, r1 = min(ny, r0 + per);
            unsigned run = 0;
            for (int r = r0; r < r1; ++r) run += hist[r];
            unsigned incl = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += t;
            }
            unsigned acc = incl - run;
            for (int r = r0; r < r1; ++r) {
                const unsigned c = hist[r];
                hist[r] = acc;
                acc += c;
            }
        }
        __syncthreads();
        if (tid == 0) {
            const long long n = S.n;
            int start = 0;
            s_cut[0] = 0;
            s_off[0] = 0;
            for (unsigned b = 0; b < cl; ++b) {
                int end;
                if (b + 1 == cl) {
                    end = ny;
                } else {
                    const long long target = n * (b + 1) / cl;
                    // first row whose start offset reaches the target
                    int lo_r = start, hi_r = ny;
                    while (lo_r < hi_r) {
                        const int mid = (lo_r + hi_r) >> 1;
                        if ((long long)hist[mid] >= target) hi_r = mid;
                        else lo_r = mid + 1;
                    }
                    end = lo_r;
                    const int rest = (int)(cl - b - 1);
                    end = max(end, ny - rest * max_rows);  // the remaining CTAs must hold the rest
                    end = min(end, start + max_rows);
                    end = max(end, start);
                    end = min(end, ny);
                }
                s_cut[b + 1] = end;
                s_off[b + 1] = end < ny ? (int)hist[end] : S.n;
                start = end;
            }
        }
    }
    cluster.sync();
    if (rank != 0 && tid <= (int)cl) {
        s_cut[tid] = (int)cluster_ld_u32(cluster_map(smem_addr(s_cut + tid), 0));
        s_off[tid] = (int)cluster_ld_u32(cluster_map(smem_addr(s_off + tid), 0));
    }
    // scatter: slot = row start + arrival order within the row
    for (long long i = lo + tid; i < hi; i += THREADS) {
        const float y = F.x[N + i];
        const long long j = S.p0 + cluster_atom_add_u32(hist0 + 4u * (uint32_t)cell_row(y, S.C.H), 1u);
        T.x[j] = F.x[i];
        T.x[N + j] = y;
#pragma unroll
        for (int k = 0; k < 2; ++k) T.v[k * N + j] = F.v[k * N + i];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            T.B[k * N + j] = F.B[k * N + i];
            T.Fe[k * N + j] = F.Fe[k * N + i];
            T.A[k * N + j] = F.A[k * N + i];
        }
        T.Jp[j] = F.Jp[i];
        T.mass[j] = F.mass[i];
        T.vol[j] = F.vol[i];
        T.id[j] = F.id[i];
    }
    cluster.sync();
    if (rank == 0)
        for (int r = tid; r < ny; r += THREADS) hist[r] = 0u;
    // the next cluster barrier (before any use of the arrays) orders this clear
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_batch_run(BatchParticles P, BatchRun R) {
    extern __shared__ __align__(16) unsigned long long sgrid[];
    __shared__ int s_item, s_parity, s_step0, s_sorted;
    __shared__ int s_cut[kBatchMaxCluster + 1], s_off[kBatchMaxCluster + 1];
    __shared__ unsigned char s_owner[kBatchMaxRows];
    __shared__ int s_base[kBatchMaxRows];
    __shared__ StepConsts sC;
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank(), cl = cluster.num_blocks();
    const int tid = threadIdx.x;
    const int cap = R.cap;
    unsigned long long* a0 = sgrid;
    unsigned long long* a1 = sgrid + cap;
    unsigned long long* a2 = sgrid + 2 * (long long)cap;
    const uint32_t g0 = smem_addr(sgrid);
    const BatchRowMap M{s_owner, s_base};
    // the accumulators are all-zero between steps; start from there
    for (int j = tid; j < kBatchAccs * cap; j += THREADS) sgrid[j] = 0ull;
    for (;;) {
        if (rank == 0 && tid == 0) s_item = atomicAdd(R.queue, 1);
        cluster.sync();
        const int item = *cluster.map_shared_rank(&s_item, 0);
        cluster.sync();  // every CTA has read the item before CTA 0 may change it or exit
        if (item >= R.count) break;
        const int sc = R.order[item];
        const BatchScene& S = R.scenes[sc];
        BatchSceneState& G = R.state[sc];
        if (tid == 0) {
            sC = S.C;
            s_parity = G.parity;
            s_step0 = G.step;
            s_sorted = G.sorted;
        }
        if (tid <= (int)cl) {
            s_cut[tid] = G.cut[tid];
            s_off[tid] = G.off[tid];
        }
        __syncthreads();
        if (tid == 0 && s_sorted) {
            // stored bands are used only if they partition this scene for this cluster size
            bool ok = s_cut[0] == 0 && s_cut[cl] == S.C.ny && s_off[0] == 0 && s_off[cl] == S.n;
            for (unsigned b = 0; b < cl; ++b)
                ok = ok && s_cut[b] <= s_cut[b + 1] && s_cut[b + 1] - s_cut[b] <= S.rows && s_off[b] <= s_off[b + 1];
            if (!ok) s_sorted = 0;
        }
        __syncthreads();
        const StepConsts& C = sC;
        unsigned* status = R.status + sc;
        const int nx = C.nx, ny = C.ny;
        int parity = s_parity;
        const bool banded = cl > 1;
        if (!banded || !s_sorted) {
            // equal bands of rows and of particles, until the first sort
            if (tid <= (int)cl) {
                s_cut[tid] = min(ny, tid * ((ny + (int)cl - 1) / (int)cl));
                s_off[tid] = (int)((long long)S.n * tid / cl);
            }
            __syncthreads();
        }
        if (R.needs_affine[sc]) {
            const BatchBuffers& F = P.buf[parity];
            const long long lo = S.p0 + s_off[rank], hi = S.p0 + s_off[rank + 1];
            for (long long i = lo + tid; i < hi; i += THREADS) {
                float B[4], Fe[4], A[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) { B[k] = F.B[k * P.N + i]; Fe[k] = F.Fe[k * P.N + i]; }
                mls_affine<2>(C, B, Fe, F.Jp[i], F.mass[i], F.vol[i], A);
#pragma unroll
                for (int k = 0; k < 4; ++k) F.A[k * P.N + i] = A[k];
            }
        }
        unsigned long long* stamp = R.stamps ? R.stamps + (long long)sc * (R.steps + 1) : nullptr;
        if (stamp && rank == 0 && tid == 0) stamp[0] = device_ns();
        bool sorted = s_sorted != 0;
        for (int step = 0; step < R.steps; ++step) {
            if (banded && (!sorted || (R.sort_period > 0 && (s_step0 + step) % R.sort_period == 0))) {
                cluster.sync();  // A of every particle is written before it moves
                batch_sort<THREADS>(P, parity, S, S.rows, rank, cl, S.p0 + s_off[rank], S.p0 + s_off[rank + 1],
                                    a0, s_cut, s_off, cluster);
                parity ^= 1;
                sorted = true;
            }
            if (step == 0 || banded) {
                // row -> (owner, offset) for the current bands
                for (int r = tid; r < ny; r += THREADS) {
                    int b = 0;
                    while (b + 1 < (int)cl && r >= s_cut[b + 1]) ++b;
                    s_owner[r] = (unsigned char)b;
                    s_base[r] = (r - s_cut[b]) * nx;
                }
            }
            cluster.sync();
            const BatchBuffers& F = P.buf[parity];
            const long long lo = S.p0 + s_off[rank], hi = S.p0 + s_off[rank + 1];
            const int row0 = s_cut[rank];
            const int my_nodes = (s_cut[rank + 1] - row0) * nx;
            batch_p2g<THREADS>(F, P.N, C, lo, hi, M, g0, cap, status);
            cluster.sync();
            for (int j = tid; j < my_nodes; j += THREADS) {
                const long long q[3] = {(long long)a0[j], (long long)a1[j], (long long)a2[j]};
                const int iy = row0 + j / nx, ix = j - (j / nx) * nx;
                float vc[3], vf[3];
                grid_node_velocity<2, kMLS>(C, q, ix, iy, 0, status, vc, vf);
                a0[j] = pack_f2(vf[0], vf[1]);
                a1[j] = pack_f2(vc[0], vc[1]);
                a2[j] = 0ull;
            }
            cluster.sync();
            batch_g2p<THREADS>(F, P.N, C, lo, hi, M, g0, cap, status);
            cluster.sync();
            for (int j = tid; j < my_nodes; j += THREADS) { a0[j] = 0ull; a1[j] = 0ull; }
            if (stamp && rank == 0 && tid == 0) stamp[step + 1] = device_ns();
        }
        cluster.sync();  // the arrays are clear and every CTA is done with the scene
        if (rank == 0 && tid == 0) {
            R.needs_affine[sc] = 0;
            G.parity = parity;
            G.step = s_step0 + R.steps;
            G.sorted = sorted ? 1 : 0;
        }
        if (rank == 0 && tid <= (int)cl) {
            G.cut[tid] = s_cut[tid];
            G.off[tid] = s_off[tid];
        }
    }
}

}  // namespace mpm
