// Batched 2D scenes: many independent MLS scenes of uneven size in one
// persistent launch per cluster size.
//
// Each scene runs on a thread-block cluster of 1, 2, 4 or 8 CTAs that holds the
// scene's whole grid in distributed shared memory: node rows are split in
// bands across the cluster's CTAs, three int64 fixed-point accumulators per
// node (mass, momentum x, momentum y; 24 bytes, so a 257 x 257 grid fits in 8
// CTAs). A step is
//   P2G   each CTA scatters its slice of the scene's particles into the
//         owning CTAs' shared memory (red.shared::cluster.add.u64)
//   grid  each CTA turns its own node band into velocities (vf, vc) in place
//   G2P   each CTA gathers its particles' stencils from the owning CTAs
//         (ld.shared::cluster), updates them and the return map, and writes
//         the next step's affine matrix
// with a cluster barrier between phases. No grid touches HBM and no global
// atomics are issued; particle state streams through HBM once per phase.
// The per-particle arithmetic is that of the single-scene kernels (the same
// device functions), and the int64 sums are exact, so a scene's result does
// not depend on its cluster size or on the other scenes of the batch.
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
constexpr int kBatchAccs = 3;  // mass, momentum x, momentum y

struct BatchScene {
    StepConsts C;
    long long p0;  // first particle slot of the scene
    int n;         // particles
    int cl;        // CTAs of the scene's cluster
    int rows;      // node rows held by each CTA
    int pad;
};

struct BatchParticles {
    float* x;
    float* v;
    float* B;
    float* Fe;
    float* Jp;
    float* A;  // P2G affine matrix of the next step (written by G2P)
    const float* mass;
    const float* vol;
    long long N;  // component stride of the SoA arrays
};

struct BatchRun {
    const BatchScene* scenes;
    const int* order;          // this class's scenes, most expensive first
    int count;                 // scenes in this class
    int cap;                   // nodes per accumulator array in each CTA
    int* queue;                // next work item; zero before the launch
    int* needs_affine;         // per scene: derive A from (B, F_E, J_p) first
    unsigned* status;          // per scene: MPM_FLAG_* bits
    unsigned long long* stamps;  // per scene: steps + 1 device timestamps (ns), or null
    int steps;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Address of the same shared-memory offset in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_map(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_red_add(uint32_t addr, long long v) {
    if (v != 0)
        asm volatile("red.relaxed.cluster.shared::cluster.add.u64 [%0], %1;" ::"r"(addr), "l"((unsigned long long)v)
                     : "memory");
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

// P2G of particles [lo, hi) of one scene (MLS, src/gpu/shaders/2d/p2g.glsl:29-92):
//   m_i += w m_p,  p_i += w (m_p v_p + A_p (x_i - x_p)),  int64 fixed point.
template <int THREADS>
__device__ __forceinline__ void batch_p2g(const BatchParticles& P, const StepConsts& C, long long lo, long long hi,
                                          int rows, uint32_t g0, int cap, unsigned* status) {
    const int nx = C.nx;
    for (long long i = lo + threadIdx.x; i < hi; i += THREADS) {
        const float vol = P.vol[i];
        if (vol == 0.f) continue;
        const float x[2] = {P.x[i], P.x[P.N + i]};
        const float mass = P.mass[i];
        const float mv[2] = {mass * P.v[i], mass * P.v[P.N + i]};
        float A[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) A[k] = P.A[k * P.N + i];
        const int ext[2] = {C.W, C.H};
        int base[2];
        float wk[2][4], off[2][4];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            base[k] = stencil_base(x[k], ext[k]);
#pragma unroll
            for (int o = 0; o < 4; ++o) {
                const float dist = x[k] - float(base[k] + o);
                wk[k][o] = bspline_n(dist);
                off[k][o] = -dist;
            }
        }
        bool outside = false;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int iy = base[1] + b;
            if (iy < 0 || iy > C.H) { outside = true; continue; }
            const int owner = iy / rows;
            const uint32_t row = cluster_map(g0, owner) + 8u * (uint32_t)((iy - owner * rows) * nx);
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
__device__ __forceinline__ void batch_g2p(const BatchParticles& P, const StepConsts& C, long long lo, long long hi,
                                          int rows, uint32_t g0, int cap, unsigned* status) {
    const int nx = C.nx;
    for (long long i = lo + threadIdx.x; i < hi; i += THREADS) {
        const float x[2] = {P.x[i], P.x[P.N + i]};
        const int ext[2] = {C.W, C.H};
        int base[2];
        float wk[2][4], off[2][4];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            base[k] = stencil_base(x[k], ext[k]);
#pragma unroll
            for (int o = 0; o < 4; ++o) {
                const float dist = x[k] - float(base[k] + o);
                wk[k][o] = bspline_n(dist);
                off[k][o] = -dist;
            }
        }
        uint32_t row[4];
        bool row_in[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int iy = base[1] + b;
            row_in[b] = iy >= 0 && iy <= C.H;
            const int owner = row_in[b] ? iy / rows : 0;
            row[b] = cluster_map(g0, owner) + 8u * (uint32_t)((row_in[b] ? iy - owner * rows : 0) * nx);
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
            P.v[k * P.N + i] = nv[k];
            P.x[k * P.N + i] = xn;
            finite = finite && isfinite(xn);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) P.B[k * P.N + i] = nB[k];
        float Fe[4], L[4], Fh[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            Fe[k] = P.Fe[k * P.N + i];
            L[k] = ((k % 3) == 0 ? 1.f : 0.f) + C.dt * (3.f * nB[k]);
        }
        matmul<2>(L, Fe, Fh);
        float Jp = P.Jp[i];
        plasticity<2, kMLS>(C, Fh, Fe, Jp, status);
        float Anext[4];
        mls_affine<2>(C, nB, Fe, Jp, P.mass[i], P.vol[i], Anext);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            P.Fe[k * P.N + i] = Fe[k];
            P.A[k * P.N + i] = Anext[k];
        }
        P.Jp[i] = Jp;
        if (!finite || !isfinite(Jp)) raise_flag(status, 1u);
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_batch_run(BatchParticles P, BatchRun R) {
    extern __shared__ __align__(16) unsigned long long sgrid[];
    __shared__ int s_item;
    __shared__ StepConsts sC;
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank(), cl = cluster.num_blocks();
    const int tid = threadIdx.x;
    const int cap = R.cap;
    unsigned long long* a0 = sgrid;
    unsigned long long* a1 = sgrid + cap;
    unsigned long long* a2 = sgrid + 2 * (long long)cap;
    const uint32_t g0 = smem_addr(sgrid);
    for (;;) {
        if (rank == 0 && tid == 0) s_item = atomicAdd(R.queue, 1);
        cluster.sync();
        const int item = *cluster.map_shared_rank(&s_item, 0);
        cluster.sync();  // every CTA has read the item before CTA 0 may change it or exit
        if (item >= R.count) break;
        const int sc = R.order[item];
        const BatchScene& S = R.scenes[sc];
        if (tid == 0) sC = S.C;
        __syncthreads();
        const StepConsts& C = sC;
        unsigned* status = R.status + sc;
        const int rows = S.rows, nx = C.nx;
        const int row0 = (int)rank * rows;
        const int my_rows = max(0, min(C.ny - row0, rows));
        const int my_nodes = my_rows * nx;
        const long long lo = S.p0 + (long long)S.n * rank / cl, hi = S.p0 + (long long)S.n * (rank + 1) / cl;
        for (int j = tid; j < my_nodes; j += THREADS) { a0[j] = 0ull; a1[j] = 0ull; a2[j] = 0ull; }
        if (R.needs_affine[sc]) {
            for (long long i = lo + tid; i < hi; i += THREADS) {
                float B[4], Fe[4], A[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) { B[k] = P.B[k * P.N + i]; Fe[k] = P.Fe[k * P.N + i]; }
                mls_affine<2>(C, B, Fe, P.Jp[i], P.mass[i], P.vol[i], A);
#pragma unroll
                for (int k = 0; k < 4; ++k) P.A[k * P.N + i] = A[k];
            }
        }
        cluster.sync();
        unsigned long long* stamp = R.stamps ? R.stamps + (long long)sc * (R.steps + 1) : nullptr;
        if (stamp && rank == 0 && tid == 0) stamp[0] = device_ns();
        for (int step = 0; step < R.steps; ++step) {
            batch_p2g<THREADS>(P, C, lo, hi, rows, g0, cap, status);
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
            batch_g2p<THREADS>(P, C, lo, hi, rows, g0, cap, status);
            cluster.sync();
            for (int j = tid; j < my_nodes; j += THREADS) { a0[j] = 0ull; a1[j] = 0ull; }
            cluster.sync();
            if (stamp && rank == 0 && tid == 0) stamp[step + 1] = device_ns();
        }
        if (rank == 0 && tid == 0) R.needs_affine[sc] = 0;
    }
}

}  // namespace mpm
