// Fused transfer for the tiled MLS path: G2P of step n and P2G of step n+1 in
// one kernel per step (the G2P2G scheme of Wang et al., "A Massively Parallel
// and Scalable Multi-GPU Material Point Method", ACM TOG 39(4), 2020).
//
// One CTA per non-empty cell tile of the last sort (tiles handed out from a
// counter). The CTA stages the node velocities of a fixed box of BE^D nodes
// around its tile in shared memory (the stencils of every particle sorted into
// the tile that has since moved less than a cell): in k_g2p2g all threads load
// it between two CTA barriers; k_g2p2g_pipe (MPM_BOX_LOAD=tma) instead runs a
// two-stage pipeline of TMA tensor loads (cp.async.bulk.tensor, out-of-grid
// nodes zero-filled) with mbarriers and no CTA barrier. Then each warp, on its own,
// takes windows of 32 consecutive slots of the tile (handed out from a shared
// counter) and for its window
//   1. per particle (one lane each): gathers the grid from the box
//      (src/gpu/shaders/3d/g2p.glsl:28-71), updates x, v, B and the trial F_E,
//      and when the return map is provably the identity (elastic band)
//      computes the next step's P2G affine matrix A = 3 m B - 3 dt V sigma in
//      registers (3d/p2g.glsl:44-90); the rest are queued for the exact (or
//      learned) return map with their trial F;
//   2. writes each in-band particle's P2G payload (stencil weights at the new
//      position, m v, A) to the warp's shared-memory window, groups
//      consecutive slots that share a stencil into runs, and SPLIT lanes per
//      run (longest runs first) sum the run's node contributions in FP32
//      registers in slot order and add them to the global grid as int64 fixed
//      point (red.global, no return value).
// Warps synchronise only per tile (staging the box), so a warp with slow
// particles or a long run holds up no other. Particles whose stencil leaves
// the box (drifted more than a cell since the sort) gather from global memory
// and their runs add bounds-checked. Queued particles (out of the elastic
// band, or a stencil clipped by the grid edge) are scattered after their
// return map: the warp records its window (first slot, mask of the queued
// lanes), and k_p2g_windows repeats the window's run scatter over those lanes.
//
// Determinism: every cross-run sum is an integer add, and the runs are a
// function of the slot order, the window boundaries (fixed offsets inside a
// tile) and which particles were queued -- all functions of the state. After
// creation or a state upload a P2G-only pass of the same kernel (reading the
// stored state) forms the first sums. A checkpoint stores the pending sums
// themselves, so a resumed run never recomputes them.
#pragma once

#include <cuda.h>

#include "mpm_tiled.cuh"

namespace mpm {

#ifndef MPM_FUSED_THREADS
#define MPM_FUSED_THREADS 128
#endif
template <int D> struct FusedGeom {
    static constexpr int T = TileGeom<D>::T;            // cells per tile edge: 4 (3D), 8 (2D)
    static constexpr int BE = T + 5;                    // box edge in nodes: tile nodes - 2 .. tile + T + 2
    static constexpr int BN = D == 3 ? BE * BE * BE : BE * BE;  // 729 (3D), 169 (2D)
    static constexpr int BNP = (BN + 7) / 8 * 8;        // box rows padded to 128 bytes (TMA destinations)
    static constexpr int THREADS = MPM_FUSED_THREADS;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int WIN = 32;                      // slots per warp window (one per lane)
    static constexpr int PS = D == 3 ? 40 : 20;         // payload floats per particle (layout: p2g_payload)
    static constexpr int KEYF = PS - 2;                 // payload floats holding the 64-bit stencil key
    static_assert(THREADS % 32 == 0, "whole warps");
};

template <int D> struct FusedSmem {
    using G = FusedGeom<D>;
    float4 box[G::BN];                                  // 3D: (vf, wall flag); 2D: (vf, vc)
    int tile_next;                                      // tile-list entry of the CTA's current tile
    float4 pay[G::WARPS][G::WIN * G::PS / 4];           // per warp: the window's P2G payloads
    int run[G::WARPS][G::WIN + 1];                      // per warp: start slot of each run, then the window end
    int order[G::WARPS][G::WIN];                        // per warp: runs, longest first
    int next_win;                                       // next window of the tile to hand out
    unsigned bmask;                                     // node blocks (3^D around the tile) that received sums
};

// CTAs per SM the register budget is sized for: 20 warps per SM, 96
// registers (measured on the 128^3 snowball scene: 6 % faster than 24 warps at
// 80 registers, which spill)
#ifndef MPM_FUSED_MIN_BLOCKS
#define MPM_FUSED_MIN_BLOCKS (640 / MPM_FUSED_THREADS)
#endif

// ---------------------------------------------------------------------------
// Interior gather from a node array with strides (sy, sz): the box in shared
// memory (SMEM) or the global grid. Same sums and order as gather_interior.
// `gc0`, `gsy`, `gsz`: the global node id of the first stencil node and the
// global strides, for the wall-velocity pass (3D vc of nodes a wall moved is
// only kept in global memory).
template <int D, int S, bool SMEM, typename I>
__device__ __forceinline__ void gather_nodes(const StepConsts& C, const float4* nodes, I c0, I sy, I sz,
                                             const float4* __restrict__ gv, long long gc0, long long gsy, long long gsz,
                                             const float (*wk)[S], const float (*off)[S], float* nv, float* nB,
                                             float* nx) {
    float wd[3][S];
#pragma unroll
    for (int k = 0; k < D; ++k)
#pragma unroll
        for (int o = 0; o < S; ++o) wd[k][o] = wk[k][o] * off[k][o];
    float vc[D];
    bool wall = false;
#pragma unroll
    for (int r = 0; r < D; ++r) { nv[r] = 0.f; vc[r] = 0.f; }
#pragma unroll
    for (int k = 0; k < D * D; ++k) nB[k] = 0.f;
#pragma unroll 1
    for (int a = 0; a < S; ++a) {
        float Q[D], Qy[D], Qz[D], Qc[D];
#pragma unroll
        for (int r = 0; r < D; ++r) { Q[r] = 0.f; Qy[r] = 0.f; Qz[r] = 0.f; Qc[r] = 0.f; }
#pragma unroll
        for (int b = 0; b < S; ++b) {
            if constexpr (D == 3) {
                float Pv[3] = {0.f, 0.f, 0.f}, Pd[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int c = 0; c < S; ++c) {
                    const I cid = c0 + a + b * sy + c * sz;
                    const float4 g = SMEM ? nodes[cid] : __ldg(&nodes[cid]);
                    wall = wall || g.w != 0.f;
                    const float z = wk[2][c], zd = wd[2][c];
                    Pv[0] += z * g.x; Pv[1] += z * g.y; Pv[2] += z * g.z;
                    Pd[0] += zd * g.x; Pd[1] += zd * g.y; Pd[2] += zd * g.z;
                }
                const float y = wk[1][b], yd = wd[1][b];
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    Q[r] += y * Pv[r];
                    Qy[r] += yd * Pv[r];
                    Qz[r] += y * Pd[r];
                }
            } else {
                const I cid = c0 + a + b * sy;
                const float4 g = SMEM ? nodes[cid] : __ldg(&nodes[cid]);
                const float y = wk[1][b], yd = wd[1][b];
                Q[0] += y * g.x; Q[1] += y * g.y;
                Qy[0] += yd * g.x; Qy[1] += yd * g.y;
                Qc[0] += y * g.z; Qc[1] += y * g.w;
            }
        }
        const float x = pick<S>(wk[0], a);
        const float xd = pick<S>(wd[0], a);
#pragma unroll
        for (int r = 0; r < D; ++r) {
            nv[r] += x * Q[r];
            nB[r * D + 0] += xd * Q[r];
            nB[r * D + 1] += x * Qy[r];
            if (D == 3) nB[r * D + 2] += x * Qz[r];
            else vc[r] += x * Qc[r];
        }
    }
    if constexpr (D == 3) {
        if (!wall) {
#pragma unroll
            for (int r = 0; r < 3; ++r) vc[r] = nv[r];
        } else {
#pragma unroll 1
            for (int a = 0; a < S; ++a) {
                float Qc[3] = {0.f, 0.f, 0.f};
#pragma unroll 1
                for (int b = 0; b < S; ++b) {
                    float Pc[3] = {0.f, 0.f, 0.f};
#pragma unroll
                    for (int c = 0; c < S; ++c) {
                        float f[3], g[3];
                        load_node3(gv, C.nodes, gc0 + a + b * gsy + c * gsz, f, g);
                        const float z = wk[2][c];
                        Pc[0] += z * g[0]; Pc[1] += z * g[1]; Pc[2] += z * g[2];
                    }
                    const float y = pick<S>(wk[1], b);  // loop index not unrolled: no local array
#pragma unroll
                    for (int r = 0; r < 3; ++r) Qc[r] += y * Pc[r];
                }
                const float x = pick<S>(wk[0], a);
#pragma unroll
                for (int r = 0; r < 3; ++r) vc[r] += x * Qc[r];
            }
        }
    }
    float sw[3], swd[3];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        sw[k] = sum_s<S>(wk[k]);
        swd[k] = sum_s<S>(wd[k]);
    }
#pragma unroll
    for (int r = 0; r < D; ++r) {
        float t = swd[r];
#pragma unroll
        for (int l = 0; l < D; ++l)
            if (l != r) t *= sw[l];
        nx[r] = t + C.dt * vc[r];
    }
}

// ---------------------------------------------------------------------------
// P2G payload of one particle at position x; the 64-bit stencil key goes in
// the last two floats. f = x - (base + 1) is the offset in the particle's cell.
//   3D (40): wx[4] | wy[4] | wz[4] | yd[4] | zd[4] | s0 s1 m s2 |
//            A00 A10 0 A20 | A01 A11 0 A21 | A02 A12 0 A22 | pad pad key
//            with yd[b] = wy[b] (b - 1 - fy), zd[c] = wz[c] (c - 1 - fz),
//            s_r = m v_r - fx A_r0: the momentum channels in pairs (0, 1) and
//            (mass, 2) for the packed FP32 accumulation of fused_run.
//   2D (20): wx[4] | wy[4] | fx fy m mv0 | mv1 A00 A01 A10 | A11 pad key
template <int D, int S>
__device__ __forceinline__ unsigned long long p2g_payload(const StepConsts& C, const float* x, const float* v,
                                                          const float* A, float mass, float* q) {
    using St = Stencil<S>;
    unsigned long long k3 = 0;
    float f[3], mv[3];
#pragma unroll
    for (int k = D - 1; k >= 0; --k) {
        const int extk = k == 0 ? C.W : (k == 1 ? C.H : C.Dp);
        const int base = St::base(x[k], extk);
        float wt[S];
        St::weights(x[k], base, wt);
#pragma unroll
        for (int o = 0; o < 4; ++o) q[4 * k + o] = o < S ? wt[o] : 0.f;
        f[k] = x[k] - float(base + 1);
        mv[k] = mass * v[k];
        k3 |= (unsigned long long)(base + 9) << (StencilKey<D>::BITS * k);
    }
    if constexpr (D == 3) {
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            q[12 + o] = q[4 + o] * (float(o - 1) - f[1]);
            q[16 + o] = q[8 + o] * (float(o - 1) - f[2]);
        }
        reinterpret_cast<float4*>(q)[5] = make_float4(mv[0] - f[0] * A[0], mv[1] - f[0] * A[3], mass, mv[2] - f[0] * A[6]);
        reinterpret_cast<float4*>(q)[6] = make_float4(A[0], A[3], 0.f, A[6]);
        reinterpret_cast<float4*>(q)[7] = make_float4(A[1], A[4], 0.f, A[7]);
        reinterpret_cast<float4*>(q)[8] = make_float4(A[2], A[5], 0.f, A[8]);
    } else {
        reinterpret_cast<float4*>(q)[2] = make_float4(f[0], f[1], mass, mv[0]);
        reinterpret_cast<float4*>(q)[3] = make_float4(mv[1], A[0], A[1], A[2]);
        q[16] = A[3];
        q[17] = 0.f;
    }
    return k3;
}

// ---------------------------------------------------------------------------
// One work item of the run accumulation: split `a` of the run [j0, j1) of a
// warp's payload window `pay`, stencil key kk. Sums in registers in slot
// order and adds them to the global grid as int64 fixed point. When `boxed`
// and the whole stencil lies in the tile's node box (origin bo) and in the
// grid, the adds need no bounds checks and the function returns the node
// blocks they touched, as bits of the 3^D blocks around the tile (tile
// coordinates tc); otherwise the adds are bounds-checked, the node blocks
// marked here, and it returns 0. Same arithmetic as k_p2g_warp.
template <int D, int S>
__device__ __forceinline__ unsigned fused_run(const StepConsts& C, const TileInfo& TI, const float4* pay, bool boxed,
                                              const int* bo, const int* tc, int j0, int j1, unsigned long long kk,
                                              int a, unsigned long long* __restrict__ acc,
                                              unsigned* __restrict__ status) {
    using G = FusedGeom<D>;
    using W = WarpGeom<D, S>;
    constexpr int T = TileGeom<D>::T;
    const float* payf = reinterpret_cast<const float*>(pay);
    int cell[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < D; ++k) cell[k] = int((kk >> (StencilKey<D>::BITS * k)) & StencilKey<D>::MASK) - 8;
    // stencil nodes cell - 1 .. cell + S - 2 per axis
    bool in_box = boxed, in_grid = true;
    const int ext[3] = {C.W, C.H, C.Dp};
#pragma unroll
    for (int k = 0; k < D; ++k) {
        in_box = in_box && cell[k] - 1 - bo[k] >= 0 && cell[k] + S - 2 - bo[k] <= G::BE - 1;
        in_grid = in_grid && cell[k] - 1 >= 0 && cell[k] + S - 2 <= ext[k];
    }
    if constexpr (D == 3) {
        constexpr int NB = S * S / W::SPLIT;
        constexpr int NN = NB * S;
        const int ax = a % S, by0 = (a / S) * NB;
        // channel pairs (a0, a1) and (am, a2) per node, in packed FP32
        // (fma.rn.f32x2: two FP32 FMAs per instruction)
        float2 p01[NN], pm2[NN];
#pragma unroll
        for (int k = 0; k < NN; ++k) { p01[k] = make_float2(0.f, 0.f); pm2[k] = make_float2(0.f, 0.f); }
        const float2 da2 = make_float2(float(ax - 1), float(ax - 1));
        for (int j = j0; j < j1; ++j) {
            const float4* pp = pay + j * (G::PS / 4);
            const float alpha = payf[j * G::PS + ax];
            const float2 al2 = make_float2(alpha, alpha);
            const float4 wy = pp[1], wz = pp[2], yd = pp[3], zd = pp[4], p5 = pp[5], p6 = pp[6], p7 = pp[7],
                         p8 = pp[8];
            // (e0, e1) = alpha (s0 + da A00, s1 + da A10); (ma, e2) = alpha (m, s2 + da A20)
            const float2 e01 = __fmul2_rn(al2, __ffma2_rn(da2, make_float2(p6.x, p6.y), make_float2(p5.x, p5.y)));
            const float2 me2 = __fmul2_rn(al2, __ffma2_rn(da2, make_float2(p6.z, p6.w), make_float2(p5.z, p5.w)));
            const float2 f01 = __fmul2_rn(al2, make_float2(p7.x, p7.y)), f_2 = __fmul2_rn(al2, make_float2(p7.z, p7.w));
            const float2 g01 = __fmul2_rn(al2, make_float2(p8.x, p8.y)), g_2 = __fmul2_rn(al2, make_float2(p8.z, p8.w));
            const float Z[4] = {wz.x, wz.y, wz.z, wz.w};
            const float Zd[4] = {zd.x, zd.y, zd.z, zd.w};
            const float Yv[4] = {wy.x, wy.y, wy.z, wy.w};
            const float Ydv[4] = {yd.x, yd.y, yd.z, yd.w};
            float2 Z2[S], Zd2[S];
#pragma unroll
            for (int cc = 0; cc < S; ++cc) { Z2[cc] = make_float2(Z[cc], Z[cc]); Zd2[cc] = make_float2(Zd[cc], Zd[cc]); }
#pragma unroll
            for (int bb = 0; bb < NB; ++bb) {
                const int b = by0 + bb;
                const float Y = NB == S ? Yv[bb] : (b == 0 ? wy.x : b == 1 ? wy.y : b == 2 ? wy.z : wy.w);
                const float Yd = NB == S ? Ydv[bb] : (b == 0 ? yd.x : b == 1 ? yd.y : b == 2 ? yd.z : yd.w);
                const float2 Y2 = make_float2(Y, Y), Yd2 = make_float2(Yd, Yd);
                // (h0, h1), (mY, h2): h_r = e_r Y + f_r Yd, mY = ma Y; (k0, k1), (0, k2): k_r = g_r Y
                const float2 h01 = __ffma2_rn(e01, Y2, __fmul2_rn(f01, Yd2));
                const float2 hm2 = __ffma2_rn(me2, Y2, __fmul2_rn(f_2, Yd2));
                const float2 k01 = __fmul2_rn(g01, Y2), k_2 = __fmul2_rn(g_2, Y2);
#pragma unroll
                for (int cc = 0; cc < S; ++cc) {
                    const int idx = bb * S + cc;
                    p01[idx] = __ffma2_rn(h01, Z2[cc], __ffma2_rn(k01, Zd2[cc], p01[idx]));
                    pm2[idx] = __ffma2_rn(hm2, Z2[cc], __ffma2_rn(k_2, Zd2[cc], pm2[idx]));
                }
            }
        }
        float am[NN], a0[NN], a1[NN], a2[NN];
#pragma unroll
        for (int k = 0; k < NN; ++k) { am[k] = pm2[k].x; a2[k] = pm2[k].y; a0[k] = p01[k].x; a1[k] = p01[k].y; }
        float mx_m = 0.f, mx_p = 0.f;
#pragma unroll
        for (int k = 0; k < NN; ++k) {
            mx_m = fmaxf(mx_m, fabsf(am[k]));
            mx_p = fmaxf(mx_p, fmaxf(fabsf(a0[k]), fmaxf(fabsf(a1[k]), fabsf(a2[k]))));
        }
        if (!(mx_m * C.sm < kFixedLimit && mx_p * C.sp < kFixedLimit))
            raise_flag(status, (mx_m != mx_m || mx_p != mx_p) ? 1u : 2u);
        const int gx = cell[0] - 1 + ax;
        if (in_box && in_grid) {
            const long long sy = C.nx, sz = (long long)C.nx * C.ny;
            const long long g0 = ((long long)(cell[2] - 1) * C.ny + (cell[1] - 1 + by0)) * C.nx + gx;
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
            // blocks of the thread's nodes: one x block, a y range, a z range
            // (all within one block of the tile's, since the stencil is in the box)
            unsigned bits = 0u;
            const int rx = gx / T - tc[0] + 1;
            const int y0 = (cell[1] - 1 + by0) / T - tc[1] + 1, y1 = (cell[1] - 2 + by0 + NB) / T - tc[1] + 1;
            const int z0 = (cell[2] - 1) / T - tc[2] + 1, z1 = (cell[2] + S - 2) / T - tc[2] + 1;
            for (int rz = z0; rz <= z1; ++rz)
                for (int ry = y0; ry <= y1; ++ry) bits |= 1u << ((rz * 3 + ry) * 3 + rx);
            return bits;
        }
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
        if (gx >= 0 && gx <= C.W) {
            const int y0 = max(0, cell[1] - 1 + by0), y1 = min(C.H, cell[1] - 2 + by0 + NB);
            const int z0 = max(0, cell[2] - 1), z1 = min(C.Dp, cell[2] + (S - 2));
            if (y0 <= y1 && z0 <= z1)
                for (int bz = z0 / T; bz <= z1 / T; ++bz)
                    for (int by = y0 / T; by <= y1 / T; ++by)
                        mark_block_once(TI, (bz * TI.nblk[1] + by) * TI.nblk[0] + gx / T);
        }
        return 0u;
    } else {
        constexpr int NA = S / W::SPLIT;
        const int gx0 = cell[0] - 1 + a * NA;
        float am[NA * S], a0[NA * S], a1[NA * S];
#pragma unroll
        for (int k = 0; k < NA * S; ++k) { am[k] = 0.f; a0[k] = 0.f; a1[k] = 0.f; }
        for (int j = j0; j < j1; ++j) {
            const float4* pp = pay + j * (G::PS / 4);
            const float4 wx = pp[0], wy = pp[1], p2 = pp[2], p3 = pp[3];
            const float a11 = payf[j * G::PS + 16];
            // f = (p2.x, p2.y), m = p2.z, mv = (p2.w, p3.x), A = (p3.y p3.z | p3.w a11)
            const float Xv[4] = {wx.x, wx.y, wx.z, wx.w};
            const float Y[4] = {wy.x, wy.y, wy.z, wy.w};
            float Yd[4];
#pragma unroll
            for (int b = 0; b < S; ++b) Yd[b] = Y[b] * (float(b - 1) - p2.y);
#pragma unroll
            for (int i = 0; i < NA; ++i) {
                const int aa = a * NA + i;
                const float X = NA == S ? Xv[i] : payf[j * G::PS + aa];
                const float Xd = X * (float(aa - 1) - p2.x);
                const float e0 = p2.w * X + p3.y * Xd, e1 = p3.x * X + p3.w * Xd;
                const float f0 = p3.z * X, f1 = a11 * X, mX = p2.z * X;
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
        if (in_box && in_grid) {
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
            unsigned bits = 0u;
            const int x0 = gx0 / T - tc[0] + 1, x1 = (gx0 + NA - 1) / T - tc[0] + 1;
            const int y0 = (cell[1] - 1) / T - tc[1] + 1, y1 = (cell[1] + S - 2) / T - tc[1] + 1;
            for (int ry = y0; ry <= y1; ++ry)
                for (int rx = x0; rx <= x1; ++rx) bits |= 1u << (ry * 3 + rx);
            return bits;
        }
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
        const int x0 = max(0, gx0), x1 = min(C.W, gx0 + (NA - 1));
        const int y0 = max(0, cell[1] - 1), y1 = min(C.H, cell[1] + (S - 2));
        if (x0 <= x1 && y0 <= y1)
            for (int by = y0 / T; by <= y1 / T; ++by)
                for (int bx = x0 / T; bx <= x1 / T; ++bx) mark_block_once(TI, by * TI.nblk[0] + bx);
        return 0u;
    }
}

// ---------------------------------------------------------------------------
// The scatter of one warp's window of payloads (`pay`, the stencil key in the
// last two floats of each; kNoStencil for slots that add nothing): runs of
// consecutive slots with one key, longest first, SPLIT lanes per run summing
// it (fused_run). The first `cnt` slots of the window are filled. Returns this
// lane's node-block bits (boxed runs only).
template <int D, int S>
__device__ __forceinline__ unsigned scatter_window(const StepConsts& C, const TileInfo& TI, const float4* pay,
                                                   int* run, int* order, int cnt, bool boxed, const int* bo,
                                                   const int* tc, unsigned long long* __restrict__ acc,
                                                   unsigned* __restrict__ status) {
    using G = FusedGeom<D>;
    using W = WarpGeom<D, S>;
    const int lane = threadIdx.x & 31;
    const bool valid = lane < cnt;
    // runs: maximal stretches of consecutive slots with one stencil key
    const unsigned long long* keyp = reinterpret_cast<const unsigned long long*>(
        reinterpret_cast<const float*>(pay) + G::KEYF);
    auto key_at = [&](int j) { return keyp[j * (G::PS / 2)]; };
    const bool is_start = valid && (lane == 0 || key_at(lane) != key_at(lane - 1));
    const unsigned starts = __ballot_sync(0xffffffffu, is_start);
    const int nruns = __popc(starts);
    const int r_me = __popc(starts & ((1u << lane) - 1));
    if (is_start) run[r_me] = lane;
    if (lane == 0) run[nruns] = cnt;
    __syncwarp();
    // runs longest first, so that the SPLIT-lane groups sharing a pass have
    // similar lengths; which lanes sum a run changes no result
    {
        const int len = lane < nruns ? run[lane + 1] - run[lane] : 0;
        int rank = 0;
        for (int qr = 0; qr < nruns; ++qr) {
            const int lq = __shfl_sync(0xffffffffu, len, qr);
            rank += lq > len || (lq == len && qr < lane);
        }
        if (lane < nruns) order[rank] = lane;
    }
    __syncwarp();
    unsigned bits = 0u;
    for (int u = lane; u < nruns * W::SPLIT; u += 32) {
        const int r = order[u / W::SPLIT], a = u % W::SPLIT;
        const int j0 = run[r], j1 = run[r + 1];
        const unsigned long long kk = key_at(j0);
        if (kk == kNoStencil) continue;
        bits |= fused_run<D, S>(C, TI, pay, boxed, bo, tc, j0, j1, kk, a, acc, status);
    }
    __syncwarp();  // the window's payload and runs are reused by the next window
    return bits;
}

// P2G of the queued particles after their return map, by the windows the
// fused kernel recorded: one warp per window, the window's queued slots
// (x, v, A as the G2P and return-map kernels left them) grouped into runs of
// one stencil and summed as in the fused kernel. The grouping is a function
// of the window and of which of its particles were queued, so the int64 sums
// do not depend on the order in which windows were recorded.
template <int D, int S>
__global__ void __launch_bounds__(FusedGeom<D>::THREADS) k_p2g_windows(Particles P, StepConsts C, TileInfo TI,
                                                                      SlowQueue Q,
                                                                      unsigned long long* __restrict__ acc,
                                                                      unsigned* __restrict__ status) {
    using G = FusedGeom<D>;
    __shared__ float4 pay_s[G::WARPS][G::WIN * G::PS / 4];
    __shared__ int run_s[G::WARPS][G::WIN + 1];
    __shared__ int order_s[G::WARPS][G::WIN];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = min(*Q.nwin, Q.win_capacity);
    const int n = P.n;
    const int none[3] = {0, 0, 0};
    float4* pay = pay_s[wid];
    for (int r = blockIdx.x * G::WARPS + wid; r < nw; r += gridDim.x * G::WARPS) {
        const int2 rec = Q.win[r];
        const unsigned mask = (unsigned)rec.y;
        if ((mask >> lane) & 1u) {
            // the queued slots packed in slot order, so that particles of one
            // cell form one run even when in-band ones sat between them
            float* q = reinterpret_cast<float*>(pay) + __popc(mask & ((1u << lane) - 1)) * G::PS;
            const int i = rec.x + lane;
            const float mass = P.mass ? P.mass[i] : P.mass_u;
            float x[D], v[D], A[D * D];
#pragma unroll
            for (int k = 0; k < D; ++k) { x[k] = P.x[k * n + i]; v[k] = P.v[k * n + i]; }
#pragma unroll
            for (int k = 0; k < D * D; ++k) A[k] = P.A[k * n + i];
            reinterpret_cast<unsigned long long*>(q + G::KEYF)[0] = p2g_payload<D, S>(C, x, v, A, mass, q);
        }
        __syncwarp();
        scatter_window<D, S>(C, TI, pay, run_s[wid], order_s[wid], __popc(mask), false, none, none, acc, status);
    }
}

// ---------------------------------------------------------------------------
// TMA load of a tile's node box and its mbarrier (sm_90+ PTX): each CTA loads
// its own boxes from this GPU's memory.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Waits for the phase `parity` of the mbarrier to complete; false after
// `limit` polls (each poll may suspend the thread for a short while).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit) {
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
constexpr int kBoxWaitPolls = 1 << 20;

// One arrival on the mbarrier (release at CTA scope).
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// The node box of tile t (origin node bo) into `dst`: one tensor load of the
// node-velocity array viewed as [nz][ny][nx][4] floats (gv's first half);
// nodes outside the grid read as zero. The mbarrier expects the box's bytes.
template <int D>
__device__ __forceinline__ void box_load(const CUtensorMap& map, const int* bo, float4* dst, unsigned long long* bar) {
    constexpr uint32_t bytes = FusedGeom<D>::BN * sizeof(float4);
    const uint32_t b = smem_u32(bar), d = smem_u32(dst);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    if constexpr (D == 3) {
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
            ::"r"(d), "l"(reinterpret_cast<uint64_t>(&map)), "r"(0), "r"(bo[0]), "r"(bo[1]), "r"(bo[2]), "r"(b)
            : "memory");
    } else {
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
            ::"r"(d), "l"(reinterpret_cast<uint64_t>(&map)), "r"(0), "r"(bo[0]), "r"(bo[1]), "r"(b)
            : "memory");
    }
}

// Tile coordinates and box origin node of tile t.
template <int D>
__device__ __forceinline__ void tile_origin(const TileInfo& TI, int t, int* tc, int* bo) {
#pragma unroll
    for (int k = 0; k < D; ++k) { tc[k] = t % TI.tiles[k]; t /= TI.tiles[k]; bo[k] = tc[k] * FusedGeom<D>::T - 2; }
}

// ---------------------------------------------------------------------------
// Window w (slots start + 32 w ...) of a tile of m slots, by one warp: G2P of
// each slot's particle against the tile's node box (G2P = true) or the stored
// state (G2P = false), then the scatter of the in-band particles' payloads.
// Returns this lane's node-block bits of the tile (tile coordinates tc, box
// origin bo).
template <int D, int S, bool G2P>
__device__ __forceinline__ unsigned fused_window(const Particles& P, const StepConsts& C, const TileInfo& TI,
                                                 const float4* __restrict__ gv, unsigned long long* __restrict__ acc,
                                                 const SlowQueue& Q, unsigned* __restrict__ status, const float4* box,
                                                 const int* bo, const int* tc, int start, int m, int w, float4* pay,
                                                 int* run, int* order) {
    using G = FusedGeom<D>;
    using St = Stencil<S>;
    const int lane = threadIdx.x & 31;
    const int n = P.n;
    const long long gsy = C.nx, gsz = (long long)C.nx * C.ny;
    const int cnt = min(G::WIN, m - w * G::WIN);
    const bool valid = lane < cnt;
    const int i = start + w * G::WIN + lane;
    unsigned long long key = kNoStencil;
    bool deferred = false;  // queued: scattered after the return map (k_p2g_windows)
    float* q = reinterpret_cast<float*>(pay) + lane * G::PS;
    if (valid) {
        const float mass = P.mass ? P.mass[i] : P.mass_u, vol = P.vol ? P.vol[i] : P.vol_u;
        float x[D], v[D], A[D * D];
        bool scatter = vol != 0.f;  // p2g.glsl:42
        if constexpr (G2P) {
            float xo[D];
#pragma unroll
            for (int k = 0; k < D; ++k) xo[k] = P.x[k * n + i];
            int base[3] = {0, 0, 0};
            float wk[3][S], off[3][S];
            bool interior = true, boxed = true;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                const int ext = k == 0 ? C.W : (k == 1 ? C.H : C.Dp);
                base[k] = St::base(xo[k], ext);
                interior = interior && base[k] >= 0 && base[k] + (S - 1) <= ext;
                boxed = boxed && base[k] - bo[k] >= 0 && base[k] + (S - 1) - bo[k] <= G::BE - 1;
                St::weights(xo[k], base[k], wk[k]);
#pragma unroll
                for (int o = 0; o < S; ++o) off[k][o] = float(base[k] + o) - xo[k];
            }
            if (!interior) {
                // stencil partly outside the grid: the general kernel does the whole G2P
                Q.list[queue_slot(Q)] = -1 - i;
                deferred = scatter;
                scatter = false;
            } else {
                float nv[D], nx[D], nB[D * D];
                const long long gc0 = (D == 3 ? base[2] * gsz : 0) + base[1] * gsy + base[0];
                if (boxed) {
                    const int l0 = (D == 3 ? (base[2] - bo[2]) * G::BE * G::BE : 0) + (base[1] - bo[1]) * G::BE +
                                   (base[0] - bo[0]);
                    gather_nodes<D, S, true, int>(C, box, l0, G::BE, G::BE * G::BE, gv, gc0, gsy, gsz, wk, off,
                                                  nv, nB, nx);
                } else {
                    gather_nodes<D, S, false, long long>(C, gv, gc0, gsy, gsz, gv, gc0, gsy, gsz, wk, off, nv, nB,
                                                         nx);
                }
                bool finite = true;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    x[k] = xo[k] + nx[k];
                    v[k] = nv[k];
                    P.v[k * n + i] = nv[k];
                    P.x[k * n + i] = x[k];
                    finite = finite && isfinite(x[k]);
                }
                if (!finite) raise_flag(status, 1u);
#pragma unroll
                for (int k = 0; k < D * D; ++k) P.B[k * n + i] = nB[k];
                float Fe[D * D], Fh[D * D];
#pragma unroll
                for (int k = 0; k < D * D; ++k) Fe[k] = P.Fe[k * n + i];
#pragma unroll
                for (int r = 0; r < D; ++r)
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        float s = Fe[r * D + c];
#pragma unroll
                        for (int k = 0; k < D; ++k) s += (C.dt * St::DINV * nB[r * D + k]) * Fe[k * D + c];
                        Fh[r * D + c] = s;
                    }
                float sig[D * D];
                const float Jp = P.Jp[i];
                if (det<D>(Fh) > 0.f && band_gershgorin<D>(Fh, 1.f - C.theta_c, 1.f + C.theta_s) &&
                    hardened_stress_series<D>(Fh, Jp, C.mu0, C.la0, C.xi, sig)) {
#pragma unroll
                    for (int k = 0; k < D * D; ++k) {
                        P.Fe[k * n + i] = Fh[k];
                        A[k] = St::DINV * mass * nB[k] - St::DINV * C.dt * vol * sig[k];
                    }
                } else {
                    const int slot = queue_slot(Q);
                    Q.list[slot] = i;
#pragma unroll
                    for (int k = 0; k < D * D; ++k) Q.fh[k * Q.capacity + slot] = Fh[k];
                    deferred = scatter;
                    scatter = false;
                }
            }
        } else {
            float B[D * D], Fe[D * D];
#pragma unroll
            for (int k = 0; k < D; ++k) { x[k] = P.x[k * n + i]; v[k] = P.v[k * n + i]; }
#pragma unroll
            for (int k = 0; k < D * D; ++k) { B[k] = P.B[k * n + i]; Fe[k] = P.Fe[k * n + i]; }
            mls_affine<D, S>(C, B, Fe, P.Jp[i], mass, vol, A);
        }
        if (scatter) key = p2g_payload<D, S>(C, x, v, A, mass, q);
    }
    if constexpr (G2P) {
        // record the window if some of its particles wait for the return map
        const unsigned dm = __ballot_sync(0xffffffffu, deferred);
        if (dm && lane == 0) {
            const int r = atomicAdd(Q.nwin, 1);
            if (r < Q.win_capacity) Q.win[r] = make_int2(start + w * G::WIN, (int)dm);
        }
    }
    reinterpret_cast<unsigned long long*>(q + G::KEYF)[0] = key;
    __syncwarp();
    return scatter_window<D, S>(C, TI, pay, run, order, cnt, true, bo, tc, acc, status);
}

// ---------------------------------------------------------------------------
// The fused kernel. G2P = true: one step (G2P of the state, then the next
// step's P2G into `acc`). G2P = false: the P2G of the stored state only (after
// creation or a state upload), reading B, F_E, J_p and forming A as every
// other path does (mls_affine).
template <int D, int S, bool G2P>
__global__ void __launch_bounds__(FusedGeom<D>::THREADS, MPM_FUSED_MIN_BLOCKS)
    k_g2p2g(Particles P, StepConsts C, TileInfo TI, const float4* __restrict__ gv, unsigned long long* __restrict__ acc,
            SlowQueue Q, unsigned* __restrict__ status) {
    using G = FusedGeom<D>;
    extern __shared__ __align__(128) unsigned char fused_smem[];
    FusedSmem<D>& SM = *reinterpret_cast<FusedSmem<D>*>(fused_smem);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int ntl = *TI.n_tile_list;
    const long long gsy = C.nx, gsz = (long long)C.nx * C.ny;
    float4* pay = SM.pay[wid];
    int* run = SM.run[wid];
    int* order = SM.order[wid];
    for (;;) {
        if (tid == 0) {
            SM.tile_next = atomicAdd(TI.fused_next, 1);
            SM.next_win = 0;
            SM.bmask = 0u;
        }
        __syncthreads();
        const int e = SM.tile_next;
        if (e >= ntl) break;
        const float4* box = SM.box;
        const int t = TI.tile_list[e];
        const int start = TI.tile_start[t], m = TI.tile_len[e];
        int tc[3] = {0, 0, 0}, bo[3] = {0, 0, 0};  // tile coordinates, box origin node
        tile_origin<D>(TI, t, tc, bo);
        if constexpr (G2P) {  // stage the node velocities of the box
            for (int l = tid; l < G::BN; l += G::THREADS) {
                const int lx = l % G::BE, ly = (l / G::BE) % G::BE, lz = D == 3 ? l / (G::BE * G::BE) : 0;
                const int gx = bo[0] + lx, gy = bo[1] + ly, gz = D == 3 ? bo[2] + lz : 0;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (gx >= 0 && gx <= C.W && gy >= 0 && gy <= C.H && (D == 2 || (gz >= 0 && gz <= C.Dp)))
                    v = __ldg(&gv[gz * gsz + gy * gsy + gx]);
                SM.box[l] = v;
            }
            // the tile's G2P inputs (x, F_E, J_p) towards L2 ahead of the windows
            // that read them; one prefetch per 128-byte line, addresses kept
            // inside the arrays
            {
                constexpr int NF = D + D * D + 1;
                const int lines = (m + 31) / 32 + 1;
                const int n = P.n;
                for (int l = tid; l < NF * lines; l += G::THREADS) {
                    const int f = l / lines, k = l % lines;
                    const float* a = f < D ? P.x + (long long)f * n
                                           : (f < D + D * D ? P.Fe + (long long)(f - D) * n : P.Jp);
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a + min(start + 32 * k, n - 1)));
                }
            }
            __syncthreads();
        }
        unsigned bits = 0u;  // node blocks this lane's in-box runs added to
        const int nwin = (m + G::WIN - 1) / G::WIN;
        for (;;) {
            int w = 0;
            if (lane == 0) w = atomicAdd(&SM.next_win, 1);
            w = __shfl_sync(0xffffffffu, w, 0);
            if (w >= nwin) break;
            bits |= fused_window<D, S, G2P>(P, C, TI, gv, acc, Q, status, box, bo, tc, start, m, w, pay, run, order);
        }
        // mark the node blocks the tile's in-box runs added to
        bits = __reduce_or_sync(0xffffffffu, bits);
        if (lane == 0 && bits) atomicOr(&SM.bmask, bits);
        __syncthreads();
        constexpr int NBLK = D == 3 ? 27 : 9;
        if (tid < NBLK && (SM.bmask >> tid) & 1u) {
            const int rx = tid % 3, ry = (tid / 3) % 3, rz = tid / 9;
            const int bx = tc[0] - 1 + rx, by = tc[1] - 1 + ry, bz = D == 3 ? tc[2] - 1 + rz : 0;
            mark_block_once(TI, (bz * TI.nblk[1] + by) * TI.nblk[0] + bx);
        }
        __syncthreads();  // SM.bmask, the tile and the box are reset for the next tile
    }
}

// ---------------------------------------------------------------------------
// The fused step with the node boxes brought in by TMA and no CTA barrier
// after the start: a two-stage pipeline per CTA. Stage k (tile k of the CTA)
// lives in buffer k & 1: its tile, its box (one TMA tensor load, whose
// mbarrier `full` completes when the bytes have landed), a window counter,
// a count of the warps that have left it, and its node-block bits. Each warp
// waits for the stage's box, takes windows of the tile until none are left,
// and moves on to stage k + 1, which is already loaded; the last warp to leave
// stage k marks the tile's node blocks and refills the buffer with stage
// k + 2 (the next tile from the global counter, or an empty stage that ends
// the CTA). A warp is thus held up only by a box that has not arrived, never
// by the other warps' windows. Stages are refilled in order, so tile numbers
// grow with the stage and the first empty stage ends the work for every warp.
// Every wait is bounded: a box that does not arrive raises MPM_FLAG_TIMEOUT.
template <int D> struct PipeSmem {
    using G = FusedGeom<D>;
    alignas(128) float4 box[2][G::BNP];                 // (vf, wall flag) per node
    unsigned long long full[2];                         // the stage's box arrived (or the stage is empty)
    int tile[2];                                        // tile-list entry of the stage (>= count: empty)
    int next_win[2];
    int left[2];                                        // warps done with the stage
    unsigned bmask[2];
    float4 pay[G::WARPS][G::WIN * G::PS / 4];
    int run[G::WARPS][G::WIN + 1];
    int order[G::WARPS][G::WIN];
};

// Stage for buffer b: the next tile of the global counter and its box load,
// or an empty stage. One thread.
template <int D>
__device__ __forceinline__ void pipe_refill(PipeSmem<D>& SM, int b, const TileInfo& TI, int ntl,
                                            const CUtensorMap& map) {
    const int e = atomicAdd(TI.fused_next, 1);
    SM.tile[b] = e;
    if (e < ntl) {
        int tc[3], bo[3];
        tile_origin<D>(TI, TI.tile_list[e], tc, bo);
        fence_proxy_async_smem();
        box_load<D>(map, bo, SM.box[b], &SM.full[b]);
    } else {
        mbar_arrive(&SM.full[b]);
    }
}

template <int D, int S>
__global__ void __launch_bounds__(FusedGeom<D>::THREADS, MPM_FUSED_MIN_BLOCKS)
    k_g2p2g_pipe(Particles P, StepConsts C, TileInfo TI, const float4* __restrict__ gv,
                 unsigned long long* __restrict__ acc, SlowQueue Q, unsigned* __restrict__ status,
                 const __grid_constant__ CUtensorMap gv_map) {
    using G = FusedGeom<D>;
    constexpr int NBLK = D == 3 ? 27 : 9;
    extern __shared__ __align__(128) unsigned char fused_smem[];
    PipeSmem<D>& SM = *reinterpret_cast<PipeSmem<D>*>(fused_smem);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int ntl = *TI.n_tile_list;
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(&SM.full[b], 1);
            SM.next_win[b] = 0;
            SM.left[b] = 0;
            SM.bmask[b] = 0u;
        }
        mbar_init_fence();
        pipe_refill<D>(SM, 0, TI, ntl, gv_map);
        pipe_refill<D>(SM, 1, TI, ntl, gv_map);
    }
    __syncthreads();
    for (int k = 0;; ++k) {
        const int b = k & 1;
        const unsigned par = (unsigned)(k >> 1) & 1u;
        if (!__all_sync(0xffffffffu, mbar_wait(&SM.full[b], par, kBoxWaitPolls))) {
            // the box never arrived (flagged); let the other buffer's load land first
            if (lane == 0) {
                raise_flag(status, 16u);
                mbar_wait(&SM.full[b ^ 1], (unsigned)((k + 1) >> 1) & 1u, kBoxWaitPolls);
            }
            return;
        }
        const int e = SM.tile[b];
        if (e >= ntl) break;
        const int t = TI.tile_list[e];
        const int start = TI.tile_start[t], m = TI.tile_len[e];
        int tc[3] = {0, 0, 0}, bo[3] = {0, 0, 0};
        tile_origin<D>(TI, t, tc, bo);
        const int nwin = (m + G::WIN - 1) / G::WIN;
        unsigned bits = 0u;
        for (;;) {
            int w = 0;
            if (lane == 0) w = atomicAdd(&SM.next_win[b], 1);
            w = __shfl_sync(0xffffffffu, w, 0);
            if (w >= nwin) break;
            bits |= fused_window<D, S, true>(P, C, TI, gv, acc, Q, status, SM.box[b], bo, tc, start, m, w,
                                             SM.pay[wid], SM.run[wid], SM.order[wid]);
        }
        bits = __reduce_or_sync(0xffffffffu, bits);
        int last = 0;
        if (lane == 0) {
            if (bits) atomicOr(&SM.bmask[b], bits);
            __threadfence_block();  // the bits and this warp's reads of the box before the count
            last = atomicAdd(&SM.left[b], 1) == G::WARPS - 1;
        }
        if (__shfl_sync(0xffffffffu, last, 0)) {
            // last warp out: mark the tile's node blocks, then stage k + 2 into this buffer
            __threadfence_block();
            unsigned bm = 0u;
            if (lane == 0) bm = atomicOr(&SM.bmask[b], 0u);
            bm = __shfl_sync(0xffffffffu, bm, 0);
            if (lane < NBLK && (bm >> lane) & 1u) {
                const int rx = lane % 3, ry = (lane / 3) % 3, rz = lane / 9;
                const int bx = tc[0] - 1 + rx, by = tc[1] - 1 + ry, bz = D == 3 ? tc[2] - 1 + rz : 0;
                mark_block_once(TI, (bz * TI.nblk[1] + by) * TI.nblk[0] + bx);
            }
            __syncwarp();
            if (lane == 0) {
                SM.bmask[b] = 0u;
                SM.next_win[b] = 0;
                SM.left[b] = 0;
                pipe_refill<D>(SM, b, TI, ntl, gv_map);
            }
            __syncwarp();
        }
    }
}

}  // namespace mpm
