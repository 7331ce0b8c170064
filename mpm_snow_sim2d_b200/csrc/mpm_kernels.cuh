// Step kernels of the B200 MLS-MPM solver: P2G scatter, grid update, G2P with
// plasticity, plus state import/export. Templated on the dimension D and the
// formulation FORM (kMLS: the reference GPU shaders; kClassic: the reference
// CPU path, 2D).
//
// HBM layout (structure of arrays, FP32, component-major with stride n):
//   x[D][n], v[D][n], B[D*D][n], Fe[D*D][n], Jp[n]
//   mass/vol: per particle or a uniform scalar (pointer == nullptr)
// Grid (nodes = (W+1)(H+1)(D+1), x fastest):
//   acc[NACC][nodes]  int64 fixed-point sums: mass, momentum[D] (+ force[D] CLASSIC)
//   gv                node velocities for G2P: 2D float4 (vf.x, vf.y, vc.x, vc.y);
//                     3D two float4 per node (vf.xyz, 0), (vc.xyz, 0)
#pragma once

#include "mpm_math.cuh"

namespace mpm {

struct StepConsts {
    int W, H, Dp;             // cells per axis (WIDTH, HEIGHT, DEPTH)
    int nx, ny, nz;           // nodes per axis
    long long nodes;
    float dt, gravity, friction, theta_c, theta_s, xi, mu0, la0, margin;
    float sm, sp, sf;         // fixed-point scales: mass, momentum, force (powers of two)
    float inv_sm, inv_sp, inv_sf;
    float v_cap;              // |node velocity| above this means the momentum scale may have wrapped
    int boundary;
};

struct Particles {
    float* x;
    float* v;
    float* B;
    float* Fe;
    float* Jp;
    float* A;           // MLS path: P2G affine matrix of the next step (nullptr elsewhere)
    const float* mass;  // nullptr: uniform mass_u
    const float* vol;   // nullptr: uniform vol_u
    float mass_u, vol_u;
    int n;
};

template <int D, int FORM> struct Layout {
    static constexpr int NACC = (FORM == kClassic) ? 1 + 2 * D : 1 + D;
};

__device__ __forceinline__ void raise_flag(unsigned* status, unsigned bit) {
    atomicOr(status, bit);
}

// Largest magnitude one fixed-point contribution may take (2^62): leaves room
// for partial sums; a node velocity above v_cap flags a possible wrap instead.
constexpr float kFixedLimit = 4.611686e18f;

__device__ __forceinline__ long long to_fixed(float val, float scale, unsigned* status) {
    float t = val * scale;
    if (!(fabsf(t) < kFixedLimit)) {
        raise_flag(status, (t != t) ? 1u /*NAN*/ : 2u /*OVERFLOW*/);
        t = (t != t) ? 0.f : copysignf(kFixedLimit, t);
    }
    return __float2ll_rn(t);
}

__device__ __forceinline__ void red_add(unsigned long long* p, long long v) {
    if (v != 0) atomicAdd(p, (unsigned long long)v);
}

// First stencil node int(x) - 1 (C truncation, as int() in p2g.glsl:61 and
// static_cast<int> in src/cpu/Grid.cpp:122). x is first clamped to
// [-8, extent + 8] so that non-finite or far-away positions cannot overflow the
// index arithmetic; their stencils then lie wholly outside the grid, as they
// would in the reference.
__device__ __forceinline__ int stencil_base(float x, int extent) {
    return int(fminf(fmaxf(x, -8.f), float(extent) + 8.f)) - 1;
}

// A stencil of S nodes per axis: first node base(x), weight w(x - x_i), the
// MLS factor D^-1, and the shift that makes floor(x + SHIFT) = base + 1 (the
// particle's cell for the cubic stencil, its nearest node for the quadratic).
template <int S> struct Stencil;
// weights(x, base, w) gives all S weights of a particle at x: the kernel's
// pieces as polynomials of t = x - (base + 1) where t is in the regular range
// (every particle whose stencil base came from its own position), else the
// kernel evaluated node by node (positions clamped far outside the grid).
template <> struct Stencil<4> {  // cubic, the reference's: nodes int(x) - 1 .. int(x) + 2
    static constexpr float DINV = 3.f, SHIFT = 0.f;
    __device__ static __forceinline__ int base(float x, int ext) { return stencil_base(x, ext); }
    __device__ static __forceinline__ float w(float d) { return bspline_n(d); }
    __device__ static __forceinline__ void weights(float x, int b, float* wt) {
        const float t = x - float(b + 1);
        if (t >= 0.f && t < 1.f) {
            const float s = 1.f - t, t2 = t * t, t3 = t2 * t;
            wt[0] = s * s * s * (1.f / 6.f);                           // (2 - |1 + t|)^3 / 6
            wt[1] = 0.5f * t3 - t2 + (2.f / 3.f);                       // |t|^3 / 2 - t^2 + 2/3
            wt[2] = (0.5f * t2 - 0.5f * t3) + (0.5f * t + (1.f / 6.f));  // the inner piece at 1 - t
            wt[3] = t3 * (1.f / 6.f);                                   // (2 - |t - 2|)^3 / 6
            return;
        }
#pragma unroll
        for (int o = 0; o < 4; ++o) wt[o] = bspline_n(x - float(b + o));
    }
};
template <> struct Stencil<3> {  // quadratic: nodes floor(x - 1/2) .. floor(x - 1/2) + 2
    static constexpr float DINV = 4.f, SHIFT = 0.5f;
    __device__ static __forceinline__ int base(float x, int ext) {
        return int(floorf(fminf(fmaxf(x, -8.f), float(ext) + 8.f) - 0.5f));
    }
    __device__ static __forceinline__ float w(float d) { return quad_n(d); }
    __device__ static __forceinline__ void weights(float x, int b, float* wt) {
        const float t = x - float(b + 1);
        if (t >= -0.5f && t < 0.5f) {
            const float a = 0.5f - t, c = 0.5f + t;
            wt[0] = 0.5f * a * a;
            wt[1] = 0.75f - t * t;
            wt[2] = 0.5f * c * c;
            return;
        }
#pragma unroll
        for (int o = 0; o < 3; ++o) wt[o] = quad_n(x - float(b + o));
    }
};

// ---------------------------------------------------------------------------
// P2G, one thread per particle.
// MLS (src/gpu/shaders/2d/p2g.glsl:29-92, 3d/p2g.glsl:31-96): per node
//   m_i += w m_p
//   p_i += w (m_p v_p + A_p (x_i - x_p)),  A_p = 3 m_p B_p - 3 dt V_p sigma_p
// which is the shader's  m (v + 3 B (-dist)) + w V sigma dist 3 dt  regrouped.
// CLASSIC (src/cpu/Grid.cpp:118-163): p_i += w m_p (v_p + 3 B_p (x_i - x_p)),
//   f_i += A_p^T grad w (A_p = V_p sigma_p, glm row-vector product).
// QUAD: the MLS sums on the quadratic stencil, A_p = 4 m_p B_p - 4 dt V_p sigma_p.
// Sums are int64 fixed point (exact, order independent).
template <int D, int FORM>
__global__ void __launch_bounds__(256) k_p2g_simple(Particles P, StepConsts C, unsigned long long* __restrict__ acc,
                                                    unsigned* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int n = P.n;
    float x[D], v[D], B[D * D], Fe[D * D];
#pragma unroll
    for (int k = 0; k < D; ++k) { x[k] = P.x[k * n + i]; v[k] = P.v[k * n + i]; }
#pragma unroll
    for (int k = 0; k < D * D; ++k) { B[k] = P.B[k * n + i]; Fe[k] = P.Fe[k * n + i]; }
    const float Jp = P.Jp[i];
    const float mass = P.mass ? P.mass[i] : P.mass_u;
    const float vol = P.vol ? P.vol[i] : P.vol_u;
    constexpr bool MLS = FORM != kClassic;
    constexpr int S = stencil_of(FORM);
    using St = Stencil<S>;
    if (MLS && vol == 0.f) return;

    float sig[D * D];
    if (vol != 0.f) hardened_stress_polar<D, math_form(FORM)>(Fe, Jp, C.mu0, C.la0, C.xi, sig);
    else {
#pragma unroll
        for (int k = 0; k < D * D; ++k) sig[k] = 0.f;
    }
    float A[D * D], mv[D];
#pragma unroll
    for (int r = 0; r < D; ++r) {
        mv[r] = mass * v[r];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            if (MLS) A[r * D + c] = St::DINV * mass * B[r * D + c] - St::DINV * C.dt * vol * sig[r * D + c];
            else A[r * D + c] = vol * sig[r * D + c];
        }
    }

    const int ext[3] = {C.W, C.H, C.Dp};
    int base[3] = {0, 0, 0};
    float wk[3][S], dwk[3][S], off[3][S];  // off = x_i - x_p per axis
#pragma unroll
    for (int k = 0; k < D; ++k) {
        base[k] = St::base(x[k], ext[k]);
#pragma unroll
        for (int o = 0; o < S; ++o) {
            const float dist = x[k] - float(base[k] + o);
            wk[k][o] = St::w(dist);
            dwk[k][o] = (FORM == kClassic) ? bspline_dn(dist) : 0.f;
            off[k][o] = -dist;
        }
    }
    const int lim[3] = {C.W, C.H, C.Dp};
    bool outside = false;
    constexpr int NACC = Layout<D, FORM>::NACC;
    const int nzs = (D == 3) ? S : 1;
#pragma unroll
    for (int a = 0; a < S; ++a) {
        const int ix = base[0] + a;
        if (ix < 0 || ix > lim[0]) { outside = true; continue; }
#pragma unroll
        for (int b = 0; b < S; ++b) {
            const int iy = base[1] + b;
            if (iy < 0 || iy > lim[1]) { outside = true; continue; }
#pragma unroll
            for (int c = 0; c < nzs; ++c) {
                const int iz = (D == 3) ? base[2] + c : 0;
                if (D == 3 && (iz < 0 || iz > lim[2])) { outside = true; continue; }
                const long long cid = ((long long)iz * C.ny + iy) * C.nx + ix;
                const float w = (D == 3) ? wk[0][a] * wk[1][b] * wk[2][c] : wk[0][a] * wk[1][b];
                const float d[3] = {off[0][a], off[1][b], D == 3 ? off[2][c] : 0.f};
                red_add(&acc[cid], to_fixed(w * mass, C.sm, status));
                if (MLS) {
#pragma unroll
                    for (int r = 0; r < D; ++r) {
                        float s = mv[r];
#pragma unroll
                        for (int k = 0; k < D; ++k) s += A[r * D + k] * d[k];
                        red_add(&acc[(1 + r) * C.nodes + cid], to_fixed(w * s, C.sp, status));
                    }
                } else {
                    float dw[3];
                    dw[0] = dwk[0][a] * wk[1][b];
                    dw[1] = wk[0][a] * dwk[1][b];
                    if (D == 3) { dw[0] *= wk[2][c]; dw[1] *= wk[2][c]; dw[2] = wk[0][a] * wk[1][b] * dwk[2][c]; }
#pragma unroll
                    for (int r = 0; r < D; ++r) {
                        float bd = 0.f, f = 0.f;
#pragma unroll
                        for (int k = 0; k < D; ++k) { bd += B[r * D + k] * d[k]; f += dw[k] * A[k * D + r]; }
                        red_add(&acc[(1 + r) * C.nodes + cid], to_fixed((w * mass) * (v[r] + 3.f * bd), C.sp, status));
                        red_add(&acc[(1 + D + r) * C.nodes + cid], to_fixed(f, C.sf, status));
                    }
                }
            }
        }
    }
    (void)NACC;
    if (outside) raise_flag(status, 4u);
}

// ---------------------------------------------------------------------------
// Wall response on one node. MLS: src/gpu/shaders/2d/grid_update.glsl:17-80
// (3D :19-86); CLASSIC: src/cpu/Grid.cpp:15-59 (same planes and order).
template <int D, int FORM>
__device__ __forceinline__ void collide(const StepConsts& C, const float* loc, const float* vel, float* vc, float* vf) {
    const float w = float(C.W), h = float(C.H), dd = float(C.Dp), m = C.margin;
    // plane point component along the normal's axis, normal sign, axis
    float pp[6];
    float ns[6];
    int ax[6];
    int nb;
    if (D == 2) {
        // right, bottom, left, top
        pp[0] = w - m; ns[0] = -1.f; ax[0] = 0;
        pp[1] = m;     ns[1] = 1.f;  ax[1] = 1;
        pp[2] = m;     ns[2] = 1.f;  ax[2] = 0;
        pp[3] = h - m; ns[3] = -1.f; ax[3] = 1;
        nb = 4;
    } else {
        // +x, -x, +y, -y, +z, -z
        pp[0] = w - m;  ns[0] = -1.f; ax[0] = 0;
        pp[1] = m;      ns[1] = 1.f;  ax[1] = 0;
        pp[2] = h - m;  ns[2] = -1.f; ax[2] = 1;
        pp[3] = m;      ns[3] = 1.f;  ax[3] = 1;
        pp[4] = dd - m; ns[4] = -1.f; ax[4] = 2;
        pp[5] = m;      ns[5] = 1.f;  ax[5] = 2;
        nb = 6;
    }
#pragma unroll
    for (int k = 0; k < D; ++k) vc[k] = vel[k];
    // the planes that acted, as bits in plane order (a mask rather than a
    // list, so that every index below is a compile-time constant)
    unsigned hit = 0u;
#pragma unroll
    for (int b = 0; b < 6; ++b) {
        if (b >= nb) break;
        const int a = ax[b];
        // n . (loc - P): only the normal's axis contributes (the other terms are 0 * x)
        const float dist = ns[b] * (loc[a] - pp[b]);
        const float test = ns[b] * ((loc[a] + C.dt * vc[a]) - pp[b]);
        const float delta = test - fminf(dist, 0.f);
        if (delta < 0.f) {
            if (FORM == kClassic) vc[a] -= (delta * ns[b]) / C.dt;
            else vc[a] -= (delta / C.dt) * ns[b];
            hit |= 1u << b;
        }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) vf[k] = vc[k];
#pragma unroll
    for (int b = 0; b < 6; ++b) {
        if (b >= nb) break;
        if (!((hit >> b) & 1u)) continue;
        const int a = ax[b];
        // vt = vc - n (n . vf)
        float vt[3];
#pragma unroll
        for (int k = 0; k < D; ++k) vt[k] = vc[k];
        vt[a] = vc[a] - ns[b] * (ns[b] * vf[a]);
        float vt2 = 0.f, dc2 = 0.f;
#pragma unroll
        for (int k = 0; k < D; ++k) { vt2 += vt[k] * vt[k]; const float e = vc[k] - vel[k]; dc2 += e * e; }
        const float vtn = sqrtf(vt2);
        if (vtn <= 1e-7f) continue;
        const float mag = fminf(vtn, C.friction * sqrtf(dc2));
#pragma unroll
        for (int k = 0; k < D; ++k) vf[k] -= mag * (vt[k] / vtn);
    }
}

// Grid update of one node from its summed fixed-point accumulators q (MLS:
// src/gpu/shaders/2d/grid_update.glsl:82-108, 3D :88-117; CLASSIC:
// src/cpu/Grid.cpp:165-184): node velocity after gravity (vc, after the wall
// planes; vf, after friction as well). Zero where the node mass is below 1e-6.
template <int D, int FORM>
__device__ __forceinline__ void grid_node_velocity(const StepConsts& C, const long long* q, long long ix, long long iy,
                                                   long long iz, unsigned* __restrict__ status, float* vc, float* vf) {
#pragma unroll
    for (int k = 0; k < 3; ++k) { vc[k] = 0.f; vf[k] = 0.f; }
    const float mass = __ll2float_rn(q[0]) * C.inv_sm;
    if (mass >= 1e-6f) {
        float vel[3] = {0.f, 0.f, 0.f};
        if (FORM != kClassic) {
#pragma unroll
            for (int k = 0; k < D; ++k) vel[k] = (__ll2float_rn(q[1 + k]) * C.inv_sp) / mass;
            vel[1] += C.gravity * C.dt;
        } else {
#pragma unroll
            for (int k = 0; k < D; ++k) {
                const float vk = (__ll2float_rn(q[1 + k]) * C.inv_sp) / mass;
                const float fk = (k == 1 ? C.gravity : 0.f) + (-(__ll2float_rn(q[1 + D + k]) * C.inv_sf) / mass);
                vel[k] = vk + fk * C.dt;
            }
        }
        float sp2 = 0.f;
#pragma unroll
        for (int k = 0; k < D; ++k) sp2 += vel[k] * vel[k];
        if (!(sp2 <= C.v_cap * C.v_cap)) raise_flag(status, (sp2 != sp2) ? 1u : 2u);
        const float loc[3] = {float(ix), float(iy), float(iz)};
        if (C.boundary == kBoundarySticky) {
            const int mm = int(C.margin);
            const bool wall = ix < mm || ix > C.W - mm || iy < mm || iy > C.H - mm ||
                              (D == 3 && (iz < mm || iz > C.Dp - mm));
#pragma unroll
            for (int k = 0; k < D; ++k) { vc[k] = wall ? 0.f : vel[k]; vf[k] = vc[k]; }
        } else {
            collide<D, FORM>(C, loc, vel, vc, vf);
        }
    }
}

// Grid update of one node of the global grid. Reads and clears the
// fixed-point accumulators (the reference's separate reset pass,
// reset.glsl:13-23, is fused here) and writes the velocities G2P gathers.
template <int D, int FORM>
__device__ __forceinline__ void grid_node_at(const StepConsts& C, unsigned long long* __restrict__ acc,
                                             float4* __restrict__ gv, unsigned* __restrict__ status, long long id,
                                             int ix, int iy, int iz) {
    constexpr int NACC = Layout<D, FORM>::NACC;
    long long q[NACC];
#pragma unroll
    for (int c = 0; c < NACC; ++c) {
        q[c] = (long long)acc[c * C.nodes + id];
        if (q[c] != 0) acc[c * C.nodes + id] = 0ull;
    }
    float vc[3], vf[3];
    grid_node_velocity<D, FORM>(C, q, ix, iy, iz, status, vc, vf);
    if (D == 2) {
        gv[id] = make_float4(vf[0], vf[1], vc[0], vc[1]);
    } else {
        // vc differs from vf only where a wall plane acted on the node: flag
        // those in .w and store their vc in the second half of the array, so
        // that the gather reads one float4 per node elsewhere.
        const bool hit = vc[0] != vf[0] || vc[1] != vf[1] || vc[2] != vf[2];
        gv[id] = make_float4(vf[0], vf[1], vf[2], hit ? 1.f : 0.f);
        if (hit) gv[C.nodes + id] = make_float4(vc[0], vc[1], vc[2], 0.f);
    }
}

// The same for a node given by its id alone.
template <int D, int FORM>
__device__ __forceinline__ void grid_node(const StepConsts& C, unsigned long long* __restrict__ acc,
                                          float4* __restrict__ gv, unsigned* __restrict__ status, long long id) {
    grid_node_at<D, FORM>(C, acc, gv, status, id, int(id % C.nx), int((id / C.nx) % C.ny),
                          int(id / ((long long)C.nx * C.ny)));
}

// 3D node velocities as grid_node stores them: vf, and vc (= vf unless flagged).
__device__ __forceinline__ void load_node3(const float4* __restrict__ gv, long long nodes, long long cid, float* vf,
                                           float* vc) {
    const float4 g = __ldg(&gv[cid]);
    vf[0] = g.x; vf[1] = g.y; vf[2] = g.z;
    if (g.w != 0.f) {
        const float4 h = __ldg(&gv[nodes + cid]);
        vc[0] = h.x; vc[1] = h.y; vc[2] = h.z;
    } else {
        vc[0] = g.x; vc[1] = g.y; vc[2] = g.z;
    }
}

// Dense grid update, one thread per node.
template <int D, int FORM>
__global__ void __launch_bounds__(256) k_grid_update(StepConsts C, unsigned long long* __restrict__ acc,
                                                     float4* __restrict__ gv, unsigned* __restrict__ status) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= C.nodes) return;
    grid_node<D, FORM>(C, acc, gv, status, id);
}

// ---------------------------------------------------------------------------
// Plasticity return map shared by every G2P variant (src/gpu/shaders/2d/
// g2p.glsl:73-93, 3d/g2p.glsl:73-104, src/cpu/Particles.cpp:64-106):
//   F_hat = (I + dt L) F_E;  U S V^T = svd(F_hat);  S' = max(clamp(S, 1-tc, 1+ts), 1e-6)
//   F_E' = U S' V^T;  J_p' = J_p prod(S / S')  (= det of V diag(S/S') V^T F_P)
// When every singular value of F_hat is inside [1-tc, 1+ts] (and det > 0),
// S' = S and the map returns F_hat and J_p unchanged; that case is proven
// first (in_elastic_band) and skips the SVD.
// The FP32 SVD is recomputed in FP64 when F_hat is near-degenerate
// (sigma_min^2 < 1e-2 sigma_max^2), where squaring in M^T M loses FP32 digits.
template <int D, int FORM>
__device__ __forceinline__ void plasticity(const StepConsts& C, const float* Fh, float* Fe_out, float& Jp,
                                           unsigned* status) {
    // Inside the elastic band the return map is the identity: no SVD.
    if (in_elastic_band<D>(Fh, 1.f - C.theta_c, 1.f + C.theta_s)) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) Fe_out[k] = Fh[k];
        return;
    }
    float U[D * D], S[D], V[D * D];
    svd<D, FORM>(Fh, U, S, V);
    float smin = fabsf(S[0]), smax = fabsf(S[0]);
#pragma unroll
    for (int k = 1; k < D; ++k) { smin = fminf(smin, fabsf(S[k])); smax = fmaxf(smax, fabsf(S[k])); }
    if (!(smin * smin >= 1e-2f * smax * smax)) {
        double Md[D * D], Ud[D * D], Sd[D], Vd[D * D];
#pragma unroll
        for (int k = 0; k < D * D; ++k) Md[k] = double(Fh[k]);
        svd<D, FORM, double>(Md, Ud, Sd, Vd);
#pragma unroll
        for (int k = 0; k < D * D; ++k) { U[k] = float(Ud[k]); V[k] = float(Vd[k]); }
#pragma unroll
        for (int k = 0; k < D; ++k) S[k] = float(Sd[k]);
        raise_flag(status, 8u);
    }
    const float t0 = 1.f - C.theta_c, t1 = 1.f + C.theta_s;
    float ratio = 1.f, Sc[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        Sc[k] = fmaxf(fminf(fmaxf(S[k], t0), t1), 1e-6f);
        ratio *= S[k] / Sc[k];
    }
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
        for (int c = 0; c < D; ++c) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) s += (U[r * D + k] * Sc[k]) * V[c * D + k];
            Fe_out[r * D + c] = s;
        }
    Jp *= ratio;
}

// G2P + APIC + plasticity, one thread per particle (MLS: src/gpu/shaders/2d/
// g2p.glsl:21-93, 3d/g2p.glsl:22-104; CLASSIC: src/cpu/Particles.cpp:133-216;
// QUAD: the MLS update on the quadratic stencil, F_hat = (I + 4 dt B) F_E).
// The new position  sum w (x_i + dt v_col)  is evaluated as
// x_p * sum(w) + sum w ((x_i - x_p) + dt v_col), with sum(w) taken as exactly 1
// when the whole stencil lies inside the grid (partition of unity): the same
// value in exact arithmetic, without rounding node coordinates of O(W) into
// every term. Where the reference skipped out-of-grid nodes the partial weight
// sum is kept, as there.
template <int D, int FORM>
__global__ void __launch_bounds__(256) k_g2p_simple(Particles P, StepConsts C, const float4* __restrict__ gv,
                                                    unsigned* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int n = P.n;
    constexpr int S = stencil_of(FORM);
    using St = Stencil<S>;
    float x[D];
#pragma unroll
    for (int k = 0; k < D; ++k) x[k] = P.x[k * n + i];
    const int ext[3] = {C.W, C.H, C.Dp};
    int base[3] = {0, 0, 0};
    float wk[3][S], dwk[3][S], off[3][S];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        base[k] = St::base(x[k], ext[k]);
#pragma unroll
        for (int o = 0; o < S; ++o) {
            const float dist = x[k] - float(base[k] + o);
            wk[k][o] = St::w(dist);
            dwk[k][o] = (FORM == kClassic) ? bspline_dn(dist) : 0.f;
            off[k][o] = -dist;
        }
    }
    float nv[D], nx[D], nB[D * D], gvel[D * D];
#pragma unroll
    for (int k = 0; k < D; ++k) { nv[k] = 0.f; nx[k] = 0.f; }
#pragma unroll
    for (int k = 0; k < D * D; ++k) { nB[k] = 0.f; gvel[k] = 0.f; }
    const int lim[3] = {C.W, C.H, C.Dp};
    const int nzs = (D == 3) ? S : 1;
    float wsum = 0.f;
    bool clipped = false;
    // CLASSIC grad v = sum v_col (x) grad w. With the whole stencil in the grid,
    // sum grad w = 0, so any constant may be taken off v_col first: the
    // particle's old velocity, which leaves small differences to sum instead
    // of ~|v| terms that cancel (the reference sums v_col itself; the exact
    // value is the same).
    float vref[3] = {0.f, 0.f, 0.f};
    if (FORM == kClassic) {
        bool whole = true;
#pragma unroll
        for (int k = 0; k < D; ++k) whole = whole && base[k] >= 0 && base[k] + (S - 1) <= lim[k];
        if (whole) {
#pragma unroll
            for (int k = 0; k < D; ++k) vref[k] = P.v[k * n + i];
        }
    }
#pragma unroll
    for (int a = 0; a < S; ++a) {
        const int ix = base[0] + a;
        if (ix < 0 || ix > lim[0]) { clipped = true; continue; }
#pragma unroll
        for (int b = 0; b < S; ++b) {
            const int iy = base[1] + b;
            if (iy < 0 || iy > lim[1]) { clipped = true; continue; }
#pragma unroll
            for (int c = 0; c < nzs; ++c) {
                const int iz = (D == 3) ? base[2] + c : 0;
                if (D == 3 && (iz < 0 || iz > lim[2])) { clipped = true; continue; }
                const long long cid = ((long long)iz * C.ny + iy) * C.nx + ix;
                const float w = (D == 3) ? wk[0][a] * wk[1][b] * wk[2][c] : wk[0][a] * wk[1][b];
                const float d[3] = {off[0][a], off[1][b], D == 3 ? off[2][c] : 0.f};
                wsum += w;
                float vf[3], vc[3];
                if (D == 2) {
                    const float4 g = gv[cid];
                    vf[0] = g.x; vf[1] = g.y; vc[0] = g.z; vc[1] = g.w;
                } else {
                    load_node3(gv, C.nodes, cid, vf, vc);
                }
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    nv[r] += vf[r] * w;
#pragma unroll
                    for (int k = 0; k < D; ++k) nB[r * D + k] += w * (vf[r] * d[k]);
                    nx[r] += (d[r] + C.dt * vc[r]) * w;
                }
                if (FORM == kClassic) {
                    float dw[3];
                    dw[0] = dwk[0][a] * wk[1][b];
                    dw[1] = wk[0][a] * dwk[1][b];
                    if (D == 3) { dw[0] *= wk[2][c]; dw[1] *= wk[2][c]; dw[2] = wk[0][a] * wk[1][b] * dwk[2][c]; }
#pragma unroll
                    for (int r = 0; r < D; ++r)
#pragma unroll
                        for (int k = 0; k < D; ++k) gvel[r * D + k] += (vc[r] - vref[r]) * dw[k];
                }
            }
        }
    }
    bool finite = true;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const float xn = (clipped ? x[k] * wsum : x[k]) + nx[k];
        P.v[k * n + i] = nv[k];
        P.x[k * n + i] = xn;
        finite = finite && isfinite(xn);
    }
#pragma unroll
    for (int k = 0; k < D * D; ++k) P.B[k * n + i] = nB[k];

    float Fe[D * D], A[D * D], Fh[D * D];
#pragma unroll
    for (int k = 0; k < D * D; ++k) {
        Fe[k] = P.Fe[k * n + i];
        const float L = (FORM != kClassic) ? St::DINV * nB[k] : gvel[k];
        A[k] = ((k % (D + 1)) == 0 ? 1.f : 0.f) + C.dt * L;
    }
    matmul<D>(A, Fe, Fh);
    float Jp = P.Jp[i];
    plasticity<D, math_form(FORM)>(C, Fh, Fe, Jp, status);
#pragma unroll
    for (int k = 0; k < D * D; ++k) P.Fe[k * n + i] = Fe[k];
    P.Jp[i] = Jp;
    if (!finite || !isfinite(Jp)) raise_flag(status, 1u);
}

// ---------------------------------------------------------------------------
// MLS affine matrix of one particle, the per-particle factor of the P2G
// scatter (src/gpu/shaders/2d/p2g.glsl:44-90): A = 3 m B - 3 dt V sigma(F_E, J_p),
// so that a node receives w (m v + A (x_i - x_p)). Computed by G2P for the next
// step (and by k_prepare_affine after any state upload), always with this one
// function, so the value depends on (B, F_E, J_p, m, V) alone. On the
// quadratic stencil (S = 3) the factor is D^-1 = 4 instead of 3.
template <int D, int S = 4>
__device__ __forceinline__ void mls_affine(const StepConsts& C, const float* B, const float* Fe, float Jp, float mass,
                                           float vol, float* A) {
    constexpr float K = Stencil<S>::DINV;
    float sig[D * D];
    hardened_stress_fast<D, kMLS>(Fe, Jp, C.mu0, C.la0, C.xi, sig);
#pragma unroll
    for (int k = 0; k < D * D; ++k) A[k] = K * mass * B[k] - K * C.dt * vol * sig[k];
}

template <int D, int S = 4>
__global__ void __launch_bounds__(256) k_prepare_affine(Particles P, StepConsts C) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int n = P.n;
    float B[D * D], Fe[D * D], A[D * D];
#pragma unroll
    for (int k = 0; k < D * D; ++k) { B[k] = P.B[k * n + i]; Fe[k] = P.Fe[k * n + i]; }
    mls_affine<D, S>(C, B, Fe, P.Jp[i], P.mass ? P.mass[i] : P.mass_u, P.vol ? P.vol[i] : P.vol_u, A);
#pragma unroll
    for (int k = 0; k < D * D; ++k) P.A[k * n + i] = A[k];
}

// ---------------------------------------------------------------------------
// G2P split in two for the MLS path. k_g2p_gather does the gather, APIC
// update and the return map of every particle whose trial F is proven inside
// the elastic band by the FP32 Gershgorin test (the map is then the identity),
// and writes the next step's affine matrix; the others are queued with their
// trial F for k_g2p_plastic, which runs the full return map (FP64 band test,
// else the SVD) and then writes theirs. The split keeps the SVD's registers out
// of the gather kernel so that it runs at higher occupancy.
// Queue entry already finished by the learned return map (never a slot: the
// clipped-stencil entries are -1 - slot >= -n).
constexpr int kQueueDone = -2147483647 - 1;

struct SlowQueue {
    int* list;    // slots needing the full return map
    int* count;   // device scalar
    float* fh;    // trial F per queue entry, [D*D][capacity]
    int capacity;
    // fused path: the 32-slot windows holding queued particles, as (first
    // slot, lane mask of the queued slots); their P2G runs after the return map
    int2* win;
    int* nwin;    // device scalar (count[1])
    int win_capacity;
};

// Element a of an S-vector held in registers, for a loop index the compiler
// does not unroll.
template <int S> __device__ __forceinline__ float pick(const float* v, int a) {
    if constexpr (S == 4) return a == 0 ? v[0] : a == 1 ? v[1] : a == 2 ? v[2] : v[3];
    else return a == 0 ? v[0] : a == 1 ? v[1] : v[2];
}

// Sum of an S-vector, pairwise for S = 4.
template <int S> __device__ __forceinline__ float sum_s(const float* v) {
    if constexpr (S == 4) return (v[0] + v[1]) + (v[2] + v[3]);
    else return (v[0] + v[1]) + v[2];
}

// Interior gather: every stencil node inside the grid. The sums
//   v = sum w vf,  B = sum w vf (x_i - x_p)^T,  x' = x + sum w (x_i - x_p) + dt sum w vc
// are contracted axis by axis (z, then y, then x) with the separable weights.
template <int D, int S = 4>
__device__ __forceinline__ void gather_interior(const StepConsts& C, const float4* __restrict__ gv, const int* base,
                                                const float (*wk)[S], const float (*off)[S], float* nv, float* nB,
                                                float* nx) {
    float wd[3][S];
#pragma unroll
    for (int k = 0; k < D; ++k)
#pragma unroll
        for (int o = 0; o < S; ++o) wd[k][o] = wk[k][o] * off[k][o];
    const long long sy = C.nx, sz = (long long)C.nx * C.ny;
    const long long c0 = (D == 3 ? base[2] * sz : 0) + base[1] * sy + base[0];
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
                // vc = vf at every node the wall planes left alone (flag .w = 0):
                // the vc sum is then the vf sum; flagged nodes are handled below.
                float Pv[3] = {0.f, 0.f, 0.f}, Pd[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int c = 0; c < S; ++c) {
                    const long long cid = c0 + a + b * sy + c * sz;
                    const float4 g = __ldg(&gv[cid]);
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
                const long long cid = c0 + a + b * sy;
                const float4 g = __ldg(&gv[cid]);
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
            // a stencil node was moved by a wall plane: the vc sum, in the same
            // order as the vf sum above
#pragma unroll 1
            for (int a = 0; a < S; ++a) {
                float Qc[3] = {0.f, 0.f, 0.f};
#pragma unroll 1
                for (int b = 0; b < S; ++b) {
                    float Pc[3] = {0.f, 0.f, 0.f};
#pragma unroll
                    for (int c = 0; c < S; ++c) {
                        float f[3], g[3];
                        load_node3(gv, C.nodes, c0 + a + b * sy + c * sz, f, g);
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
    // sum w (x_i - x_p) per axis is separable: (sum wd_k) prod_{l != k} (sum w_l)
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

// General gather (stencil partly outside the grid: those nodes are skipped,
// as in the reference, and the partial weight sum is returned).
template <int D, int S = 4>
__device__ __forceinline__ float gather_clipped(const StepConsts& C, const float4* __restrict__ gv, const int* base,
                                             const float (*wk)[S], const float (*off)[S], float* nv, float* nB,
                                             float* nx) {
    const int ext[3] = {C.W, C.H, C.Dp};
#pragma unroll
    for (int k = 0; k < D; ++k) { nv[k] = 0.f; nx[k] = 0.f; }
#pragma unroll
    for (int k = 0; k < D * D; ++k) nB[k] = 0.f;
    float wsum = 0.f;
    const int nzs = (D == 3) ? S : 1;
    for (int a = 0; a < S; ++a) {
        const int ix = base[0] + a;
        if (ix < 0 || ix > ext[0]) continue;
        for (int b = 0; b < S; ++b) {
            const int iy = base[1] + b;
            if (iy < 0 || iy > ext[1]) continue;
            for (int c = 0; c < nzs; ++c) {
                const int iz = (D == 3) ? base[2] + c : 0;
                if (D == 3 && (iz < 0 || iz > ext[2])) continue;
                const long long cid = ((long long)iz * C.ny + iy) * C.nx + ix;
                const float w = (D == 3) ? wk[0][a] * wk[1][b] * wk[2][c] : wk[0][a] * wk[1][b];
                const float d[3] = {off[0][a], off[1][b], D == 3 ? off[2][c] : 0.f};
                wsum += w;
                float vf[3], vc[3];
                if (D == 2) {
                    const float4 g = __ldg(&gv[cid]);
                    vf[0] = g.x; vf[1] = g.y; vc[0] = g.z; vc[1] = g.w;
                } else {
                    load_node3(gv, C.nodes, cid, vf, vc);
                }
                for (int r = 0; r < D; ++r) {
                    const float wv = w * vf[r];
                    nv[r] += wv;
                    for (int k = 0; k < D; ++k) nB[r * D + k] += wv * d[k];
                    nx[r] += (d[r] + C.dt * vc[r]) * w;
                }
            }
        }
    }
    return wsum;
}

__device__ __forceinline__ int queue_slot(const SlowQueue& Q) {
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31, leader = __ffs(act) - 1;
    int slot = 0;
    if (lane == leader) slot = atomicAdd(Q.count, __popc(act));
    return __shfl_sync(act, slot, leader) + __popc(act & ((1u << lane) - 1));
}

#ifndef MPM_G2P_MIN_BLOCKS
#define MPM_G2P_MIN_BLOCKS 4
#endif
#ifndef MPM_G2P_MIN_BLOCKS_Q
#define MPM_G2P_MIN_BLOCKS_Q 4
#endif
template <int D, int S = 4>
__global__ void __launch_bounds__(256, S == 3 ? MPM_G2P_MIN_BLOCKS_Q : MPM_G2P_MIN_BLOCKS) k_g2p_gather(Particles P, StepConsts C, const float4* __restrict__ gv,
                                                       SlowQueue Q, unsigned* __restrict__ status) {
    using St = Stencil<S>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int n = P.n;
    float x[D];
#pragma unroll
    for (int k = 0; k < D; ++k) x[k] = P.x[k * n + i];
    int base[3] = {0, 0, 0};
    float wk[3][S], off[3][S];
    bool interior = true;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int ext = k == 0 ? C.W : (k == 1 ? C.H : C.Dp);
        base[k] = St::base(x[k], ext);
        interior = interior && base[k] >= 0 && base[k] + (S - 1) <= ext;
        St::weights(x[k], base[k], wk[k]);
#pragma unroll
        for (int o = 0; o < S; ++o) off[k][o] = float(base[k] + o) - x[k];
    }
    if (!interior) {  // stencil partly outside the grid: the general kernel does it all
        Q.list[queue_slot(Q)] = -1 - i;
        return;
    }
    float nv[D], nx[D], nB[D * D];
    gather_interior<D, S>(C, gv, base, wk, off, nv, nB, nx);
    bool finite = true;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const float xn = x[k] + nx[k];
        P.v[k * n + i] = nv[k];
        P.x[k * n + i] = xn;
        finite = finite && isfinite(xn);
    }
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
        const float mass = P.mass ? P.mass[i] : P.mass_u, vol = P.vol ? P.vol[i] : P.vol_u;
#pragma unroll
        for (int k = 0; k < D * D; ++k) {
            P.Fe[k * n + i] = Fh[k];
            P.A[k * n + i] = St::DINV * mass * nB[k] - St::DINV * C.dt * vol * sig[k];
        }
    } else {
        const int slot = queue_slot(Q);
        Q.list[slot] = i;
#pragma unroll
        for (int k = 0; k < D * D; ++k) Q.fh[k * Q.capacity + slot] = Fh[k];
    }
    if (!finite) raise_flag(status, 1u);
}

// Optional log of exact return-map pairs (F_hat[9], J_p, F_E'[9], J_p') for
// training the learned surrogate; appended while room is left.
struct PairLog {
    float* data;            // [capacity][20]
    unsigned long long* n;  // device counter (may exceed capacity: excess dropped)
    long long capacity;
};

// One queued particle: the full return map for an out-of-band trial F (entry
// i), or the whole G2P with a grid-clipped stencil (entry -1 - i).
template <int D, int S = 4>
__device__ __forceinline__ void g2p_queued_exact(const Particles& P, const StepConsts& C, const float4* __restrict__ gv,
                                                 const SlowQueue& Q, int e, unsigned* __restrict__ status,
                                                 PairLog L = PairLog{nullptr, nullptr, 0}) {
    const int n = P.n;
    const int entry = Q.list[e];
    const int i = entry >= 0 ? entry : -1 - entry;
    float Fh[D * D], Fe[D * D], B[D * D], A[D * D];
    if (entry >= 0) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) { Fh[k] = Q.fh[k * Q.capacity + e]; B[k] = P.B[k * n + i]; }
    } else {
        float x[D];
#pragma unroll
        for (int k = 0; k < D; ++k) x[k] = P.x[k * n + i];
        int base[3] = {0, 0, 0};
        float wk[3][S], off[3][S];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const int ext = k == 0 ? C.W : (k == 1 ? C.H : C.Dp);
            base[k] = Stencil<S>::base(x[k], ext);
#pragma unroll
            for (int o = 0; o < S; ++o) {
                const float dist = x[k] - float(base[k] + o);
                wk[k][o] = Stencil<S>::w(dist);
                off[k][o] = -dist;
            }
        }
        float nv[D], nx[D];
        const float wsum = gather_clipped<D, S>(C, gv, base, wk, off, nv, B, nx);
        bool finite = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float xn = x[k] * wsum + nx[k];
            P.v[k * n + i] = nv[k];
            P.x[k * n + i] = xn;
            finite = finite && isfinite(xn);
        }
        if (!finite) raise_flag(status, 1u);
#pragma unroll
        for (int k = 0; k < D * D; ++k) { P.B[k * n + i] = B[k]; Fe[k] = P.Fe[k * n + i]; }
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) {
                float s = Fe[r * D + c];
#pragma unroll
                for (int k = 0; k < D; ++k) s += (C.dt * Stencil<S>::DINV * B[r * D + k]) * Fe[k * D + c];
                Fh[r * D + c] = s;
            }
    }
    const float Jp0 = P.Jp[i];
    float Jp = Jp0;
    plasticity<D, kMLS>(C, Fh, Fe, Jp, status);
#pragma unroll
    for (int k = 0; k < D * D; ++k) P.Fe[k * n + i] = Fe[k];
    P.Jp[i] = Jp;
    mls_affine<D, S>(C, B, Fe, Jp, P.mass ? P.mass[i] : P.mass_u, P.vol ? P.vol[i] : P.vol_u, A);
#pragma unroll
    for (int k = 0; k < D * D; ++k) P.A[k * n + i] = A[k];
    if (!isfinite(Jp)) raise_flag(status, 1u);
    if (D == 3 && L.data && entry >= 0) {
        const unsigned long long slot = atomicAdd(L.n, 1ull);
        if ((long long)slot < L.capacity) {
            float* d = L.data + slot * 20;
#pragma unroll
            for (int k = 0; k < 9; ++k) { d[k] = Fh[k]; d[10 + k] = Fe[k]; }
            d[9] = Jp0;
            d[19] = Jp;
        }
    }
}

template <int D, int S = 4>
__global__ void __launch_bounds__(256) k_g2p_plastic(Particles P, StepConsts C, const float4* __restrict__ gv,
                                                     SlowQueue Q, PairLog L, unsigned* __restrict__ status) {
    const int m = *Q.count;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x)
        if (Q.list[e] != kQueueDone) g2p_queued_exact<D, S>(P, C, gv, Q, e, status, L);
}

// ---------------------------------------------------------------------------
// Import / export between the caller's interleaved per-particle arrays (in
// creation order) and the device SoA (in slot order; slot s holds particle id[s]).
static __global__ void k_export_soa(const float* __restrict__ soa, int comps, int n, const int* __restrict__ id,
                             float* __restrict__ aos) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = id ? id[s] : s;
    for (int c = 0; c < comps; ++c) aos[(long long)p * comps + c] = soa[(long long)c * n + s];
}

static __global__ void k_import_soa(float* __restrict__ soa, int comps, int n, const int* __restrict__ id,
                             const float* __restrict__ aos) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = id ? id[s] : s;
    for (int c = 0; c < comps; ++c) soa[(long long)c * n + s] = aos[(long long)p * comps + c];
}

}  // namespace mpm
