// TEST INFRASTRUCTURE — the oracle. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load this library; the product path never does.
//
// A CPU restatement of one MPM step of the reference, templated on the real type:
//   * double: the FP64 oracle the CUDA solver is checked against;
//   * float (+ OpenMP): the multi-core CPU baseline ("port") timed by bench.py.
//
// Three formulations, all in the reference's grid units (dx = 1, node i at x = i):
//   MLS     — the reference GPU path, src/gpu/shaders/{2d,3d}/{common,p2g,
//             grid_update,g2p}.glsl (force folded into momentum, C = 3 B).
//   CLASSIC — the reference CPU path, src/cpu/{Grid,Particles}.cpp (separate
//             grid force f = sum grad(w) A_p, grad(v) = sum v_col (x) grad(w),
//             Eigen JacobiSVD conventions). 2D only, as in the reference.
//   QUAD    — the MLS step on the quadratic B-spline stencil (3 nodes per axis
//             from floor(x - 1/2), C = 4 B, stress factor 4); the reference has
//             no quadratic variant, so this is the MLS restatement with the
//             textbook quadratic kernel and D^-1 = 4 substituted.
//
// Every function cites the reference lines it restates. Matrices are row-major
// (M[r*D+c]); GLSL mat constructors are column-major and are translated here.
//
// Parity of CLASSIC is pinned against the reference's own CPU code compiled
// from its sources (oracle/_ref/refcpu_driver, fixtures in tests/golden/).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

enum { MLS = 0, CLASSIC = 1, QUAD = 2 };
enum { BOUNDARY_FRICTION = 0, BOUNDARY_STICKY = 1 };

template <typename R> struct Params {
    int dim, width, height, depth, formulation, boundary;
    R margin, dt, gravity, friction, theta_c, theta_s, xi, mu, lambda;
};

// ---------------------------------------------------------------------------
// Cubic B-spline, src/gpu/shaders/2d/common.glsl:43-69 (= src/cpu/Grid.h:86-116)
// (the shader's pow form, so that the FP32 instantiation rounds as the shader does)
template <typename R> inline R bspline_n(R x) {
    R a = std::fabs(x);
    if (a < R(1)) return (R(0.5) * std::pow(a, R(3))) - std::pow(a, R(2)) + R(2) / R(3);
    if (a < R(2)) return std::pow(R(2) - a, R(3)) / R(6);
    return R(0);
}
// Quadratic B-spline (QUAD): 3/4 - x^2 for |x| < 1/2, (3/2 - |x|)^2 / 2 for |x| < 3/2.
template <typename R> inline R quad_n(R x) {
    R a = std::fabs(x);
    if (a < R(0.5)) return R(0.75) - a * a;
    if (a < R(1.5)) { R t = R(1.5) - a; return R(0.5) * t * t; }
    return R(0);
}

// Stencil of a formulation: first node per axis, nodes per axis, weight, D^-1.
inline int stencil_nodes(int form) { return form == QUAD ? 3 : 4; }
template <typename R> inline int stencil_first(R x, int form) {
    return form == QUAD ? int(std::floor(x - R(0.5))) : int(x) - 1;
}
template <typename R> inline R stencil_w(R d, int form) { return form == QUAD ? quad_n(d) : bspline_n(d); }
template <typename R> inline R stencil_dinv(int form) { return form == QUAD ? R(4) : R(3); }

template <typename R> inline R bspline_dn(R x) {
    R a = std::fabs(x);
    if (a < R(1)) return R(1.5) * a * x - R(2) * x;
    if (a < R(2)) return R(-0.5) * a * x + R(2) * x - (R(2) * x) / a;
    return R(0);
}

// ---------------------------------------------------------------------------
// Small dense helpers (row-major).
template <int D, typename R> inline void matmul(const R* A, const R* B, R* C) {
    R t[D * D];
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            R s = 0;
            for (int k = 0; k < D; ++k) s += A[i * D + k] * B[k * D + j];
            t[i * D + j] = s;
        }
    std::memcpy(C, t, sizeof(t));
}
template <int D, typename R> inline void transpose(const R* A, R* T) {
    R t[D * D];
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) t[j * D + i] = A[i * D + j];
    std::memcpy(T, t, sizeof(t));
}
template <int D, typename R> inline R det(const R* A) {
    if (D == 2) return A[0] * A[3] - A[1] * A[2];
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
}

// ---------------------------------------------------------------------------
// 2x2 SVD, src/gpu/shaders/2d/common.glsl:2-37 (eigen-decomposition of M^T M by
// one analytic rotation; a reflection is folded into the sign of Sigma[1]).
template <typename R> void svd2_glsl(const R* M, R* U, R* S, R* V) {
    R a = M[0] * M[0] + M[2] * M[2];  // (M^T M)_00
    R b = M[0] * M[1] + M[2] * M[3];  // (M^T M)_01
    R d = M[1] * M[1] + M[3] * M[3];  // (M^T M)_11
    R theta = (std::fabs(b) < R(1e-10) && std::fabs(a - d) < R(1e-10)) ? R(0) : R(0.5) * std::atan2(R(2) * b, a - d);
    R ct = std::cos(theta), st = std::sin(theta);
    V[0] = ct; V[1] = -st; V[2] = st; V[3] = ct;  // GLSL mat2(ct, st, -st, ct)
    R MtM[4] = {a, b, b, d}, Vt[4], tmp[4], dg[4];
    transpose<2>(V, Vt);
    matmul<2>(Vt, MtM, tmp);
    matmul<2>(tmp, V, dg);
    S[0] = std::sqrt(std::max(dg[0], R(1e-12)));
    S[1] = std::sqrt(std::max(dg[3], R(1e-12)));
    R MV[4];
    matmul<2>(M, V, MV);
    // U = M V diag(1 / Sigma), the reciprocals formed first as in the shader
    const R i0 = R(1) / S[0], i1 = R(1) / S[1];
    for (int r = 0; r < 2; ++r) { U[r * 2 + 0] = MV[r * 2 + 0] * i0; U[r * 2 + 1] = MV[r * 2 + 1] * i1; }
    if (det<2>(U) < R(0)) { U[1] = -U[1]; U[3] = -U[3]; S[1] = -S[1]; }
}

// 3x3 SVD, src/gpu/shaders/3d/common.glsl:8-105: 6 cyclic Jacobi sweeps over
// (0,1), (0,2), (1,2) on S = M^T M, then U = M V Sigma^-1, reflection folded
// into Sigma[2].
template <typename R> inline void schur_decomp(R app, R apq, R aqq, R& c, R& s) {  // :8-22
    if (std::fabs(apq) < R(1e-10)) { c = R(1); s = R(0); return; }
    R tau = (aqq - app) / (R(2) * apq);
    R stt = std::sqrt(R(1) + tau * tau);
    R tn = R(1) / (std::fabs(tau) + stt);
    if (tau < R(0)) tn = -tn;
    c = R(1) / std::sqrt(R(1) + tn * tn);
    s = tn * c;
}
template <typename R> inline void jacobi_rot_cols(R* A, int p, int q, R c, R s) {  // :25-31 (columns)
    for (int r = 0; r < 3; ++r) {
        R ap = A[r * 3 + p], aq = A[r * 3 + q];
        A[r * 3 + p] = c * ap - s * aq;
        A[r * 3 + q] = s * ap + c * aq;
    }
}
template <typename R> inline void jacobi_rot_sym(R* S, int p, int q, R c, R s) {  // :34-54
    R Spp = S[p * 3 + p], Sqq = S[q * 3 + q], Spq = S[p * 3 + q];
    S[p * 3 + p] = c * c * Spp - R(2) * s * c * Spq + s * s * Sqq;
    S[q * 3 + q] = s * s * Spp + R(2) * s * c * Spq + c * c * Sqq;
    S[p * 3 + q] = R(0);
    S[q * 3 + p] = R(0);
    for (int i = 0; i < 3; ++i) {
        if (i == p || i == q) continue;
        R Sip = S[i * 3 + p], Siq = S[i * 3 + q];
        S[i * 3 + p] = c * Sip - s * Siq;
        S[p * 3 + i] = S[i * 3 + p];
        S[i * 3 + q] = s * Sip + c * Siq;
        S[q * 3 + i] = S[i * 3 + q];
    }
}
template <typename R> void svd3_glsl(const R* M, R* U, R* Sig, R* V) {
    R Mt[9], S[9];
    transpose<3>(M, Mt);
    matmul<3>(Mt, M, S);
    for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? R(1) : R(0);
    const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
    for (int sweep = 0; sweep < 6; ++sweep)
        for (int r = 0; r < 3; ++r) {
            R c, s;
            schur_decomp(S[P[r] * 3 + P[r]], S[P[r] * 3 + Q[r]], S[Q[r] * 3 + Q[r]], c, s);
            jacobi_rot_sym(S, P[r], Q[r], c, s);
            jacobi_rot_cols(V, P[r], Q[r], c, s);
        }
    for (int i = 0; i < 3; ++i) Sig[i] = std::sqrt(std::max(S[i * 4], R(1e-12)));
    R MV[9];
    matmul<3>(M, V, MV);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) U[r * 3 + c] = MV[r * 3 + c] * (R(1) / Sig[c]);
    if (det<3>(U) < R(0)) { U[2] = -U[2]; U[5] = -U[5]; U[8] = -U[8]; Sig[2] = -Sig[2]; }
}

// 2x2 two-sided Jacobi SVD with Eigen 3.4 JacobiSVD conventions (singular
// values >= 0, descending): the decomposition the reference CPU path calls at
// src/cpu/Particles.cpp:31-32,73-78 (algorithm: external/eigen-3.4.0/Eigen/
// src/SVD/JacobiSVD.h:666-780, Eigen/src/misc/RealSvd2x2.h:18-49).
template <typename R> void svd2_eigen(const R* A, R* U, R* S, R* V) {
    struct Rot { R c, s; };
    auto rot_t = [](Rot j) { return Rot{j.c, -j.s}; };
    auto rot_mul = [](Rot a, Rot b) { return Rot{a.c * b.c - a.s * b.s, a.c * b.s + a.s * b.c}; };
    auto pair = [](R& x, R& y, Rot j) { R xi = x, yi = y; x = j.c * xi + j.s * yi; y = -j.s * xi + j.c * yi; };
    auto left = [&](R* m, int p, int q, Rot j) { for (int k = 0; k < 2; ++k) pair(m[p * 2 + k], m[q * 2 + k], j); };
    auto right = [&](R* m, int p, int q, Rot j) { Rot t = rot_t(j); for (int k = 0; k < 2; ++k) pair(m[k * 2 + p], m[k * 2 + q], t); };
    const R eps = std::numeric_limits<R>::epsilon(), tiny = std::numeric_limits<R>::min();
    R scale = std::max(std::max(std::fabs(A[0]), std::fabs(A[1])), std::max(std::fabs(A[2]), std::fabs(A[3])));
    for (int i = 0; i < 4; ++i) { U[i] = (i % 3 == 0) ? R(1) : R(0); V[i] = U[i]; }
    if (!std::isfinite(scale)) { S[0] = S[1] = std::numeric_limits<R>::quiet_NaN(); return; }
    if (scale == R(0)) scale = R(1);
    R w[4] = {A[0] / scale, A[1] / scale, A[2] / scale, A[3] / scale};
    R maxd = std::max(std::fabs(w[0]), std::fabs(w[3]));
    for (int guard = 0; guard < 64; ++guard) {
        const int p = 1, q = 0;
        R thr = std::max(tiny, R(2) * eps * maxd);
        if (!(std::fabs(w[p * 2 + q]) > thr || std::fabs(w[q * 2 + p]) > thr)) break;
        R m[4] = {w[p * 2 + p], w[p * 2 + q], w[q * 2 + p], w[q * 2 + q]};
        R t = m[0] + m[3], d = m[2] - m[1];
        Rot rot1{R(1), R(0)};
        if (!(std::fabs(d) < tiny)) { R u = t / d, tmp = std::sqrt(R(1) + u * u); rot1 = Rot{u / tmp, R(1) / tmp}; }
        left(m, 0, 1, rot1);
        Rot jr{R(1), R(0)};
        R deno = R(2) * std::fabs(m[1]);
        if (!(deno < tiny)) {
            R tau = (m[0] - m[3]) / deno, ww = std::sqrt(tau * tau + R(1));
            R tt = tau > R(0) ? R(1) / (tau + ww) : R(1) / (tau - ww);
            R sg = tt > R(0) ? R(1) : R(-1), n = R(1) / std::sqrt(tt * tt + R(1));
            jr = Rot{n, -sg * (m[1] / std::fabs(m[1])) * std::fabs(tt) * n};
        }
        Rot jl = rot_mul(rot1, rot_t(jr));
        left(w, p, q, jl);
        right(U, p, q, rot_t(jl));
        right(w, p, q, jr);
        right(V, p, q, jr);
        maxd = std::max(maxd, std::max(std::fabs(w[p * 2 + p]), std::fabs(w[q * 2 + q])));
    }
    for (int i = 0; i < 2; ++i) {
        R d = w[i * 3];
        S[i] = std::fabs(d);
        if (d < R(0)) { U[i] = -U[i]; U[2 + i] = -U[2 + i]; }
    }
    S[0] *= scale; S[1] *= scale;
    if (S[1] > S[0]) {
        std::swap(S[0], S[1]);
        std::swap(U[0], U[1]); std::swap(U[2], U[3]);
        std::swap(V[0], V[1]); std::swap(V[2], V[3]);
    }
}

template <int D, typename R> inline void svd(const R* M, R* U, R* S, R* V, int formulation) {
    if (D == 2) {
        if (formulation == CLASSIC) svd2_eigen(M, U, S, V);
        else svd2_glsl(M, U, S, V);
    } else {
        svd3_glsl(M, U, S, V);
    }
}

// ---------------------------------------------------------------------------
// Kirchhoff-type stress with Stomakhin hardening, src/gpu/shaders/2d/p2g.glsl:
// 44-59 (3d/p2g.glsl:46-61; CPU: src/cpu/Particles.cpp:21-48):
//   sigma = 2 mu(J_p) (F_E - R) F_E^T + lambda(J_p) (J_e - 1) J_e I.
template <int D, typename R> void stress(const Params<R>& p, const R* Fe, const R* Fp, R* out) {
    R Je = det<D>(Fe), Jp = det<D>(Fp);
    R U[D * D], S[D], V[D * D], Vt[D * D], Rm[D * D];
    svd<D>(Fe, U, S, V, p.formulation);
    transpose<D>(V, Vt);
    matmul<D>(U, Vt, Rm);
    R h = std::exp(p.xi * (R(1) - Jp));
    R mu = p.mu * h, la = p.lambda * h;
    // evaluated in glm's order, as both reference paths write it:
    // ((2 mu) (F - R)) F^T + ((lambda (J_e - 1)) J_e) I
    const R two_mu = R(2) * mu, dg = (la * (Je - R(1))) * Je;
    R FmR[D * D], FeT[D * D], P[D * D];
    for (int i = 0; i < D * D; ++i) FmR[i] = two_mu * (Fe[i] - Rm[i]);
    transpose<D>(Fe, FeT);
    matmul<D>(FmR, FeT, P);
    for (int i = 0; i < D * D; ++i) out[i] = P[i] + ((i % (D + 1) == 0) ? dg : R(0));
}

// ---------------------------------------------------------------------------
// Wall planes and their inward normals: src/gpu/shaders/2d/grid_update.glsl:
// 22-33 (right, bottom, left, top; = src/cpu/Grid.cpp:62-89) and
// 3d/grid_update.glsl:24-39 (+x, -x, +y, -y, +z, -z).
template <int D, typename R> int wall_planes(const Params<R>& p, R P[][3], R Nn[][3]) {
    R w = R(p.width), h = R(p.height), d = R(p.depth), m = p.margin;
    if (D == 2) {
        const R pts[4][2] = {{w - m, m}, {m, m}, {m, h - m}, {w - m, h - m}};
        const R nrm[4][2] = {{-1, 0}, {0, 1}, {1, 0}, {0, -1}};
        for (int b = 0; b < 4; ++b) for (int k = 0; k < 2; ++k) { P[b][k] = pts[b][k]; Nn[b][k] = nrm[b][k]; }
        return 4;
    }
    const R pts[6][3] = {{w - m, 0, 0}, {m, 0, 0}, {0, h - m, 0}, {0, m, 0}, {0, 0, d - m}, {0, 0, m}};
    const R nrm[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int b = 0; b < 6; ++b) for (int k = 0; k < 3; ++k) { P[b][k] = pts[b][k]; Nn[b][k] = nrm[b][k]; }
    return 6;
}

// Predictive wall separation + Coulomb friction on one node:
// src/gpu/shaders/2d/grid_update.glsl:17-80 (3D :19-86; CPU src/cpu/Grid.cpp:15-59).
template <int D, typename R> void collide(const Params<R>& p, const R* loc, const R* vel, R* vcol, R* vfric) {
    R P[6][3], Nn[6][3];
    int nb = wall_planes<D>(p, P, Nn);
    int hit[6], nh = 0;
    for (int k = 0; k < D; ++k) vcol[k] = vel[k];
    for (int b = 0; b < nb; ++b) {
        R dist = 0, test = 0;
        for (int k = 0; k < D; ++k) {
            dist += Nn[b][k] * (loc[k] - P[b][k]);
            test += Nn[b][k] * ((loc[k] + p.dt * vcol[k]) - P[b][k]);
        }
        R delta = test - std::min(dist, R(0));
        if (delta < R(0)) {
            for (int k = 0; k < D; ++k) {
                if (p.formulation == CLASSIC) vcol[k] -= (delta * Nn[b][k]) / p.dt;
                else vcol[k] -= (delta / p.dt) * Nn[b][k];
            }
            hit[nh++] = b;
        }
    }
    for (int k = 0; k < D; ++k) vfric[k] = vcol[k];
    for (int c = 0; c < nh; ++c) {
        const R* n = Nn[hit[c]];
        R ndotf = 0;
        for (int k = 0; k < D; ++k) ndotf += n[k] * vfric[k];
        R vt[3], vtn2 = 0, dc2 = 0;
        for (int k = 0; k < D; ++k) { vt[k] = vcol[k] - n[k] * ndotf; vtn2 += vt[k] * vt[k]; }
        R vtn = std::sqrt(vtn2);
        if (vtn <= R(1e-7)) continue;
        for (int k = 0; k < D; ++k) { R dk = vcol[k] - vel[k]; dc2 += dk * dk; }
        R mag = std::min(vtn, p.friction * std::sqrt(dc2));
        for (int k = 0; k < D; ++k) vfric[k] -= mag * (vt[k] / vtn);
    }
}

// ---------------------------------------------------------------------------
template <int D, typename R> struct Grid {
    int64_t nx, ny, nz, nodes;
    std::vector<R> mass, mom, force, vcol, vfric;
    explicit Grid(const Params<R>& p)
        : nx(p.width + 1), ny(p.height + 1), nz(D == 3 ? p.depth + 1 : 1), nodes(nx * ny * nz),
          mass(nodes), mom(nodes * D), force(nodes * D), vcol(nodes * D), vfric(nodes * D) {}
    void reset() {  // src/gpu/shaders/2d/reset.glsl:13-23, src/cpu/Grid.cpp:186-190
        std::fill(mass.begin(), mass.end(), R(0));
        std::fill(mom.begin(), mom.end(), R(0));
        std::fill(force.begin(), force.end(), R(0));
        std::fill(vcol.begin(), vcol.end(), R(0));
        std::fill(vfric.begin(), vfric.end(), R(0));
    }
};

template <typename R> inline void add_to(R* dst, R val, bool atomic) {
#ifdef _OPENMP
    if (atomic) {
#pragma omp atomic
        *dst += val;
        return;
    }
#endif
    (void)atomic;
    *dst += val;
}

// Stencil of one particle: base node int(x) - 1 per axis (C truncation, as the
// reference's int()/static_cast<int>), 4 nodes per axis; out-of-grid nodes are
// skipped (src/gpu/shaders/2d/p2g.glsl:61-69).
template <int D> struct Stencil {
    int base[3];
};

template <int D, typename R> struct State {
    int64_t n;
    R *x, *v, *B, *Fe, *Fp;
    const R *mass, *vol;
};

// P2G. MLS: src/gpu/shaders/2d/p2g.glsl:29-92, 3d/p2g.glsl:31-96.
// CLASSIC: src/cpu/Grid.cpp:118-163 with Particle::PreComputeForces
// (src/cpu/Particles.cpp:21-62).
template <int D, typename R> void p2g(const Params<R>& p, State<D, R>& s, Grid<D, R>& g, int threads) {
    const bool atomic = threads > 1;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
#endif
    for (int64_t pi = 0; pi < s.n; ++pi) {
        const R* x = s.x + pi * D;
        const R* v = s.v + pi * D;
        const R* B = s.B + pi * D * D;
        const R* Fe = s.Fe + pi * D * D;
        const R* Fp = s.Fp + pi * D * D;
        const R mass = s.mass[pi], vol = s.vol[pi];
        R st[D * D];
        const bool mls = p.formulation != CLASSIC;
        const int S = stencil_nodes(p.formulation);
        const R dinv = stencil_dinv<R>(p.formulation);
        if (mls) {
            if (vol == R(0)) continue;  // p2g.glsl:42
            stress<D>(p, Fe, Fp, st);
        } else {
            // A_p = V sigma; a zero-volume particle keeps A_p = 0 (Particles.cpp:23)
            if (vol == R(0)) for (int i = 0; i < D * D; ++i) st[i] = R(0);
            else { stress<D>(p, Fe, Fp, st); for (int i = 0; i < D * D; ++i) st[i] *= vol; }
        }
        int base[3] = {0, 0, 0};
        for (int k = 0; k < D; ++k) base[k] = stencil_first(x[k], p.formulation);
        const int nzs = D == 3 ? S : 1;
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b)
                for (int c = 0; c < nzs; ++c) {
                    int idx[3] = {base[0] + a, base[1] + b, D == 3 ? base[2] + c : 0};
                    if (idx[0] < 0 || idx[0] > p.width || idx[1] < 0 || idx[1] > p.height) continue;
                    if (D == 3 && (idx[2] < 0 || idx[2] > p.depth)) continue;
                    int64_t cid = (int64_t(idx[2]) * g.ny + idx[1]) * g.nx + idx[0];
                    R dist[3], w = R(1), dw[3] = {1, 1, 1}, Nk[3], dNk[3];
                    for (int k = 0; k < D; ++k) {
                        dist[k] = x[k] - R(idx[k]);
                        Nk[k] = stencil_w(dist[k], p.formulation);
                        dNk[k] = bspline_dn(dist[k]);
                        w *= Nk[k];
                    }
                    const R m = w * mass;
                    if (mls) {
                        R wv[3];
                        // p2g.glsl:80-86 in glm's order: v + (3 B) (-dist) and
                        // (((V sigma) dist) 3) dt
                        for (int r = 0; r < D; ++r) {
                            R Bd = 0, Sd = 0;
                            for (int k = 0; k < D; ++k) {
                                Bd += (dinv * B[r * D + k]) * (-dist[k]);
                                Sd += (vol * st[r * D + k]) * dist[k];
                            }
                            R apic = v[r] + Bd;
                            R force = (Sd * dinv) * p.dt;
                            wv[r] = m * apic + w * force;
                        }
                        add_to(&g.mass[cid], m, atomic);
                        for (int r = 0; r < D; ++r) add_to(&g.mom[cid * D + r], wv[r], atomic);
                    } else {
                        for (int k = 0; k < D; ++k) {
                            dw[k] = dNk[k];
                            for (int l = 0; l < D; ++l) if (l != k) dw[k] *= Nk[l];
                        }
                        add_to(&g.mass[cid], m, atomic);
                        for (int r = 0; r < D; ++r) {
                            R Bd = 0, f = 0;
                            for (int k = 0; k < D; ++k) Bd += B[r * D + k] * (-dist[k]);
                            // glm: dWeight * A_p = A_p^T dWeight (row vector times matrix)
                            for (int k = 0; k < D; ++k) f += dw[k] * st[k * D + r];
                            add_to(&g.mom[cid * D + r], m * (v[r] + R(3) * Bd), atomic);
                            add_to(&g.force[cid * D + r], f, atomic);
                        }
                    }
                }
    }
}

// Grid update. MLS: src/gpu/shaders/2d/grid_update.glsl:82-108 (3D :88-117).
// CLASSIC: src/cpu/Grid.cpp:165-184.
template <int D, typename R> void grid_update(const Params<R>& p, Grid<D, R>& g, int threads) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
#endif
    for (int64_t id = 0; id < g.nodes; ++id) {
        const R m = g.mass[id];
        if (m < R(1e-6)) continue;
        R vel[3] = {0, 0, 0}, loc[3] = {0, 0, 0};
        const int gaxis = 1;  // gravity acts along y in 2D and 3D
        if (p.formulation != CLASSIC) {
            for (int k = 0; k < D; ++k) vel[k] = g.mom[id * D + k] / m;
            vel[gaxis] += p.gravity * p.dt;
        } else {
            for (int k = 0; k < D; ++k) {
                R vk = g.mom[id * D + k] / m;
                R fk = (k == gaxis ? p.gravity : R(0)) + (-g.force[id * D + k] / m);
                vel[k] = vk + fk * p.dt;
            }
        }
        int64_t ix = id % g.nx, iy = (id / g.nx) % g.ny, iz = id / (g.nx * g.ny);
        loc[0] = R(ix); loc[1] = R(iy); loc[2] = R(iz);
        R* vc = &g.vcol[id * D];
        R* vf = &g.vfric[id * D];
        if (p.boundary == BOUNDARY_STICKY) {
            const int m_ = int(p.margin);
            bool wall = ix < m_ || ix > p.width - m_ || iy < m_ || iy > p.height - m_ ||
                        (D == 3 && (iz < m_ || iz > p.depth - m_));
            for (int k = 0; k < D; ++k) { vc[k] = wall ? R(0) : vel[k]; vf[k] = vc[k]; }
        } else {
            collide<D>(p, loc, vel, vc, vf);
        }
    }
}

// G2P + plasticity. MLS: src/gpu/shaders/2d/g2p.glsl:21-93 (3D :22-104).
// CLASSIC: src/cpu/Particles.cpp:133-216 and UpdateDeformationGrad (:64-106).
template <int D, typename R> void g2p(const Params<R>& p, State<D, R>& s, const Grid<D, R>& g, int threads) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
#endif
    for (int64_t pi = 0; pi < s.n; ++pi) {
        R* x = s.x + pi * D;
        R* v = s.v + pi * D;
        R* B = s.B + pi * D * D;
        R* Fe = s.Fe + pi * D * D;
        R* Fp = s.Fp + pi * D * D;
        R old[3] = {0, 0, 0};
        for (int k = 0; k < D; ++k) old[k] = x[k];
        const int NS = stencil_nodes(p.formulation);
        int base[3] = {0, 0, 0};
        for (int k = 0; k < D; ++k) base[k] = stencil_first(old[k], p.formulation);
        R nv[3] = {0, 0, 0}, nx[3] = {0, 0, 0}, nB[9] = {0}, gv[9] = {0};
        const int nzs = D == 3 ? NS : 1;
        for (int a = 0; a < NS; ++a)
            for (int b = 0; b < NS; ++b)
                for (int c = 0; c < nzs; ++c) {
                    int idx[3] = {base[0] + a, base[1] + b, D == 3 ? base[2] + c : 0};
                    if (idx[0] < 0 || idx[0] > p.width || idx[1] < 0 || idx[1] > p.height) continue;
                    if (D == 3 && (idx[2] < 0 || idx[2] > p.depth)) continue;
                    int64_t cid = (int64_t(idx[2]) * g.ny + idx[1]) * g.nx + idx[0];
                    R dist[3], w = R(1), Nk[3], dNk[3];
                    for (int k = 0; k < D; ++k) {
                        dist[k] = old[k] - R(idx[k]);
                        Nk[k] = stencil_w(dist[k], p.formulation);
                        dNk[k] = bspline_dn(dist[k]);
                        w *= Nk[k];
                    }
                    const R* vf = &g.vfric[cid * D];
                    const R* vc = &g.vcol[cid * D];
                    for (int r = 0; r < D; ++r) {
                        nv[r] += vf[r] * w;
                        for (int k = 0; k < D; ++k) nB[r * D + k] += w * (vf[r] * (-dist[k]));
                        nx[r] += (p.dt * vc[r] + R(idx[r])) * w;
                    }
                    if (p.formulation == CLASSIC) {
                        R dw[3];
                        for (int k = 0; k < D; ++k) {
                            dw[k] = dNk[k];
                            for (int l = 0; l < D; ++l) if (l != k) dw[k] *= Nk[l];
                        }
                        for (int r = 0; r < D; ++r)
                            for (int k = 0; k < D; ++k) gv[r * D + k] += vc[r] * dw[k];
                    }
                }
        for (int k = 0; k < D; ++k) { v[k] = nv[k]; x[k] = nx[k]; }
        for (int i = 0; i < D * D; ++i) B[i] = nB[i];
        // F_E_hat = (I + dt L) F_E with L = 3 B (MLS, g2p.glsl:74-75), 4 B (QUAD)
        // or grad v (CLASSIC).
        R L[D * D], A[D * D], Fh[D * D];
        for (int i = 0; i < D * D; ++i) {
            L[i] = p.formulation != CLASSIC ? stencil_dinv<R>(p.formulation) * nB[i] : gv[i];
            A[i] = ((i % (D + 1) == 0) ? R(1) : R(0)) + p.dt * L[i];
        }
        matmul<D>(A, Fe, Fh);
        R U[D * D], S[D], V[D * D], Sh[D], Vt[D * D];
        svd<D>(Fh, U, S, V, p.formulation);
        const R t0 = R(1) - p.theta_c, t1 = R(1) + p.theta_s;
        for (int k = 0; k < D; ++k) {
            Sh[k] = S[k];
            S[k] = std::max(std::max(t0, std::min(S[k], t1)), R(1e-6));
        }
        transpose<D>(V, Vt);
        R US[D * D], VR[D * D], VRVt[D * D], nFp[D * D];
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) { US[r * D + c] = U[r * D + c] * S[c]; VR[r * D + c] = V[r * D + c] * (Sh[c] / S[c]); }
        matmul<D>(US, Vt, Fe);
        matmul<D>(VR, Vt, VRVt);
        matmul<D>(VRVt, Fp, nFp);
        for (int i = 0; i < D * D; ++i) Fp[i] = nFp[i];
    }
}

template <int D, typename R> void run(const Params<R>& p, State<D, R>& s, int nsteps, int threads) {
    Grid<D, R> g(p);
    for (int st = 0; st < nsteps; ++st) {
        g.reset();
        p2g<D>(p, s, g, threads);
        grid_update<D>(p, g, threads);
        g2p<D>(p, s, g, threads);
    }
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C ABI for tests (ctypes). Knobs mirror src/shared/Parameters.h.
extern "C" {

typedef struct {
    int32_t dim, width, height, depth, border_margin, formulation, boundary, reserved;
    double delta_time, gravity, friction, theta_c, theta_s, xi, nu, youngs;
} orc_params;
}

template <typename R> static orc::Params<R> to_params(const orc_params* q) {
    orc::Params<R> p;
    p.dim = q->dim; p.width = q->width; p.height = q->height; p.depth = q->depth;
    p.formulation = q->formulation; p.boundary = q->boundary;
    p.margin = R(q->border_margin); p.dt = R(q->delta_time); p.gravity = R(q->gravity);
    p.friction = R(q->friction); p.theta_c = R(q->theta_c); p.theta_s = R(q->theta_s); p.xi = R(q->xi);
    // Lame parameters, src/shared/Parameters.h:82-84
    double mu = q->youngs / (2.0 * (1.0 + q->nu));
    double la = (q->youngs * q->nu) / ((1.0 + q->nu) * (1.0 - 2.0 * q->nu));
    p.mu = R(mu); p.lambda = R(la);
    return p;
}

template <typename R>
static int step_impl(const orc_params* q, int64_t n, R* x, R* v, R* B, R* Fe, R* Fp, const R* mass,
                     const R* vol, int32_t nsteps, int32_t threads) {
    if (!q || n < 0 || nsteps < 0) return 1;
    if (q->dim != 2 && q->dim != 3) return 1;
    if (q->formulation < orc::MLS || q->formulation > orc::QUAD) return 1;
    if (q->dim == 3 && q->formulation == orc::CLASSIC) return 11;  // the reference CPU path is 2D only
    if (threads < 1) threads = 1;
    orc::Params<R> p = to_params<R>(q);
    if (q->dim == 2) {
        orc::State<2, R> s{n, x, v, B, Fe, Fp, mass, vol};
        orc::run<2, R>(p, s, nsteps, threads);
    } else {
        orc::State<3, R> s{n, x, v, B, Fe, Fp, mass, vol};
        orc::run<3, R>(p, s, nsteps, threads);
    }
    return 0;
}

extern "C" {

int orc_step_f64(const orc_params* q, int64_t n, double* x, double* v, double* B, double* Fe, double* Fp,
                 const double* mass, const double* vol, int32_t nsteps) {
    return step_impl<double>(q, n, x, v, B, Fe, Fp, mass, vol, nsteps, 1);
}

// FP64 on `threads` OpenMP threads (P2G adds with atomics, in no fixed order:
// the sums agree with the single-threaded run to FP64 rounding). For the
// workload-size parity runs.
int orc_step_f64_mt(const orc_params* q, int64_t n, double* x, double* v, double* B, double* Fe, double* Fp,
                    const double* mass, const double* vol, int32_t nsteps, int32_t threads) {
    return step_impl<double>(q, n, x, v, B, Fe, Fp, mass, vol, nsteps, threads);
}

int orc_step_f32(const orc_params* q, int64_t n, float* x, float* v, float* B, float* Fe, float* Fp,
                 const float* mass, const float* vol, int32_t nsteps, int32_t threads) {
    return step_impl<float>(q, n, x, v, B, Fe, Fp, mass, vol, nsteps, threads);
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Known-answer helpers.
void orc_bspline_f64(double x, double* n, double* dn) { *n = orc::bspline_n(x); *dn = orc::bspline_dn(x); }

void orc_svd_f64(int32_t dim, int32_t formulation, const double* M, double* U, double* S, double* V) {
    if (dim == 2) orc::svd<2>(M, U, S, V, formulation);
    else orc::svd<3>(M, U, S, V, formulation);
}

// FP32 instantiations of the same helpers (compared with the reference's
// shader functions compiled for the CPU, oracle/shader/shader_runner.cpp).
void orc_bspline_f32(float x, float* n, float* dn) { *n = orc::bspline_n(x); *dn = orc::bspline_dn(x); }

void orc_svd_f32(int32_t dim, int32_t formulation, const float* M, float* U, float* S, float* V) {
    if (dim == 2) orc::svd<2>(M, U, S, V, formulation);
    else orc::svd<3>(M, U, S, V, formulation);
}

void orc_collide_f32(const orc_params* q, const float* loc, const float* vel, float* vcol, float* vfric) {
    orc::Params<float> p = to_params<float>(q);
    if (q->dim == 2) orc::collide<2>(p, loc, vel, vcol, vfric);
    else orc::collide<3>(p, loc, vel, vcol, vfric);
}

void orc_stress_f64(const orc_params* q, const double* Fe, const double* Fp, double* out) {
    orc::Params<double> p = to_params<double>(q);
    if (q->dim == 2) orc::stress<2>(p, Fe, Fp, out);
    else orc::stress<3>(p, Fe, Fp, out);
}

void orc_collide_f64(const orc_params* q, const double* loc, const double* vel, double* vcol, double* vfric) {
    orc::Params<double> p = to_params<double>(q);
    if (q->dim == 2) orc::collide<2>(p, loc, vel, vcol, vfric);
    else orc::collide<3>(p, loc, vel, vcol, vfric);
}

// One P2G pass into caller-owned grid arrays (nodes, nodes*dim): for the
// conservation known-answer tests.
int orc_p2g_f64(const orc_params* q, int64_t n, const double* x, const double* v, const double* B,
                const double* Fe, const double* Fp, const double* mass, const double* vol, double* gmass,
                double* gmom) {
    orc::Params<double> p = to_params<double>(q);
    auto go = [&](auto dimtag) {
        constexpr int D = decltype(dimtag)::value;
        orc::Grid<D, double> g(p);
        orc::State<D, double> s{n, const_cast<double*>(x), const_cast<double*>(v), const_cast<double*>(B),
                                const_cast<double*>(Fe), const_cast<double*>(Fp), mass, vol};
        orc::p2g<D>(p, s, g, 1);
        std::memcpy(gmass, g.mass.data(), sizeof(double) * g.nodes);
        for (int64_t i = 0; i < g.nodes * D; ++i) gmom[i] = g.mom[i] - p.dt * g.force[i];
    };
    if (q->dim == 2) go(std::integral_constant<int, 2>());
    else go(std::integral_constant<int, 3>());
    return 0;
}

}  // extern "C"
