// Device math of the MLS-MPM step: cubic B-spline weights, the reference's
// SVD variants, polar rotation and the hardened stress. FP32 in the hot path;
// the same templates instantiate in FP64 for the near-degenerate SVD branch.
//
// Matrices are row-major dim x dim register arrays (M[r*D+c]).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mpm {

// Formulations: kMLS the reference GPU shaders (cubic stencil, D^-1 = 3);
// kClassic the reference CPU path (2D); kQuad the MLS step on the quadratic
// B-spline stencil (3 nodes per axis, D^-1 = 4), which the reference does not
// have.
enum : int { kMLS = 0, kClassic = 1, kQuad = 2 };
enum : int { kBoundaryFriction = 0, kBoundarySticky = 1 };

// Nodes per axis of a formulation's stencil, and the formulation whose SVD and
// stress a formulation uses (kQuad shares the shaders' math).
constexpr int stencil_of(int form) { return form == kQuad ? 3 : 4; }
constexpr int math_form(int form) { return form == kClassic ? kClassic : kMLS; }

// Cubic B-spline N(x) and dN/dx with support |x| < 2:
// src/gpu/shaders/2d/common.glsl:43-69 (src/cpu/Grid.h:86-116). pow(a, 3.0)
// is evaluated as a product.
// Cubic B-spline weight. The outer piece multiplies by the rounded 1/6
// instead of dividing (within 1 ulp of t^3 / 6; an IEEE division per weight
// would cost a subroutine call in every stencil).
template <typename R> __device__ __forceinline__ R bspline_n(R x) {
    R a = fabs(x);
    if (a < R(1)) return R(0.5) * a * a * a - a * a + R(2) / R(3);
    if (a < R(2)) { R t = R(2) - a; return t * t * t * (R(1) / R(6)); }
    return R(0);
}
// Quadratic B-spline N(x) with support |x| < 1.5 (the standard MLS-MPM
// kernel: 3/4 - x^2 inside |x| < 1/2, (3/2 - |x|)^2 / 2 outside).
template <typename R> __device__ __forceinline__ R quad_n(R x) {
    R a = fabs(x);
    if (a < R(0.5)) return R(0.75) - a * a;
    if (a < R(1.5)) { R t = R(1.5) - a; return R(0.5) * t * t; }
    return R(0);
}
template <typename R> __device__ __forceinline__ R bspline_dn(R x) {
    R a = fabs(x);
    if (a < R(1)) return R(1.5) * a * x - R(2) * x;
    if (a < R(2)) return R(-0.5) * a * x + R(2) * x - (R(2) * x) / a;
    return R(0);
}

template <int D, typename R> __device__ __forceinline__ R det(const R* A) {
    if (D == 2) return A[0] * A[3] - A[1] * A[2];
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
}

template <int D, typename R> __device__ __forceinline__ void matmul(const R* A, const R* B, R* C) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            R s = R(0);
#pragma unroll
            for (int k = 0; k < D; ++k) s += A[i * D + k] * B[k * D + j];
            C[i * D + j] = s;
        }
}

// 2x2 SVD by one analytic Jacobi rotation of M^T M (src/gpu/shaders/2d/
// common.glsl:2-37). A reflection is folded into the sign of S[1].
template <typename R> __device__ __forceinline__ void svd2_glsl(const R* M, R* U, R* S, R* V) {
    const R a = M[0] * M[0] + M[2] * M[2];
    const R b = M[0] * M[1] + M[2] * M[3];
    const R d = M[1] * M[1] + M[3] * M[3];
    const R theta = (fabs(b) < R(1e-10) && fabs(a - d) < R(1e-10)) ? R(0) : R(0.5) * atan2(R(2) * b, a - d);
    R st, ct;
    st = sin(theta);
    ct = cos(theta);
    V[0] = ct; V[1] = -st; V[2] = st; V[3] = ct;
    // diag(V^T (M^T M) V)
    const R d0 = ct * (a * ct + b * st) + st * (b * ct + d * st);
    const R d1 = -st * (-a * st + b * ct) + ct * (-b * st + d * ct);
    S[0] = sqrt(fmax(d0, R(1e-12)));
    S[1] = sqrt(fmax(d1, R(1e-12)));
    const R i0 = R(1) / S[0], i1 = R(1) / S[1];
    U[0] = (M[0] * V[0] + M[1] * V[2]) * i0;
    U[1] = (M[0] * V[1] + M[1] * V[3]) * i1;
    U[2] = (M[2] * V[0] + M[3] * V[2]) * i0;
    U[3] = (M[2] * V[1] + M[3] * V[3]) * i1;
    if (U[0] * U[3] - U[1] * U[2] < R(0)) { U[1] = -U[1]; U[3] = -U[3]; S[1] = -S[1]; }
}

// 2x2 SVD with the conventions of Eigen 3.4 JacobiSVD (singular values >= 0,
// descending), the decomposition the reference CPU path uses
// (src/cpu/Particles.cpp:31-32,73-78). Two-sided Jacobi as published in
// Eigen/src/SVD/JacobiSVD.h:666-780 and Eigen/src/misc/RealSvd2x2.h:18-49.
template <typename R> __device__ __forceinline__ void svd2_eigen(const R* A, R* U, R* S, R* V) {
    const R eps = sizeof(R) == 4 ? R(1.1920928955078125e-07) : R(2.220446049250313e-16);
    const R tiny = sizeof(R) == 4 ? R(1.1754943508222875e-38) : R(2.2250738585072014e-308);
    R scale = fmax(fmax(fabs(A[0]), fabs(A[1])), fmax(fabs(A[2]), fabs(A[3])));
    U[0] = R(1); U[1] = R(0); U[2] = R(0); U[3] = R(1);
    V[0] = R(1); V[1] = R(0); V[2] = R(0); V[3] = R(1);
    if (!isfinite(scale)) { S[0] = S[1] = scale - scale; return; }
    if (scale == R(0)) scale = R(1);
    R w[4] = {A[0] / scale, A[1] / scale, A[2] / scale, A[3] / scale};
    R maxd = fmax(fabs(w[0]), fabs(w[3]));
    for (int it = 0; it < 8; ++it) {
        const R thr = fmax(tiny, R(2) * eps * maxd);
        if (!(fabs(w[2]) > thr || fabs(w[1]) > thr)) break;
        // (p, q) = (1, 0): sub-block m = [[w11, w10], [w01, w00]]
        R m0 = w[3], m1 = w[2], m2 = w[1], m3 = w[0];
        const R t = m0 + m3, dd = m2 - m1;
        R c1 = R(1), s1 = R(0);
        if (!(fabs(dd) < tiny)) { const R u = t / dd, tmp = sqrt(R(1) + u * u); c1 = u / tmp; s1 = R(1) / tmp; }
        {   // rows 0,1 of m by rot1
            R x0 = m0, x1 = m1, y0 = m2, y1 = m3;
            m0 = c1 * x0 + s1 * y0; m1 = c1 * x1 + s1 * y1;
            m2 = -s1 * x0 + c1 * y0; m3 = -s1 * x1 + c1 * y1;
        }
        R cr = R(1), sr = R(0);
        const R deno = R(2) * fabs(m1);
        if (!(deno < tiny)) {
            const R tau = (m0 - m3) / deno, ww = sqrt(tau * tau + R(1));
            const R tt = tau > R(0) ? R(1) / (tau + ww) : R(1) / (tau - ww);
            const R sg = tt > R(0) ? R(1) : R(-1), n = R(1) / sqrt(tt * tt + R(1));
            cr = n;
            sr = -sg * (m1 / fabs(m1)) * fabs(tt) * n;
        }
        // j_left = rot1 * j_right^T
        const R cl = c1 * cr - s1 * (-sr), sl = c1 * (-sr) + s1 * cr;
        {   // w rows (1, 0) by j_left: x = row1, y = row0
            R x0 = w[2], x1 = w[3], y0 = w[0], y1 = w[1];
            w[2] = cl * x0 + sl * y0; w[3] = cl * x1 + sl * y1;
            w[0] = -sl * x0 + cl * y0; w[1] = -sl * x1 + cl * y1;
        }
        {   // U columns (1, 0) by j_left (applyOnTheRight with j_left^T)
            R x0 = U[1], x1 = U[3], y0 = U[0], y1 = U[2];
            U[1] = cl * x0 + sl * y0; U[3] = cl * x1 + sl * y1;
            U[0] = -sl * x0 + cl * y0; U[2] = -sl * x1 + cl * y1;
        }
        {   // w and V columns (1, 0) by j_right^T
            R x0 = w[1], x1 = w[3], y0 = w[0], y1 = w[2];
            w[1] = cr * x0 - sr * y0; w[3] = cr * x1 - sr * y1;
            w[0] = sr * x0 + cr * y0; w[2] = sr * x1 + cr * y1;
            x0 = V[1]; x1 = V[3]; y0 = V[0]; y1 = V[2];
            V[1] = cr * x0 - sr * y0; V[3] = cr * x1 - sr * y1;
            V[0] = sr * x0 + cr * y0; V[2] = sr * x1 + cr * y1;
        }
        maxd = fmax(maxd, fmax(fabs(w[3]), fabs(w[0])));
    }
    S[0] = fabs(w[0]);
    S[1] = fabs(w[3]);
    if (w[0] < R(0)) { U[0] = -U[0]; U[2] = -U[2]; }
    if (w[3] < R(0)) { U[1] = -U[1]; U[3] = -U[3]; }
    S[0] *= scale;
    S[1] *= scale;
    if (S[1] > S[0]) {
        R t = S[0]; S[0] = S[1]; S[1] = t;
        t = U[0]; U[0] = U[1]; U[1] = t; t = U[2]; U[2] = U[3]; U[3] = t;
        t = V[0]; V[0] = V[1]; V[1] = t; t = V[2]; V[2] = V[3]; V[3] = t;
    }
}

// 3x3 SVD of src/gpu/shaders/3d/common.glsl:8-105: cyclic Jacobi on
// S = M^T M over the pairs (0,1), (0,2), (1,2); U = M V Sigma^-1, reflection
// folded into Sigma[2]. The reference runs 6 fixed sweeps; here the iteration
// stops after the first sweep that leaves the off-diagonal of S below 2 eps of
// its diagonal (further rotations then only move rounding noise around), with
// 6 sweeps as the bound.
template <typename R> __device__ __forceinline__ void schur2(R app, R apq, R aqq, R& c, R& s) {
    if (fabs(apq) < R(1e-10)) { c = R(1); s = R(0); return; }
    const R tau = (aqq - app) / (R(2) * apq);
    const R stt = sqrt(R(1) + tau * tau);
    R tn = R(1) / (fabs(tau) + stt);
    if (tau < R(0)) tn = -tn;
    c = R(1) / sqrt(R(1) + tn * tn);
    s = tn * c;
}

template <int P, int Q, typename R> __device__ __forceinline__ void jacobi_step(R* S, R* V) {
    constexpr int O = 3 - P - Q;  // the third index
    R c, s;
    schur2(S[P * 3 + P], S[P * 3 + Q], S[Q * 3 + Q], c, s);
    const R Spp = S[P * 3 + P], Sqq = S[Q * 3 + Q], Spq = S[P * 3 + Q];
    S[P * 3 + P] = c * c * Spp - R(2) * s * c * Spq + s * s * Sqq;
    S[Q * 3 + Q] = s * s * Spp + R(2) * s * c * Spq + c * c * Sqq;
    S[P * 3 + Q] = R(0);
    S[Q * 3 + P] = R(0);
    const R Sop = S[O * 3 + P], Soq = S[O * 3 + Q];
    S[O * 3 + P] = c * Sop - s * Soq;
    S[P * 3 + O] = S[O * 3 + P];
    S[O * 3 + Q] = s * Sop + c * Soq;
    S[Q * 3 + O] = S[O * 3 + Q];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const R vp = V[r * 3 + P], vq = V[r * 3 + Q];
        V[r * 3 + P] = c * vp - s * vq;
        V[r * 3 + Q] = s * vp + c * vq;
    }
}

template <typename R> __device__ __forceinline__ void svd3_glsl(const R* M, R* U, R* Sig, R* V) {
    R S[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S[i * 3 + j] = M[0 * 3 + i] * M[0 * 3 + j] + M[1 * 3 + i] * M[1 * 3 + j] + M[2 * 3 + i] * M[2 * 3 + j];
#pragma unroll
    for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? R(1) : R(0);
    const R tol = sizeof(R) == 4 ? R(2.4e-7) : R(4.5e-16);  // 2 eps
    for (int sweep = 0; sweep < 6; ++sweep) {
        jacobi_step<0, 1>(S, V);
        jacobi_step<0, 2>(S, V);
        jacobi_step<1, 2>(S, V);
        const R off = S[1] * S[1] + S[2] * S[2] + S[5] * S[5];
        const R dia = S[0] * S[0] + S[4] * S[4] + S[8] * S[8];
        if (off <= tol * tol * dia) break;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) Sig[i] = sqrt(fmax(S[i * 4], R(1e-12)));
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            U[r * 3 + c] = (M[r * 3 + 0] * V[0 * 3 + c] + M[r * 3 + 1] * V[1 * 3 + c] + M[r * 3 + 2] * V[2 * 3 + c]) * (R(1) / Sig[c]);
    if (det<3>(U) < R(0)) { U[2] = -U[2]; U[5] = -U[5]; U[8] = -U[8]; Sig[2] = -Sig[2]; }
}

template <int D, int FORM, typename R> __device__ __forceinline__ void svd(const R* M, R* U, R* S, R* V) {
    if constexpr (D == 2) {
        if constexpr (FORM == kClassic) svd2_eigen(M, U, S, V);
        else svd2_glsl(M, U, S, V);
    } else {
        svd3_glsl(M, U, S, V);
    }
}

// Polar rotation R = U V^T of F_E and the hardened stress
// sigma = 2 mu (F_E - R) F_E^T + lambda (J_e - 1) J_e I,
// mu = MU exp(XI (1 - J_p)), lambda = LAMBDA exp(XI (1 - J_p))
// (src/gpu/shaders/2d/p2g.glsl:44-59, 3d/p2g.glsl:46-61, src/cpu/Particles.cpp:21-48).
template <int D, int FORM> __device__ __forceinline__ void hardened_stress(const float* Fe, float Jp, float mu0,
                                                                          float la0, float xi, float* sig) {
    float U[D * D], S[D], V[D * D];
    svd<D, FORM>(Fe, U, S, V);
    float Rm[D * D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) s += U[i * D + k] * V[j * D + k];
            Rm[i * D + j] = s;
        }
    const float Je = det<D>(Fe);
    const float h = expf(xi * (1.f - Jp));
    const float mu = mu0 * h, la = la0 * h;
    const float diag = la * (Je - 1.f) * Je;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) s += (Fe[i * D + k] - Rm[i * D + k]) * Fe[j * D + k];
            sig[i * D + j] = 2.f * mu * s + (i == j ? diag : 0.f);
        }
}

// Polar rotation R of F (F = R S, S symmetric positive definite) for det F > 0.
// 2D: closed form, R is the rotation by atan2(F10 - F01, F00 + F11)
//     (tr(R^T F) = tr S > 0 keeps that vector away from zero).
// 3D: Newton's iteration R <- (R + R^-T) / 2 from R = F, which converges
//     quadratically to the polar factor; stops once an update is below 1e-6.
// Returns false (R untouched) for det F <= 0 or no convergence in 12
// iterations; the caller then takes U V^T from the reference's SVD.
template <int D> __device__ __forceinline__ bool polar_rotation(const float* F, float* R) {
    if constexpr (D == 2) {
        if (!(F[0] * F[3] - F[1] * F[2] > 0.f)) return false;
        const float c = F[0] + F[3], s = F[2] - F[1];
        const float inv = rsqrtf(c * c + s * s);
        R[0] = c * inv; R[1] = -s * inv; R[2] = s * inv; R[3] = c * inv;
        return true;
    } else {
        if (!(det<3>(F) > 0.f)) return false;
        float X[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) X[i] = F[i];
        for (int it = 0; it < 12; ++it) {
            // cofactor matrix: X^-T = cof(X) / det(X)
            float cf[9];
            cf[0] = X[4] * X[8] - X[5] * X[7];
            cf[1] = X[5] * X[6] - X[3] * X[8];
            cf[2] = X[3] * X[7] - X[4] * X[6];
            cf[3] = X[2] * X[7] - X[1] * X[8];
            cf[4] = X[0] * X[8] - X[2] * X[6];
            cf[5] = X[1] * X[6] - X[0] * X[7];
            cf[6] = X[1] * X[5] - X[2] * X[4];
            cf[7] = X[2] * X[3] - X[0] * X[5];
            cf[8] = X[0] * X[4] - X[1] * X[3];
            const float dt = X[0] * cf[0] + X[1] * cf[1] + X[2] * cf[2];
            if (!(dt > 0.f)) return false;
            const float hid = 0.5f / dt;
            float diff = 0.f;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const float nx = 0.5f * X[i] + hid * cf[i];
                const float e = nx - X[i];
                diff += e * e;
                X[i] = nx;
            }
            if (diff < 1e-12f) {
#pragma unroll
                for (int i = 0; i < 9; ++i) R[i] = X[i];
                return true;
            }
        }
        return false;
    }
}

// Stress of the hardened Kirchhoff form above with the polar rotation taken
// from polar_rotation (the same R = U V^T as the reference's SVD, computed
// without the SVD); falls back to hardened_stress when it declines.
template <int D, int FORM> __device__ __forceinline__ void hardened_stress_polar(const float* Fe, float Jp, float mu0,
                                                                                float la0, float xi, float* sig) {
    float Rm[D * D];
    if (FORM != kMLS || !polar_rotation<D>(Fe, Rm)) {
        hardened_stress<D, FORM>(Fe, Jp, mu0, la0, xi, sig);
        return;
    }
    const float Je = det<D>(Fe);
    const float h = expf(xi * (1.f - Jp));
    const float mu = mu0 * h, la = la0 * h;
    const float diag = la * (Je - 1.f) * Je;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) s += (Fe[i * D + k] - Rm[i * D + k]) * Fe[j * D + k];
            sig[i * D + j] = 2.f * mu * s + (i == j ? diag : 0.f);
        }
}

// Hardened stress through the left stretch (3D): for det F > 0, F = V R with
// V = sqrt(F F^T), so (F - R) F^T = F F^T - V. With E = F F^T - I,
//   F F^T - sqrt(F F^T) = E/2 + E^2/8 - E^3/16 + 5E^4/128 - 7E^5/256 + ...
// (the binomial series of sqrt(1 + x) subtracted from 1 + x), evaluated on the
// symmetric E without forming R and without the cancellation of F F^T - V.
// Applies when ||E||_F <= 0.1 (8 terms: truncation below 1e-10 ||E||; every F
// inside the default elastic band qualifies). 2D: the closed-form polar
// rotation. Returns false (nothing written) when it does not apply.
template <int D>
__device__ __forceinline__ bool hardened_stress_series(const float* Fe, float Jp, float mu0, float la0, float xi,
                                                       float* sig) {
    if constexpr (D == 3) {
        const float J = det<3>(Fe);
        // symmetric E = F F^T - I : (00, 11, 22, 01, 02, 12)
        float e[6];
        e[0] = Fe[0] * Fe[0] + Fe[1] * Fe[1] + Fe[2] * Fe[2] - 1.f;
        e[1] = Fe[3] * Fe[3] + Fe[4] * Fe[4] + Fe[5] * Fe[5] - 1.f;
        e[2] = Fe[6] * Fe[6] + Fe[7] * Fe[7] + Fe[8] * Fe[8] - 1.f;
        e[3] = Fe[0] * Fe[3] + Fe[1] * Fe[4] + Fe[2] * Fe[5];
        e[4] = Fe[0] * Fe[6] + Fe[1] * Fe[7] + Fe[2] * Fe[8];
        e[5] = Fe[3] * Fe[6] + Fe[4] * Fe[7] + Fe[5] * Fe[8];
        const float n2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2] + 2.f * (e[3] * e[3] + e[4] * e[4] + e[5] * e[5]);
        if (!(J > 0.f && n2 <= 0.01f)) return false;
        // coefficients of E^k in 1 + x - sqrt(1 + x), k = 1..8
        const float d[8] = {0.5f, 0.125f, -0.0625f, 0.0390625f, -0.02734375f, 0.0205078125f, -0.01611328125f,
                            0.013092041015625f};
        float t[6], p[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) { p[q] = e[q]; t[q] = d[0] * e[q]; }
        // Five terms when |E| <= 0.05 (the rest is below 3.4e-10, under the
        // FP32 rounding of t), eight otherwise (|E| <= 0.1: below 1.4e-10).
        const int terms = n2 <= 0.0025f ? 5 : 8;
#pragma unroll
        for (int k = 1; k < 8; ++k) {
            if (k >= terms) break;
            // p <- p E (powers of one symmetric matrix commute: symmetric)
            float r[6];
            r[0] = p[0] * e[0] + p[3] * e[3] + p[4] * e[4];
            r[1] = p[3] * e[3] + p[1] * e[1] + p[5] * e[5];
            r[2] = p[4] * e[4] + p[5] * e[5] + p[2] * e[2];
            r[3] = p[0] * e[3] + p[3] * e[1] + p[4] * e[5];
            r[4] = p[0] * e[4] + p[3] * e[5] + p[4] * e[2];
            r[5] = p[3] * e[4] + p[1] * e[5] + p[5] * e[2];
#pragma unroll
            for (int q = 0; q < 6; ++q) { p[q] = r[q]; t[q] += d[k] * r[q]; }
        }
        const float h = expf(xi * (1.f - Jp));
        const float mu2 = 2.f * mu0 * h, diag = la0 * h * (J - 1.f) * J;
        sig[0] = mu2 * t[0] + diag; sig[4] = mu2 * t[1] + diag; sig[8] = mu2 * t[2] + diag;
        sig[1] = sig[3] = mu2 * t[3];
        sig[2] = sig[6] = mu2 * t[4];
        sig[5] = sig[7] = mu2 * t[5];
        return true;
    } else {
        float Rm[4];
        if (!polar_rotation<2>(Fe, Rm)) return false;
        const float Je = det<2>(Fe);
        const float h = expf(xi * (1.f - Jp));
        const float mu = mu0 * h, la = la0 * h;
        const float diag = la * (Je - 1.f) * Je;
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const float s = (Fe[i * 2] - Rm[i * 2]) * Fe[j * 2] + (Fe[i * 2 + 1] - Rm[i * 2 + 1]) * Fe[j * 2 + 1];
                sig[i * 2 + j] = 2.f * mu * s + (i == j ? diag : 0.f);
            }
        return true;
    }
}

// The stress of the MLS path: the series / closed form above when it applies,
// else the polar rotation (Newton, then the reference's SVD).
template <int D, int FORM> __device__ __forceinline__ void hardened_stress_fast(const float* Fe, float Jp, float mu0,
                                                                               float la0, float xi, float* sig) {
    if (FORM == kMLS && hardened_stress_series<D>(Fe, Jp, mu0, la0, xi, sig)) return;
    hardened_stress_polar<D, FORM>(Fe, Jp, mu0, la0, xi, sig);
}

// True when every singular value of F lies in [t0, t1] and det F > 0, proven
// with margin: then the return map clamps nothing and is the identity
// (F_E' = F, J_p' = J_p), so the SVD can be skipped. First Gershgorin discs of
// S = F^T F in FP32 (margin 4e-6 > the FP32 rounding of S); if they do not
// decide, Sylvester's criterion in FP64 for (t1^2 - 1e-5) I - S and
// S - (t0^2 + 1e-5) I (positive leading minors); 1e-5 exceeds the FP64
// rounding of the minors even for a triple eigenvalue at the margin.
template <int D> __device__ __forceinline__ bool band_gershgorin(const float* F, float t0, float t1) {
    float S[D * D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) s += F[k * D + i] * F[k * D + j];
            S[i * D + j] = s;
        }
    const float lo = t0 * t0 + 4e-6f, hi = t1 * t1 - 4e-6f;
    bool gersh = true;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        float r = 0.f;
#pragma unroll
        for (int j = 0; j < D; ++j)
            if (j != i) r += fabsf(S[i * D + j]);
        gersh = gersh && (S[i * D + i] - r >= lo) && (S[i * D + i] + r <= hi);
    }
    return gersh;
}

template <int D> __device__ __forceinline__ bool in_elastic_band(const float* F, float t0, float t1) {
    if (!(det<D>(F) > 0.f)) return false;
    if (band_gershgorin<D>(F, t0, t1)) return true;
    double Sd[D * D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) s += double(F[k * D + i]) * double(F[k * D + j]);
            Sd[i * D + j] = s;
        }
    const double up = double(t1) * double(t1) - 1e-5, dn = double(t0) * double(t0) + 1e-5;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        double M[D * D];
#pragma unroll
        for (int i = 0; i < D * D; ++i) M[i] = side == 0 ? -Sd[i] : Sd[i];
#pragma unroll
        for (int i = 0; i < D; ++i) M[i * D + i] += side == 0 ? up : -dn;
        if (!(M[0] > 0.0)) return false;
        if constexpr (D == 2) {
            if (!(M[0] * M[3] - M[1] * M[2] > 0.0)) return false;
        } else {
            if (!(M[0] * M[4] - M[1] * M[3] > 0.0)) return false;
            if (!(det<3>(M) > 0.0)) return false;
        }
    }
    return true;
}

}  // namespace mpm
