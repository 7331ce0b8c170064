// Learned plasticity surrogate: a 10 -> 64 -> 64 -> 64 -> 10 MLP with GELU,
// BF16 weights and activations, FP32 accumulation on the tensor cores
// (mma.sync m16n8k16 bf16), FP32 master weights trained with AdamW.
//
// It maps the trial elastic gradient and the plastic volume ratio of a particle
// whose trial F lies outside the elastic band (inputs: F_hat - I, log J_p) to
// the return map's correction (outputs: F_E' - F_hat, log J_p' - log J_p), both
// normalised per feature. Training pairs come from the exact return map of the
// plain solver (k_g2p_plastic with the pair log enabled).
#pragma once

#include <cuda_bf16.h>

#include "mpm_kernels.cuh"

namespace mpm {

constexpr int kMlpIn = 10, kMlpHid = 64, kMlpOut = 10, kMlpInPad = 16, kMlpOutPad = 16;
// Parameter block (row-major W[out][in]): W1[64][16] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] W4[16][64] b4[16]; padded rows/columns are kept at zero.
struct MlpOff {
    static constexpr int W1 = 0, b1 = W1 + kMlpHid * kMlpInPad, W2 = b1 + kMlpHid, b2 = W2 + kMlpHid * kMlpHid,
                         W3 = b2 + kMlpHid, b3 = W3 + kMlpHid * kMlpHid, W4 = b3 + kMlpHid,
                         b4 = W4 + kMlpOutPad * kMlpHid, total = b4 + kMlpOutPad;
};

struct MlpNorm {
    float in_mean[kMlpIn], in_std[kMlpIn], out_mean[kMlpOut], out_std[kMlpOut];
};

// ---------------------------------------------------------------------------
// Tensor-core fragments. Operands live in shared memory as bf16 with arbitrary
// strides: A(m, k) at A[m * sam + k * sak], B(k, n) at B[k * sbk + n * sbn].
// m16n8k16 layouts (PTX ISA): with g = lane / 4, t = lane % 4,
//   A regs: (g, 2t..2t+1), (g+8, 2t..), (g, 2t+8..), (g+8, 2t+8..)
//   B regs: (k = 2t..2t+1, n = g), (k = 2t+8.., n = g)
//   C/D   : (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1)
__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// acc[16 x 8] (C layout) += A[m0.., k0..k0+16) * B[k0.., n0..n0+8)
__device__ __forceinline__ void mma_tile(float* acc, const __nv_bfloat16* A, int sam, int sak, const __nv_bfloat16* B,
                                         int sbk, int sbn, int m0, int k0, int n0) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a[4], b[2];
    const int kk = k0 + 2 * t;
    auto ldA = [&](int m, int k) { return pack_bf16(A[m * sam + k * sak], A[m * sam + (k + 1) * sak]); };
    auto ldB = [&](int k, int n) { return pack_bf16(B[k * sbk + n * sbn], B[(k + 1) * sbk + n * sbn]); };
    a[0] = ldA(m0 + g, kk);
    a[1] = ldA(m0 + g + 8, kk);
    a[2] = ldA(m0 + g, kk + 8);
    a[3] = ldA(m0 + g + 8, kk + 8);
    b[0] = ldB(kk, n0 + g);
    b[1] = ldB(kk + 8, n0 + g);
    mma_bf16(acc, a, b);
}

// GELU in its tanh form (Hendrycks & Gimpel 2016):
//   gelu(x) = x/2 (1 + tanh(c (x + 0.044715 x^3))),  c = sqrt(2/pi),
// with the hardware tanh (PTX tanh.approx.f32, relative error ~2^-11, below the
// bf16 rounding of the stored activations). Training and inference share it.
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kGeluC = 0.7978845608028654f, kGeluA = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
    const float th = tanh_hw(kGeluC * x * fmaf(kGeluA, x * x, 1.f));
    return 0.5f * x * (1.f + th);
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float x2 = x * x;
    const float th = tanh_hw(kGeluC * x * fmaf(kGeluA, x2, 1.f));
    return 0.5f * (1.f + th) + 0.5f * x * (1.f - th * th) * kGeluC * fmaf(3.f * kGeluA, x2, 1.f);
}

// Raw pair -> normalised network input (row of kMlpInPad bf16) and target.
// Pair layout (20 floats): F_hat[9] J_p[1] F_E'[9] J_p'[1].
__device__ __forceinline__ void mlp_features(const float* Fh, float Jp, const MlpNorm& N, float* in) {
#pragma unroll
    for (int k = 0; k < 9; ++k) in[k] = ((Fh[k] - (k % 4 == 0 ? 1.f : 0.f)) - N.in_mean[k]) * (1.f / N.in_std[k]);
    in[9] = (logf(Jp) - N.in_mean[9]) * (1.f / N.in_std[9]);
}
__device__ __forceinline__ void mlp_targets(const float* pair, const MlpNorm& N, float* tg) {
#pragma unroll
    for (int k = 0; k < 9; ++k) tg[k] = ((pair[10 + k] - pair[k]) - N.out_mean[k]) / N.out_std[k];
    tg[9] = ((logf(pair[19]) - logf(pair[9])) - N.out_mean[9]) / N.out_std[9];
}

// ---------------------------------------------------------------------------
// Forward pass of one 16-row tile per warp on shared-memory activations.
// X: [rows][ldx] bf16; layer output Y (pre-activation, fp32 [rows][ldy]) and
// H = GELU(Y) as bf16 [rows][ldh] when `act`.
__device__ __forceinline__ void mlp_layer_fwd(const __nv_bfloat16* X, int ldx, int K, const __nv_bfloat16* W,
                                              const float* bias, int N, int m0, float* Y, int ldy, __nv_bfloat16* H,
                                              int ldh, bool act) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int n0 = 0; n0 < N; n0 += 8) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k0 = 0; k0 < K; k0 += 16) mma_tile(acc, X, ldx, 1, W, 1, K, m0, k0, n0);
        const int r0 = m0 + g, c0 = n0 + 2 * t;
        const float v[4] = {acc[0] + bias[c0], acc[1] + bias[c0 + 1], acc[2] + bias[c0], acc[3] + bias[c0 + 1]};
        const int rr[4] = {r0, r0, r0 + 8, r0 + 8}, cc[4] = {c0, c0 + 1, c0, c0 + 1};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (Y) Y[rr[q] * ldy + cc[q]] = v[q];
            if (H) H[rr[q] * ldh + cc[q]] = __float2bfloat16_rn(act ? gelu(v[q]) : v[q]);
        }
    }
}

// ---------------------------------------------------------------------------
// Training step on one CTA of kMlpTrainRows samples (4 warps x 16 rows):
// forward, MSE loss, backward; weight gradients accumulated (fp32 atomics)
// into `grad`, loss sum into `loss`. Samples: `idx` (explicit, may be null) or
// a hash of (seed, global row) modulo n_pairs.
constexpr int kMlpTrainRows = 64;

struct MlpTrainSmem {
    __nv_bfloat16 w[MlpOff::total];
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpHid], b4[kMlpOutPad];
    __nv_bfloat16 x0[kMlpTrainRows * kMlpInPad];
    __nv_bfloat16 h[3][kMlpTrainRows * kMlpHid];
    float y[3][kMlpTrainRows * kMlpHid];
    float out[kMlpTrainRows * kMlpOutPad];
    float tgt[kMlpTrainRows * kMlpOutPad];
    __nv_bfloat16 dy[kMlpTrainRows * kMlpHid];   // gradient wrt the current layer's pre-activation
    __nv_bfloat16 dy4[kMlpTrainRows * kMlpOutPad];
    float dh[kMlpTrainRows * kMlpHid];            // gradient wrt the previous layer's output
};

__device__ __forceinline__ unsigned hash_u32(unsigned x) {
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(128) k_mlp_train(const float* __restrict__ pairs, long long n_pairs,
                                                   const int* __restrict__ idx, int n_rows, unsigned seed,
                                                   const __nv_bfloat16* __restrict__ wbf, const float* __restrict__ wf32,
                                                   MlpNorm N, float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpTrainSmem& S = *reinterpret_cast<MlpTrainSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    for (int i = tid; i < MlpOff::total; i += blockDim.x) S.w[i] = wbf[i];
    for (int i = tid; i < kMlpHid; i += blockDim.x) {
        S.b1[i] = wf32[MlpOff::b1 + i];
        S.b2[i] = wf32[MlpOff::b2 + i];
        S.b3[i] = wf32[MlpOff::b3 + i];
    }
    for (int i = tid; i < kMlpOutPad; i += blockDim.x) S.b4[i] = wf32[MlpOff::b4 + i];
    // rows of this CTA
    const int row0 = blockIdx.x * kMlpTrainRows;
    for (int r = tid; r < kMlpTrainRows; r += blockDim.x) {
        const int gr = row0 + r;
        float in[kMlpIn], tg[kMlpOut];
        const bool valid = gr < n_rows;
        if (valid) {
            const long long p = idx ? (long long)idx[gr]
                                    : (long long)((((unsigned long long)hash_u32(seed ^ hash_u32((unsigned)gr)) << 20) ^
                                                   hash_u32((unsigned)gr * 2654435761u + seed)) % (unsigned long long)n_pairs);
            const float* pr = pairs + p * 20;
            mlp_features(pr, pr[9], N, in);
            mlp_targets(pr, N, tg);
        }
        for (int k = 0; k < kMlpInPad; ++k) S.x0[r * kMlpInPad + k] = __float2bfloat16_rn(valid && k < kMlpIn ? in[k] : 0.f);
        for (int k = 0; k < kMlpOutPad; ++k) S.tgt[r * kMlpOutPad + k] = valid && k < kMlpOut ? tg[k] : 0.f;
    }
    __syncthreads();
    const int m0 = warp * 16;
    const __nv_bfloat16* W1 = S.w + MlpOff::W1;
    const __nv_bfloat16* W2 = S.w + MlpOff::W2;
    const __nv_bfloat16* W3 = S.w + MlpOff::W3;
    const __nv_bfloat16* W4 = S.w + MlpOff::W4;
    mlp_layer_fwd(S.x0, kMlpInPad, kMlpInPad, W1, S.b1, kMlpHid, m0, S.y[0], kMlpHid, S.h[0], kMlpHid, true);
    __syncwarp();
    mlp_layer_fwd(S.h[0], kMlpHid, kMlpHid, W2, S.b2, kMlpHid, m0, S.y[1], kMlpHid, S.h[1], kMlpHid, true);
    __syncwarp();
    mlp_layer_fwd(S.h[1], kMlpHid, kMlpHid, W3, S.b3, kMlpHid, m0, S.y[2], kMlpHid, S.h[2], kMlpHid, true);
    __syncwarp();
    mlp_layer_fwd(S.h[2], kMlpHid, kMlpHid, W4, S.b4, kMlpOutPad, m0, S.out, kMlpOutPad, nullptr, 0, false);
    __syncthreads();
    // loss and dL/dY4 (mean over all rows of the launch)
    float lsum = 0.f;
    for (int e = tid; e < kMlpTrainRows * kMlpOutPad; e += blockDim.x) {
        const int r = e / kMlpOutPad, c = e % kMlpOutPad;
        const bool valid = row0 + r < n_rows && c < kMlpOut;
        const float diff = valid ? S.out[e] - S.tgt[e] : 0.f;
        lsum += diff * diff;
        S.dy4[e] = __float2bfloat16_rn(2.f * diff / float(n_rows));
        S.out[e] = 2.f * diff / float(n_rows);  // fp32 copy for the bias gradient
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0) atomicAdd(loss, lsum);
    __syncthreads();

    // backward through the 4 layers: at layer l with input X (bf16 [rows][K])
    // and dY (bf16 [rows][N]): dW = dY^T X (tensor cores, k = rows), db = sum dY,
    // dX = dY W (tensor cores), then dY_{l-1} = dX * GELU'(Y_{l-1}).
    struct L { const __nv_bfloat16* X; int K; const __nv_bfloat16* W; int N; int woff, boff; };
    const L layers[4] = {{S.x0, kMlpInPad, W1, kMlpHid, MlpOff::W1, MlpOff::b1},
                         {S.h[0], kMlpHid, W2, kMlpHid, MlpOff::W2, MlpOff::b2},
                         {S.h[1], kMlpHid, W3, kMlpHid, MlpOff::W3, MlpOff::b3},
                         {S.h[2], kMlpHid, W4, kMlpOutPad, MlpOff::W4, MlpOff::b4}};
    for (int l = 3; l >= 0; --l) {
        const L& Ly = layers[l];
        const __nv_bfloat16* dY = l == 3 ? S.dy4 : S.dy;
        const int ldd = Ly.N;
        // dW[n][k] = sum_r dY[r][n] X[r][k]: A(m = n, kk = r) = dY[r][n], B(kk = r, n = k) = X[r][k]
        const int mt = Ly.N / 16, nt = Ly.K / 8;
        for (int tile = warp; tile < mt * nt; tile += 4) {
            const int tm = (tile / nt) * 16, tn = (tile % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            for (int r0 = 0; r0 < kMlpTrainRows; r0 += 16) mma_tile(acc, dY, 1, ldd, Ly.X, Ly.K, 1, tm, r0, tn);
            const int rr = tm + g, cc = tn + 2 * t;
            atomicAdd(&grad[Ly.woff + rr * Ly.K + cc], acc[0]);
            atomicAdd(&grad[Ly.woff + rr * Ly.K + cc + 1], acc[1]);
            atomicAdd(&grad[Ly.woff + (rr + 8) * Ly.K + cc], acc[2]);
            atomicAdd(&grad[Ly.woff + (rr + 8) * Ly.K + cc + 1], acc[3]);
        }
        // db[n] = sum_r dY[r][n] (fp32 copy for the output layer)
        for (int nn = tid; nn < Ly.N; nn += blockDim.x) {
            float sdb = 0.f;
            for (int r = 0; r < kMlpTrainRows; ++r)
                sdb += l == 3 ? S.out[r * kMlpOutPad + nn] : __bfloat162float(dY[r * ldd + nn]);
            atomicAdd(&grad[Ly.boff + nn], sdb);
        }
        if (l == 0) break;
        // dX[r][k] = sum_n dY[r][n] W[n][k]: A(m = r, kk = n) = dY[r][n], B(kk = n, n = k) = W[n][k]
        for (int n0 = 0; n0 < Ly.K; n0 += 8) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            for (int k0 = 0; k0 < Ly.N; k0 += 16) mma_tile(acc, dY, ldd, 1, Ly.W, Ly.K, 1, m0, k0, n0);
            const int rr = m0 + g, cc = n0 + 2 * t;
            S.dh[rr * kMlpHid + cc] = acc[0];
            S.dh[rr * kMlpHid + cc + 1] = acc[1];
            S.dh[(rr + 8) * kMlpHid + cc] = acc[2];
            S.dh[(rr + 8) * kMlpHid + cc + 1] = acc[3];
        }
        __syncthreads();
        const float* Yp = S.y[l - 1];
        for (int e = tid; e < kMlpTrainRows * kMlpHid; e += blockDim.x)
            S.dy[e] = __float2bfloat16_rn(row0 + e / kMlpHid < n_rows ? S.dh[e] * gelu_grad(Yp[e]) : 0.f);
        __syncthreads();
    }
}

// AdamW on the fp32 master weights; refreshes the bf16 copy and clears `grad`.
// Padded entries (input columns >= 10 of W1, output rows >= 10 of W4 and b4)
// stay zero.
__global__ void k_mlp_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wbf, float* __restrict__ grad,
                           float* __restrict__ m1, float* __restrict__ m2, float lr, float beta1, float beta2,
                           float eps, float wd, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MlpOff::total) return;
    bool pad = false;
    if (i < MlpOff::b1) pad = (i % kMlpInPad) >= kMlpIn;
    else if (i >= MlpOff::W4 && i < MlpOff::b4) pad = (i - MlpOff::W4) / kMlpHid >= kMlpOut;
    else if (i >= MlpOff::b4) pad = (i - MlpOff::b4) >= kMlpOut;
    const float gr = grad[i];
    grad[i] = 0.f;
    if (pad) { w[i] = 0.f; wbf[i] = __float2bfloat16_rn(0.f); return; }
    const bool is_bias = (i >= MlpOff::b1 && i < MlpOff::W2) || (i >= MlpOff::b2 && i < MlpOff::W3) ||
                         (i >= MlpOff::b3 && i < MlpOff::W4) || i >= MlpOff::b4;
    const float a = beta1 * m1[i] + (1.f - beta1) * gr;
    const float b = beta2 * m2[i] + (1.f - beta2) * gr * gr;
    m1[i] = a;
    m2[i] = b;
    float x = w[i];
    if (!is_bias) x -= lr * wd * x;
    x -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
    w[i] = x;
    wbf[i] = __float2bfloat16_rn(x);
}

}  // namespace mpm

namespace mpm {

// ---------------------------------------------------------------------------
// Residual check of a predicted return map (3D). The exact map is
//   F_hat = U S_hat V^T,  F_E' = U S V^T,  S = clamp(S_hat, t0, t1),
// so with M = F_hat F_E'^-1 = U diag(S_hat / S) U^T and Q = F_E' F_E'^T =
// U S^2 U^T: M is symmetric and commutes with Q, every eigenvalue of Q lies in
// [t0^2, t1^2], and in each common eigendirection either m = 1 (unclamped) or
// q is at a band edge with m on the right side of 1:
//   (M - I)(Q - t0^2 I)(Q - t1^2 I) = 0,  (M - I)(Q - t0^2 I) >= 0,  (M - I)(Q - t1^2 I) >= 0.
// These conditions characterise the map (with M > 0, so that S_hat = M S keeps
// the sign of S). `tol` bounds the relative error of the predicted F_E': an
// error E in F_E' moves M and Q by O(|E|), so each condition is tested to the
// slack that |E| = tol |F_E'| can produce (asymmetry and commutator relative
// to |M| and |M||Q|; Q's eigenvalues to 2 tol outside the band; the sign
// conditions to -tol (w + 2|M - I|), w = t1^2 - t0^2). Semidefiniteness is
// tested by Gershgorin first and, when that is inconclusive, by Sylvester's
// criterion in FP64 on the shifted matrix. Any failure sends the particle to
// the exact SVD.
__device__ __forceinline__ bool gersh_min_ge(const float* S, float bound) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float r = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (j != i) r += fabsf(S[i * 3 + j]);
        if (S[i * 4] - r < bound) return false;
    }
    return true;
}

// A symmetric 3x3 S satisfies S >= bound I (bound <= 0): Gershgorin, else
// Sylvester's criterion on S - 1.0001 bound I in FP64.
__device__ __forceinline__ bool sym_min_ge(const float* S, float bound) {
    if (gersh_min_ge(S, bound)) return true;
    double D[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) D[k] = double(S[k]) - (k % 4 == 0 ? 1.0001 * double(bound) : 0.0);
    return D[0] > 0.0 && D[0] * D[4] - D[1] * D[3] > 0.0 && det<3>(D) > 0.0;
}

__device__ __forceinline__ bool mlp_residual_ok(const float* Fh, const float* Fe, float t0, float t1, float tol) {
    const float dE = det<3>(Fe);
    if (!(dE > 0.f) || !(det<3>(Fh) > 0.f)) return false;
    float inv[9];
    const float r = 1.f / dE;
    inv[0] = (Fe[4] * Fe[8] - Fe[5] * Fe[7]) * r;
    inv[1] = (Fe[2] * Fe[7] - Fe[1] * Fe[8]) * r;
    inv[2] = (Fe[1] * Fe[5] - Fe[2] * Fe[4]) * r;
    inv[3] = (Fe[5] * Fe[6] - Fe[3] * Fe[8]) * r;
    inv[4] = (Fe[0] * Fe[8] - Fe[2] * Fe[6]) * r;
    inv[5] = (Fe[2] * Fe[3] - Fe[0] * Fe[5]) * r;
    inv[6] = (Fe[3] * Fe[7] - Fe[4] * Fe[6]) * r;
    inv[7] = (Fe[1] * Fe[6] - Fe[0] * Fe[7]) * r;
    inv[8] = (Fe[0] * Fe[4] - Fe[1] * Fe[3]) * r;
    float M[9], Q[9];
    matmul<3>(Fh, inv, M);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Q[i * 3 + j] = Fe[i * 3] * Fe[j * 3] + Fe[i * 3 + 1] * Fe[j * 3 + 1] + Fe[i * 3 + 2] * Fe[j * 3 + 2];
    float asym = 0.f, nm = 0.f;
    float Ms[9], G[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float a = M[i * 3 + j] - M[j * 3 + i];
            asym += a * a;
            nm += M[i * 3 + j] * M[i * 3 + j];
            Ms[i * 3 + j] = 0.5f * (M[i * 3 + j] + M[j * 3 + i]);
            G[i * 3 + j] = Ms[i * 3 + j] - (i == j ? 1.f : 0.f);
        }
    if (asym > tol * tol * nm) return false;
    // commutation
    float MQ[9], QM[9];
    matmul<3>(Ms, Q, MQ);
    matmul<3>(Q, Ms, QM);
    float comm = 0.f, nq = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) { comm += (MQ[k] - QM[k]) * (MQ[k] - QM[k]); nq += Q[k] * Q[k]; }
    if (comm > tol * tol * nm * nq) return false;
    // band of Q
    const float a0 = t0 * t0, a1 = t1 * t1, w = a1 - a0;
    float Ql[9], Qh[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { Ql[k] = Q[k] - (k % 4 == 0 ? a0 : 0.f); Qh[k] = (k % 4 == 0 ? a1 : 0.f) - Q[k]; }
    if (!sym_min_ge(Ql, -2.f * tol) || !sym_min_ge(Qh, -2.f * tol)) return false;
    if (!gersh_min_ge(Ms, 0.5f)) return false;
    // (M - I)(Q - t0^2)(Q - t1^2) = 0 and the sign conditions
    float GL[9], GH[9], P[9];
    float Qh_neg[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Qh_neg[k] = -Qh[k];  // Q - t1^2 I
    matmul<3>(G, Ql, GL);
    matmul<3>(G, Qh_neg, GH);
    matmul<3>(GL, Qh_neg, P);
    float np = 0.f, ng = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) { np += P[k] * P[k]; ng += G[k] * G[k]; }
    if (np > tol * tol * (1.f + ng) * w * w * w * w) return false;
    float GLs[9], GHs[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            GLs[i * 3 + j] = 0.5f * (GL[i * 3 + j] + GL[j * 3 + i]);
            GHs[i * 3 + j] = 0.5f * (GH[i * 3 + j] + GH[j * 3 + i]);
        }
    const float sg = -tol * (w + 2.f * sqrtf(ng));
    if (!sym_min_ge(GLs, sg) || !sym_min_ge(GHs, sg)) return false;
    return true;
}

struct MlpParams {
    const __nv_bfloat16* wbf;
    const float* wf32;
    MlpNorm norm;
    float tol;
    unsigned long long* counters;  // [0] accepted, [1] rejected (fell back to the SVD)
};

// ---------------------------------------------------------------------------
// Warp-tiled inference for the solver. Each warp takes 32 queued particles
// (lane = particle) and runs the network on them as two 16-row tiles whose
// activations never leave registers: the m16n8 accumulators of one layer,
// after bias + GELU, are packed to bf16 pairs that are exactly the m16k16 A
// fragments of the next layer (accumulator n-tiles 2kb, 2kb+1 = A k-block kb).
// Weights sit in shared memory with rows padded by 8 bf16 so that the B
// fragment loads of a warp hit 32 distinct banks.
constexpr int kMwIn = kMlpInPad + 8;  // row stride (bf16) of W1 and of the input tile
constexpr int kMwHid = kMlpHid + 8;   // row stride (bf16) of W2, W3, W4
constexpr int kMwOut = kMlpOutPad + 2;  // row stride (fp32) of the output tile
constexpr int kMlpWarps = 8;

struct MlpWarpSmem {
    __nv_bfloat16 W1[kMlpHid * kMwIn];
    __nv_bfloat16 W2[kMlpHid * kMwHid];
    __nv_bfloat16 W3[kMlpHid * kMwHid];
    __nv_bfloat16 W4[kMlpOutPad * kMwHid];
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpHid], b4[kMlpOutPad];
    __nv_bfloat16 x[kMlpWarps][32 * kMwIn];
    float out[kMlpWarps][32 * kMwOut];
};

__device__ __forceinline__ void mlp_stage_matrix(__nv_bfloat16* dst, int ld_dst, const __nv_bfloat16* src, int rows,
                                                 int cols) {
    const int vpr = cols / 8;  // 16-byte vectors per row
    for (int v = threadIdx.x; v < rows * vpr; v += blockDim.x) {
        const int r = v / vpr, c = (v % vpr) * 8;
        *reinterpret_cast<uint4*>(dst + r * ld_dst + c) = *reinterpret_cast<const uint4*>(src + r * cols + c);
    }
}

__device__ __forceinline__ void mlp_stage_weights(MlpWarpSmem& S, const __nv_bfloat16* wbf, const float* wf32) {
    mlp_stage_matrix(S.W1, kMwIn, wbf + MlpOff::W1, kMlpHid, kMlpInPad);
    mlp_stage_matrix(S.W2, kMwHid, wbf + MlpOff::W2, kMlpHid, kMlpHid);
    mlp_stage_matrix(S.W3, kMwHid, wbf + MlpOff::W3, kMlpHid, kMlpHid);
    mlp_stage_matrix(S.W4, kMwHid, wbf + MlpOff::W4, kMlpOutPad, kMlpHid);
    for (int i = threadIdx.x; i < kMlpHid; i += blockDim.x) {
        S.b1[i] = wf32[MlpOff::b1 + i];
        S.b2[i] = wf32[MlpOff::b2 + i];
        S.b3[i] = wf32[MlpOff::b3 + i];
    }
    for (int i = threadIdx.x; i < kMlpOutPad; i += blockDim.x) S.b4[i] = wf32[MlpOff::b4 + i];
}

__device__ __forceinline__ uint32_t pack_f2_bf16(float lo, float hi) {
    return pack_bf16(__float2bfloat16_rn(lo), __float2bfloat16_rn(hi));
}

// acc[j] (n-tile j of a 16 x 8*NT output) = A (16 x 16*KB, fragments a[kb]) * W^T,
// W row-major [out][in] in shared memory with row stride ld.
template <int KB, int NT>
__device__ __forceinline__ void mlp_warp_layer(const uint32_t (*a)[4], const __nv_bfloat16* W, int ld, float (*acc)[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
        const __nv_bfloat16* w = W + (j * 8 + g) * ld + 2 * t;
#pragma unroll
        for (int kb = 0; kb < KB; ++kb) {
            uint32_t b[2];
            b[0] = *reinterpret_cast<const uint32_t*>(w + kb * 16);
            b[1] = *reinterpret_cast<const uint32_t*>(w + kb * 16 + 8);
            mma_bf16(acc[j], a[kb], b);
        }
    }
}

// bias + GELU on a 16 x 64 accumulator, packed into the A fragments of the next layer.
__device__ __forceinline__ void mlp_warp_activate(float (*acc)[4], const float* bias, uint32_t (*a)[4]) {
    const int t = threadIdx.x & 3;
#pragma unroll
    for (int kb = 0; kb < kMlpHid / 16; ++kb)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = 2 * kb + h, c = j * 8 + 2 * t;
            const float b0 = bias[c], b1 = bias[c + 1];
            a[kb][2 * h] = pack_f2_bf16(gelu(acc[j][0] + b0), gelu(acc[j][1] + b1));
            a[kb][2 * h + 1] = pack_f2_bf16(gelu(acc[j][2] + b0), gelu(acc[j][3] + b1));
        }
}

// Network on the warp's 32-row input tile X (bf16, row stride kMwIn) -> O
// (fp32, normalised outputs, row stride kMwOut).
__device__ __forceinline__ void mlp_warp_forward(const MlpWarpSmem& S, const __nv_bfloat16* X, float* O) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int mt = 0; mt < 2; ++mt) {
        const int r0 = mt * 16 + g;
        uint32_t a[kMlpHid / 16][4];
        a[0][0] = *reinterpret_cast<const uint32_t*>(X + r0 * kMwIn + 2 * t);
        a[0][1] = *reinterpret_cast<const uint32_t*>(X + (r0 + 8) * kMwIn + 2 * t);
        a[0][2] = *reinterpret_cast<const uint32_t*>(X + r0 * kMwIn + 2 * t + 8);
        a[0][3] = *reinterpret_cast<const uint32_t*>(X + (r0 + 8) * kMwIn + 2 * t + 8);
        float acc[kMlpHid / 8][4];
        mlp_warp_layer<1, kMlpHid / 8>(a, S.W1, kMwIn, acc);
        mlp_warp_activate(acc, S.b1, a);
        mlp_warp_layer<kMlpHid / 16, kMlpHid / 8>(a, S.W2, kMwHid, acc);
        mlp_warp_activate(acc, S.b2, a);
        mlp_warp_layer<kMlpHid / 16, kMlpHid / 8>(a, S.W3, kMwHid, acc);
        mlp_warp_activate(acc, S.b3, a);
        float o[kMlpOutPad / 8][4];
        mlp_warp_layer<kMlpHid / 16, kMlpOutPad / 8>(a, S.W4, kMwHid, o);
#pragma unroll
        for (int j = 0; j < kMlpOutPad / 8; ++j) {
            const int c = j * 8 + 2 * t;
            *reinterpret_cast<float2*>(O + r0 * kMwOut + c) = make_float2(o[j][0] + S.b4[c], o[j][1] + S.b4[c + 1]);
            *reinterpret_cast<float2*>(O + (r0 + 8) * kMwOut + c) =
                make_float2(o[j][2] + S.b4[c], o[j][3] + S.b4[c + 1]);
        }
    }
}

// Learned return map of the queued particles (3D tiled MLS path). Accepted
// predictions write F_E', J_p' and the next step's affine matrix and mark
// their queue entry kQueueDone; the rest (rejected by the residual check or
// by the stress series, and grid-clipped stencils) stay queued for
// k_g2p_plastic's exact return map, which runs next.
__global__ void __launch_bounds__(kMlpWarps * 32) k_return_map_mlp(Particles P, StepConsts C, SlowQueue Q,
                                                                   MlpParams ML) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpWarpSmem& S = *reinterpret_cast<MlpWarpSmem*>(smem_raw);
    const int m = *Q.count;
    // CTAs past the queue's end leave before staging the weights (the grid is
    // sized for the largest queue; most steps queue far fewer particles)
    if ((long long)blockIdx.x * kMlpWarps * 32 >= m) return;
    mlp_stage_weights(S, ML.wbf, ML.wf32);
    __syncthreads();
    const int n = P.n;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __nv_bfloat16* X = S.x[wid];
    float* O = S.out[wid];
    const float t0 = 1.f - C.theta_c, t1 = 1.f + C.theta_s;
    unsigned n_ok = 0, n_bad = 0;
    const int warps = gridDim.x * kMlpWarps;
    for (int base = (blockIdx.x * kMlpWarps + wid) * 32; base < m; base += warps * 32) {
        const int e = base + lane;
        const int entry = e < m ? Q.list[e] : -1;
        const bool valid = entry >= 0;
        float Fh[9], Jp0 = 1.f, B[9], mass = 0.f, vol = 0.f;
        float in[kMlpIn];
        if (valid) {
#pragma unroll
            for (int k = 0; k < 9; ++k) Fh[k] = Q.fh[k * Q.capacity + e];
            Jp0 = P.Jp[entry];
            // the particle's B, mass and volume, loaded now so that their
            // latency overlaps the network
#pragma unroll
            for (int k = 0; k < 9; ++k) B[k] = P.B[k * n + entry];
            mass = P.mass ? P.mass[entry] : P.mass_u;
            vol = P.vol ? P.vol[entry] : P.vol_u;
            mlp_features(Fh, Jp0, ML.norm, in);
        }
        uint32_t* xr = reinterpret_cast<uint32_t*>(X + lane * kMwIn);
#pragma unroll
        for (int k = 0; k < kMlpInPad / 2; ++k) {
            const float lo = valid && 2 * k < kMlpIn ? in[2 * k] : 0.f;
            const float hi = valid && 2 * k + 1 < kMlpIn ? in[2 * k + 1] : 0.f;
            xr[k] = pack_f2_bf16(lo, hi);
        }
        __syncwarp();
        if (__any_sync(0xffffffffu, valid)) mlp_warp_forward(S, X, O);
        __syncwarp();
        if (valid) {
            const float* o = O + lane * kMwOut;
            float Fp[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) Fp[k] = Fh[k] + (o[k] * ML.norm.out_std[k] + ML.norm.out_mean[k]);
            const float dlj = o[9] * ML.norm.out_std[9] + ML.norm.out_mean[9];
            bool ok = mlp_residual_ok(Fh, Fp, t0, t1, ML.tol);
            float ratio = 1.f;
            if (ok) {
                // J_p' = J_p det(F_hat) / det(F_E') (= J_p prod(S_hat / S)); the
                // network's log J_p' output must agree with it within the tolerance.
                ratio = det<3>(Fh) / det<3>(Fp);
                ok = fabsf(logf(ratio) - dlj) <= ML.tol * (1.f + fabsf(dlj));
            }
            float sig[9];
            const float Jp = Jp0 * ratio;
            if (ok) ok = hardened_stress_series<3>(Fp, Jp, C.mu0, C.la0, C.xi, sig);
            if (ok) {
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    P.Fe[k * n + entry] = Fp[k];
                    P.A[k * n + entry] = 3.f * mass * B[k] - 3.f * C.dt * vol * sig[k];
                }
                P.Jp[entry] = Jp;
                Q.list[e] = kQueueDone;
                ++n_ok;
            } else {
                ++n_bad;
            }
        }
        __syncwarp();
    }
    if (ML.counters) {
        n_ok = __reduce_add_sync(0xffffffffu, n_ok);
        n_bad = __reduce_add_sync(0xffffffffu, n_bad);
        if (lane == 0) {
            if (n_ok) atomicAdd(&ML.counters[0], (unsigned long long)n_ok);
            if (n_bad) atomicAdd(&ML.counters[1], (unsigned long long)n_bad);
        }
    }
}

// Batched inference on raw pairs' inputs (evaluation and tests), through the
// same warp-tiled path as the solver: out[n][10] = denormalised
// (F_E' - F_hat, log J_p' - log J_p). Rows: input + stride * i, F_hat[9], J_p.
__global__ void __launch_bounds__(kMlpWarps * 32) k_mlp_forward(const float* __restrict__ inputs, int stride, int n,
                                                                const __nv_bfloat16* __restrict__ wbf,
                                                                const float* __restrict__ wf32, MlpNorm N,
                                                                float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpWarpSmem& S = *reinterpret_cast<MlpWarpSmem*>(smem_raw);
    mlp_stage_weights(S, wbf, wf32);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __nv_bfloat16* X = S.x[wid];
    float* O = S.out[wid];
    const int row = (blockIdx.x * kMlpWarps + wid) * 32 + lane;
    const bool valid = row < n;
    float in[kMlpIn];
    if (valid) mlp_features(inputs + (long long)row * stride, inputs[(long long)row * stride + 9], N, in);
    uint32_t* xr = reinterpret_cast<uint32_t*>(X + lane * kMwIn);
#pragma unroll
    for (int k = 0; k < kMlpInPad / 2; ++k)
        xr[k] = pack_f2_bf16(valid && 2 * k < kMlpIn ? in[2 * k] : 0.f, valid && 2 * k + 1 < kMlpIn ? in[2 * k + 1] : 0.f);
    __syncwarp();
    mlp_warp_forward(S, X, O);
    __syncwarp();
    if (valid)
#pragma unroll
        for (int c = 0; c < kMlpOut; ++c) out[(long long)row * kMlpOut + c] = O[lane * kMwOut + c] * N.out_std[c] + N.out_mean[c];
}

}  // namespace mpm
