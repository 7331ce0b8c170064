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

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

// Raw pair -> normalised network input (row of kMlpInPad bf16) and target.
// Pair layout (20 floats): F_hat[9] J_p[1] F_E'[9] J_p'[1].
__device__ __forceinline__ void mlp_features(const float* Fh, float Jp, const MlpNorm& N, float* in) {
#pragma unroll
    for (int k = 0; k < 9; ++k) in[k] = ((Fh[k] - (k % 4 == 0 ? 1.f : 0.f)) - N.in_mean[k]) / N.in_std[k];
    in[9] = (logf(Jp) - N.in_mean[9]) / N.in_std[9];
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

// ---------------------------------------------------------------------------
// Inference on a tile of up to 64 particles (4 warps x 16 rows) held in
// shared memory: in (bf16 [64][16]) -> out (fp32 [64][16], normalised).
struct MlpInferSmem {
    __nv_bfloat16 w[MlpOff::total];
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpHid], b4[kMlpOutPad];
    __nv_bfloat16 x0[kMlpTrainRows * kMlpInPad];
    __nv_bfloat16 h[2][kMlpTrainRows * kMlpHid];
    float out[kMlpTrainRows * kMlpOutPad];
};

__device__ __forceinline__ void mlp_load_weights(MlpInferSmem& S, const __nv_bfloat16* wbf, const float* wf32) {
    for (int i = threadIdx.x; i < MlpOff::total; i += blockDim.x) S.w[i] = wbf[i];
    for (int i = threadIdx.x; i < kMlpHid; i += blockDim.x) {
        S.b1[i] = wf32[MlpOff::b1 + i];
        S.b2[i] = wf32[MlpOff::b2 + i];
        S.b3[i] = wf32[MlpOff::b3 + i];
    }
    for (int i = threadIdx.x; i < kMlpOutPad; i += blockDim.x) S.b4[i] = wf32[MlpOff::b4 + i];
}

__device__ __forceinline__ void mlp_infer_tile(MlpInferSmem& S) {
    const int m0 = (threadIdx.x >> 5) * 16;
    mlp_layer_fwd(S.x0, kMlpInPad, kMlpInPad, S.w + MlpOff::W1, S.b1, kMlpHid, m0, nullptr, 0, S.h[0], kMlpHid, true);
    __syncwarp();
    mlp_layer_fwd(S.h[0], kMlpHid, kMlpHid, S.w + MlpOff::W2, S.b2, kMlpHid, m0, nullptr, 0, S.h[1], kMlpHid, true);
    __syncwarp();
    mlp_layer_fwd(S.h[1], kMlpHid, kMlpHid, S.w + MlpOff::W3, S.b3, kMlpHid, m0, nullptr, 0, S.h[0], kMlpHid, true);
    __syncwarp();
    mlp_layer_fwd(S.h[0], kMlpHid, kMlpHid, S.w + MlpOff::W4, S.b4, kMlpOutPad, m0, S.out, kMlpOutPad, nullptr, 0,
                  false);
    __syncwarp();
}

// Batched inference on raw pairs' inputs (testing / evaluation): out[n][10]
// = denormalised (F_E' - F_hat, log J_p' - log J_p).
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ inputs, int stride, int n,
                                                     const __nv_bfloat16* __restrict__ wbf,
                                                     const float* __restrict__ wf32, MlpNorm N,
                                                     float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpInferSmem& S = *reinterpret_cast<MlpInferSmem*>(smem_raw);
    mlp_load_weights(S, wbf, wf32);
    const int row0 = blockIdx.x * kMlpTrainRows;
    for (int r = threadIdx.x; r < kMlpTrainRows; r += blockDim.x) {
        float in[kMlpIn];
        const bool valid = row0 + r < n;
        if (valid) mlp_features(inputs + (long long)(row0 + r) * stride, inputs[(long long)(row0 + r) * stride + 9], N, in);
        for (int k = 0; k < kMlpInPad; ++k) S.x0[r * kMlpInPad + k] = __float2bfloat16_rn(valid && k < kMlpIn ? in[k] : 0.f);
    }
    __syncthreads();
    mlp_infer_tile(S);
    __syncthreads();
    for (int e = threadIdx.x; e < kMlpTrainRows * kMlpOut; e += blockDim.x) {
        const int r = e / kMlpOut, c = e % kMlpOut;
        if (row0 + r < n) out[(long long)(row0 + r) * kMlpOut + c] = S.out[r * kMlpOutPad + c] * N.out_std[c] + N.out_mean[c];
    }
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
    inv[0] = (Fe[4] * Fe[8] - Fe[5] * Fe[7]) / dE;
    inv[1] = (Fe[2] * Fe[7] - Fe[1] * Fe[8]) / dE;
    inv[2] = (Fe[1] * Fe[5] - Fe[2] * Fe[4]) / dE;
    inv[3] = (Fe[5] * Fe[6] - Fe[3] * Fe[8]) / dE;
    inv[4] = (Fe[0] * Fe[8] - Fe[2] * Fe[6]) / dE;
    inv[5] = (Fe[2] * Fe[3] - Fe[0] * Fe[5]) / dE;
    inv[6] = (Fe[3] * Fe[7] - Fe[4] * Fe[6]) / dE;
    inv[7] = (Fe[1] * Fe[6] - Fe[0] * Fe[7]) / dE;
    inv[8] = (Fe[0] * Fe[4] - Fe[1] * Fe[3]) / dE;
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

// Queued particles of the tiled MLS path with the learned return map: out-of-
// band trial F goes through the network (64 per tile on the tensor cores) and
// the residual check; failures and grid-clipped stencils take the exact path.
__global__ void __launch_bounds__(128) k_g2p_plastic_mlp(Particles P, StepConsts C, const float4* __restrict__ gv,
                                                         SlowQueue Q, MlpParams ML, unsigned* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpInferSmem& S = *reinterpret_cast<MlpInferSmem*>(smem_raw);
    mlp_load_weights(S, ML.wbf, ML.wf32);
    const int m = *Q.count;
    const int n = P.n;
    const int tid = threadIdx.x;
    const float t0 = 1.f - C.theta_c, t1 = 1.f + C.theta_s;
    unsigned long long acc_ok = 0, acc_bad = 0;
    for (int base = blockIdx.x * kMlpTrainRows; base < m; base += gridDim.x * kMlpTrainRows) {
        __syncthreads();
        if (tid < kMlpTrainRows) {
            const int e = base + tid;
            float in[kMlpIn];
            bool valid = e < m && Q.list[e] >= 0;
            if (valid) {
                float Fh[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) Fh[k] = Q.fh[k * Q.capacity + e];
                mlp_features(Fh, P.Jp[Q.list[e]], ML.norm, in);
            }
#pragma unroll
            for (int k = 0; k < kMlpInPad; ++k)
                S.x0[tid * kMlpInPad + k] = __float2bfloat16_rn(valid && k < kMlpIn ? in[k] : 0.f);
        }
        __syncthreads();
        mlp_infer_tile(S);
        __syncthreads();
        if (tid < kMlpTrainRows && base + tid < m) {
            const int e = base + tid;
            const int entry = Q.list[e];
            const int i = entry >= 0 ? entry : -1 - entry;
            float Fh[9], Fe[9], B[9], A[9];
            bool done = false;
            if (entry >= 0) {
#pragma unroll
                for (int k = 0; k < 9; ++k) { Fh[k] = Q.fh[k * Q.capacity + e]; B[k] = P.B[k * n + i]; }
                float Fp[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) Fp[k] = Fh[k] + (S.out[tid * kMlpOutPad + k] * ML.norm.out_std[k] + ML.norm.out_mean[k]);
                const float dlj = S.out[tid * kMlpOutPad + 9] * ML.norm.out_std[9] + ML.norm.out_mean[9];
                if (mlp_residual_ok(Fh, Fp, t0, t1, ML.tol)) {
                    // J_p' = J_p det(F_hat) / det(F_E') (= J_p prod(S_hat / S)); the network's
                    // log J_p' output must agree with it within the tolerance.
                    const float ratio = det<3>(Fh) / det<3>(Fp);
                    if (fabsf(logf(ratio) - dlj) <= ML.tol * (1.f + fabsf(dlj))) {
                        float Jp = P.Jp[i] * ratio;
#pragma unroll
                        for (int k = 0; k < 9; ++k) { P.Fe[k * n + i] = Fp[k]; Fe[k] = Fp[k]; }
                        P.Jp[i] = Jp;
                        mls_affine<3>(C, B, Fe, Jp, P.mass ? P.mass[i] : P.mass_u, P.vol ? P.vol[i] : P.vol_u, A);
#pragma unroll
                        for (int k = 0; k < 9; ++k) P.A[k * n + i] = A[k];
                        done = true;
                        ++acc_ok;
                    }
                }
                if (!done) ++acc_bad;
            }
            if (!done) g2p_queued_exact<3>(P, C, gv, Q, e, status);
        }
    }
    if (ML.counters) {
        if (acc_ok) atomicAdd(&ML.counters[0], acc_ok);
        if (acc_bad) atomicAdd(&ML.counters[1], acc_bad);
    }
}

}  // namespace mpm
