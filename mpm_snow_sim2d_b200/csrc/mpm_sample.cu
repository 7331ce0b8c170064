// Seeded Poisson-disk sampling of snow shapes on the device: the reference's
// PoissonDiskCircle / PoissonDiskSphere (src/shared/Shapes.h:17-117,143-234,
// Bridson's sequential algorithm seeded from std::random_device) replaced by a
// parallel, reproducible grid-phase dart thrower.
//
// Background grid of cells of side min_dist / sqrt(dim): a cell holds at most
// one sample. Cells whose indices agree modulo 3 on every axis form a phase;
// two cells of one phase are at least 2 cell sides = 2 min_dist / sqrt(dim) >=
// min_dist apart, so every cell of a phase can try a candidate at once without
// two new samples conflicting. Each round visits the 3^dim phases in order;
// in each, every empty cell that overlaps a shape draws one candidate
// uniformly in the cell from a counter-based hash of (seed, cell, round, axis)
// and keeps it when it lies in a shape and no sample in the 5^dim surrounding
// cells is closer than min_dist. The result depends on the seed alone.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mpm/mpm.h"

namespace {

constexpr int kMaxShapes = 64;

struct SampleShapes {
    int n;
    int kind[kMaxShapes];
    float c[kMaxShapes][3], r[kMaxShapes], h[kMaxShapes][3];
};

struct SampleGrid {
    int dim;
    int nc[3];          // cells per axis
    float origin[3];
    float cell, min_dist;
    unsigned long long seed;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014)
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ float uniform01(unsigned long long seed, long long cell, int round, int axis) {
    const unsigned long long h =
        mix64(seed ^ mix64((unsigned long long)cell * 4 + (unsigned long long)axis + ((unsigned long long)round << 40)));
    return float(h >> 40) * (1.0f / 16777216.0f);  // 24 bits: exactly representable in [0, 1)
}

// Every floating-point step below is an explicitly rounded operation (no
// fused multiply-add), so that a float32 restatement on the CPU reproduces
// the samples bit for bit.
__device__ __forceinline__ bool inside(const SampleShapes& S, int dim, const float* p) {
    for (int s = 0; s < S.n; ++s) {
        if (S.kind[s] == MPM_SHAPE_BALL) {
            float d2 = 0.f;
            for (int k = 0; k < dim; ++k) {
                const float d = __fsub_rn(p[k], S.c[s][k]);
                d2 = __fadd_rn(d2, __fmul_rn(d, d));
            }
            if (d2 <= __fmul_rn(S.r[s], S.r[s])) return true;
        } else {
            bool in = true;
            for (int k = 0; k < dim; ++k) in = in && fabsf(__fsub_rn(p[k], S.c[s][k])) <= S.h[s][k];
            if (in) return true;
        }
    }
    return false;
}

// One phase of one round: cells (3a + px, 3b + py, 3c + pz).
__global__ void k_sample_phase(SampleGrid G, SampleShapes S, const unsigned char* __restrict__ live, int round,
                               int px, int py, int pz, float4* __restrict__ cells) {
    const int mx = (G.nc[0] - px + 2) / 3, my = (G.nc[1] - py + 2) / 3, mz = G.dim == 3 ? (G.nc[2] - pz + 2) / 3 : 1;
    const long long total = (long long)mx * my * mz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int ix = 3 * int(t % mx) + px, iy = 3 * int((t / mx) % my) + py, iz = G.dim == 3 ? 3 * int(t / ((long long)mx * my)) + pz : 0;
    if (ix >= G.nc[0] || iy >= G.nc[1] || (G.dim == 3 && iz >= G.nc[2])) return;
    const long long id = ((long long)iz * G.nc[1] + iy) * G.nc[0] + ix;
    if (!live[id] || cells[id].w != 0.f) return;
    const int ic[3] = {ix, iy, iz};
    float p[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < G.dim; ++k)
        p[k] = __fadd_rn(G.origin[k], __fmul_rn(__fadd_rn(float(ic[k]), uniform01(G.seed, id, round, k)), G.cell));
    if (!inside(S, G.dim, p)) return;
    const float r2 = __fmul_rn(G.min_dist, G.min_dist);
    const int zr = G.dim == 3 ? 2 : 0;
    for (int dz = -zr; dz <= zr; ++dz)
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx) {
                const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                if (jx < 0 || jy < 0 || jz < 0 || jx >= G.nc[0] || jy >= G.nc[1] || (G.dim == 3 && jz >= G.nc[2])) continue;
                const float4 q = cells[((long long)jz * G.nc[1] + jy) * G.nc[0] + jx];
                if (q.w == 0.f) continue;
                const float ddx = __fsub_rn(q.x, p[0]), ddy = __fsub_rn(q.y, p[1]), ddz = __fsub_rn(q.z, p[2]);
                if (__fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), __fmul_rn(ddz, ddz)) < r2) return;
            }
    cells[id] = make_float4(p[0], p[1], p[2], 1.f);
}

// Cells that can hold a sample: those overlapping a shape's bounding box.
__global__ void k_sample_live(SampleGrid G, SampleShapes S, long long ncells, unsigned char* __restrict__ live) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= ncells) return;
    const int ic[3] = {int(id % G.nc[0]), int((id / G.nc[0]) % G.nc[1]), int(id / ((long long)G.nc[0] * G.nc[1]))};
    bool any = false;
    for (int s = 0; s < S.n && !any; ++s) {
        bool in = true;
        for (int k = 0; k < G.dim; ++k) {
            const float lo = __fadd_rn(G.origin[k], __fmul_rn(float(ic[k]), G.cell)), hi = __fadd_rn(lo, G.cell);
            const float e = S.kind[s] == MPM_SHAPE_BALL ? S.r[s] : S.h[s][k];
            in = in && hi >= __fsub_rn(S.c[s][k], e) && lo <= __fadd_rn(S.c[s][k], e);
        }
        any = in;
    }
    live[id] = any ? 1 : 0;
}

// Which shape a sample belongs to (the first that contains it).
int shape_index(const SampleShapes& S, int dim, const float* p) {
    for (int s = 0; s < S.n; ++s) {
        if (S.kind[s] == MPM_SHAPE_BALL) {
            float d2 = 0.f;
            for (int k = 0; k < dim; ++k) { const float d = p[k] - S.c[s][k]; d2 += d * d; }
            if (d2 <= S.r[s] * S.r[s]) return s;
        } else {
            bool in = true;
            for (int k = 0; k < dim; ++k) in = in && std::fabs(p[k] - S.c[s][k]) <= S.h[s][k];
            if (in) return s;
        }
    }
    return -1;
}

}  // namespace

extern "C" {

mpm_status mpm_sample_shapes(int32_t dim, const mpm_shape* shapes, int32_t nshapes, float min_dist, uint64_t seed,
                             int32_t rounds, float* positions, int32_t* shape_of, int64_t capacity, int64_t* count) {
    if ((dim != 2 && dim != 3) || !shapes || nshapes < 1 || nshapes > kMaxShapes || !(min_dist > 0.f) ||
        !std::isfinite(min_dist) || rounds < 1 || rounds > 1000 || !count || capacity < 0 ||
        (capacity > 0 && !positions))
        return MPM_ERR_INVALID_ARGUMENT;
    *count = 0;
    SampleShapes S{};
    S.n = nshapes;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int s = 0; s < nshapes; ++s) {
        const mpm_shape& sh = shapes[s];
        if (sh.kind != MPM_SHAPE_BALL && sh.kind != MPM_SHAPE_BOX) return MPM_ERR_INVALID_ARGUMENT;
        S.kind[s] = sh.kind;
        S.r[s] = sh.radius;
        for (int k = 0; k < 3; ++k) { S.c[s][k] = sh.center[k]; S.h[s][k] = sh.half[k]; }
        for (int k = 0; k < dim; ++k) {
            const float e = sh.kind == MPM_SHAPE_BALL ? sh.radius : sh.half[k];
            if (!(e >= 0.f) || !std::isfinite(e) || !std::isfinite(sh.center[k])) return MPM_ERR_INVALID_ARGUMENT;
            lo[k] = s == 0 ? sh.center[k] - e : std::min(lo[k], sh.center[k] - e);
            hi[k] = s == 0 ? sh.center[k] + e : std::max(hi[k], sh.center[k] + e);
        }
    }
    SampleGrid G{};
    G.dim = dim;
    G.min_dist = min_dist;
    G.cell = min_dist / std::sqrt((float)dim);
    G.seed = seed;
    double ncd = 1.0;
    for (int k = 0; k < 3; ++k) {
        G.origin[k] = k < dim ? lo[k] : 0.f;
        G.nc[k] = k < dim ? std::max(1, (int)std::ceil((hi[k] - lo[k]) / G.cell) + 1) : 1;
        ncd *= G.nc[k];
    }
    if (ncd > 4.0e8) return MPM_ERR_CAPACITY;  // 6.4 GB of cells: refuse rather than exhaust the device
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return MPM_ERR_NO_DEVICE; }
    const long long ncells = (long long)ncd;
    float4* cells = nullptr;
    unsigned char* live = nullptr;
    if (cudaMalloc(&cells, sizeof(float4) * ncells) != cudaSuccess ||
        cudaMalloc(&live, (size_t)ncells) != cudaSuccess) {
        if (cells) cudaFree(cells);
        cudaGetLastError();
        return MPM_ERR_OUT_OF_MEMORY;
    }
    mpm_status st = MPM_OK;
    if (cudaMemset(cells, 0, sizeof(float4) * ncells) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(cells);
        cudaFree(live);
        return MPM_ERR_CUDA;
    }
    const int threads = 256;
    k_sample_live<<<(unsigned)((ncells + threads - 1) / threads), threads>>>(G, S, ncells, live);
    const int pz_n = dim == 3 ? 3 : 1;
    for (int r = 0; r < rounds; ++r)
        for (int pz = 0; pz < pz_n; ++pz)
            for (int py = 0; py < 3; ++py)
                for (int px = 0; px < 3; ++px) {
                    const long long mx = (G.nc[0] - px + 2) / 3, my = (G.nc[1] - py + 2) / 3,
                                    mz = dim == 3 ? (G.nc[2] - pz + 2) / 3 : 1;
                    const long long total = mx * my * mz;
                    if (total > 0)
                        k_sample_phase<<<(unsigned)((total + threads - 1) / threads), threads>>>(G, S, live, r, px, py,
                                                                                                 pz, cells);
                }
    std::vector<float4> h(ncells);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpy(h.data(), cells, sizeof(float4) * ncells, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        st = MPM_ERR_CUDA;
    }
    cudaFree(cells);
    cudaFree(live);
    if (st != MPM_OK) return st;
    // compaction in cell order (deterministic)
    int64_t n = 0;
    for (long long i = 0; i < ncells; ++i) {
        if (h[i].w == 0.f) continue;
        if (n < capacity) {
            const float p[3] = {h[i].x, h[i].y, h[i].z};
            for (int k = 0; k < dim; ++k) positions[n * dim + k] = p[k];
            if (shape_of) shape_of[n] = shape_index(S, dim, p);
        }
        ++n;
    }
    *count = n;
    return n > capacity ? MPM_ERR_CAPACITY : MPM_OK;
}

}  // extern "C"
