// Headless point rasteriser: the reference's Visualize + saveFrame
// (src/main.cpp:51-205) without a graphics API. Particles are white discs of
// PARTICLE_SIZE pixels with a smooth edge (GL_POINT_SMOOTH), the domain border
// (2D rectangle / 3D wireframe box at BORDER_MARGIN) gray lines 2 pixels wide;
// 2D maps [0, WIDTH] x [0, HEIGHT] onto the image (glOrtho), 3D uses the
// reference's orbit camera (glm::perspective 45 deg, near 1, far 1000, lookAt
// the grid centre from angle / elevation / distance).
//
// Every fragment is written as one 64-bit atomicMin of (depth bits << 32 |
// 255 - intensity) into a per-pixel word: the nearest fragment wins (the depth
// test), ties go to the brighter one, and the image does not depend on the
// order of the atomics. A final pass packs the words into RGB8 rows, top row
// first (the vertically flipped glReadPixels buffer that saveFrame writes).
#pragma once

#include "mpm_kernels.cuh"

namespace mpm {

struct RenderView {
    int dim;
    int width, height;      // image
    float radius;           // point radius in pixels (PARTICLE_SIZE / 2)
    // 2D: pixel = (x * sx, height - y * sy)
    float sx, sy;
    // 3D: eye, camera basis (s, u, f) and projection scales (1 / (aspect tan), 1 / tan)
    float eye[3], s[3], u[3], f[3];
    float px_scale, py_scale, znear, zfar;
};

__device__ __forceinline__ bool render_project(const RenderView& V, const float* p, float& px, float& py, float& depth) {
    if (V.dim == 2) {
        px = p[0] * V.sx;
        py = float(V.height) - p[1] * V.sy;
        depth = 0.f;
        return true;
    }
    const float d[3] = {p[0] - V.eye[0], p[1] - V.eye[1], p[2] - V.eye[2]};
    const float xv = V.s[0] * d[0] + V.s[1] * d[1] + V.s[2] * d[2];
    const float yv = V.u[0] * d[0] + V.u[1] * d[1] + V.u[2] * d[2];
    const float w = V.f[0] * d[0] + V.f[1] * d[1] + V.f[2] * d[2];  // distance along the view axis
    if (!(w >= V.znear && w <= V.zfar)) return false;
    const float nx = V.px_scale * xv / w, ny = V.py_scale * yv / w;
    px = (nx + 1.f) * 0.5f * float(V.width);
    py = float(V.height) - (ny + 1.f) * 0.5f * float(V.height);
    depth = w;
    return true;
}

__device__ __forceinline__ void render_splat(const RenderView& V, unsigned long long* __restrict__ fb, float px, float py,
                                             float depth, float radius, int intensity, bool smooth) {
    const int x0 = max(0, int(floorf(px - radius - 0.5f))), x1 = min(V.width - 1, int(floorf(px + radius + 0.5f)));
    const int y0 = max(0, int(floorf(py - radius - 0.5f))), y1 = min(V.height - 1, int(floorf(py + radius + 0.5f)));
    const unsigned long long dbits = (unsigned long long)__float_as_uint(fmaxf(depth, 0.f)) << 32;
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
            const float dx = float(x) + 0.5f - px, dy = float(y) + 0.5f - py;
            const float cover = smooth ? fminf(fmaxf(radius + 0.5f - sqrtf(dx * dx + dy * dy), 0.f), 1.f)
                                       : (dx * dx + dy * dy <= radius * radius ? 1.f : 0.f);
            const int level = __float2int_rn(cover * float(intensity));
            if (level > 0) atomicMin(&fb[(long long)y * V.width + x], dbits | (unsigned long long)(255 - level));
        }
}

__global__ void k_render_clear(unsigned long long* __restrict__ fb, long long pixels) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < pixels) fb[i] = ~0ull;
}

// Particles (slot order does not matter: the atomics commute).
__global__ void k_render_points(RenderView V, const float* __restrict__ x, int n, unsigned long long* __restrict__ fb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p[3] = {x[i], x[n + i], V.dim == 3 ? x[2 * n + i] : 0.f};
    float px, py, depth;
    if (!render_project(V, p, px, py, depth) || !isfinite(px) || !isfinite(py)) return;
    render_splat(V, fb, px, py, depth, V.radius, 255, true);
}

// Border lines: segment k from a[k] to b[k] (world), `samples[k]` evenly spaced
// samples, each a 2-pixel-wide gray square.
struct RenderLines {
    float a[12][3], b[12][3];
    int samples[12];
    int count;
};

__global__ void k_render_lines(RenderView V, RenderLines L, unsigned long long* __restrict__ fb) {
    const int k = blockIdx.x;
    if (k >= L.count) return;
    const int m = L.samples[k];
    for (int i = threadIdx.x; i <= m; i += blockDim.x) {
        const float t = m > 0 ? float(i) / float(m) : 0.f;
        float p[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) p[c] = L.a[k][c] + t * (L.b[k][c] - L.a[k][c]);
        float px, py, depth;
        if (!render_project(V, p, px, py, depth)) continue;
        render_splat(V, fb, px, py, depth, 1.f, 128, false);  // glLineWidth(2), glColor3f(0.5, 0.5, 0.5)
    }
}

__global__ void k_render_pack(const unsigned long long* __restrict__ fb, long long pixels, unsigned char* __restrict__ rgb) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    const unsigned long long v = fb[i];
    const unsigned char c = v == ~0ull ? 0 : (unsigned char)(255 - (int)(v & 0xffull));
    rgb[3 * i] = c;
    rgb[3 * i + 1] = c;
    rgb[3 * i + 2] = c;
}

}  // namespace mpm
