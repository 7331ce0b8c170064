// TEST INFRASTRUCTURE — the reference's GPU step executed on the CPU.
//
// Only the oracle build and tests/ use this file. It compiles the reference's
// own GLSL compute shaders (src/gpu/shaders/{2d,3d}/{reset,p2g,grid_update,
// g2p}.glsl with their common.glsl), turned into C++ fragments by
// oracle/shader/glsl_cpp.py, against the reference's vendored glm 0.9.7.1, and
// runs them the way src/gpu/GPUSolver.cpp:63-80 dispatches them: one
// invocation per particle (p2g, g2p) or per node (grid_update, reset), the four
// passes in that order every step, uniforms set as GPUSolver::DispatchParticles
// / DispatchGrid set them (:227-274). Invocations run one at a time in index
// order, so the shaders' float atomicAdd (GL_NV_shader_atomic_float) is a plain
// add in particle order — one of the orders the GPU may use. Arithmetic is FP32
// as in GLSL (the fragments are compiled with -fsingle-precision-constant so
// that unsuffixed literals are single precision, as GLSL reads them); the
// transcendental functions come from the host's libm, where the GPU's would
// use its own approximations.
//
// The C ABI (sr_*) takes row-major per-particle arrays as the oracle's:
// x[n][d], v[n][d], B[n][d][d], F_E[n][d][d], F_P[n][d][d] (B[r][c] = B_rc);
// glm matrices are column-major (m[c][r]).
#include <cstdint>
#include <cstring>
#include <vector>

#include <glm/glm.hpp>

namespace glsl_rt {
// GLSL atomicAdd on a float buffer element; invocations run one at a time here.
inline float atomicAdd(float& mem, float v) {
    const float old = mem;
    mem += v;
    return old;
}
}  // namespace glsl_rt

#define GLSL_PRELUDE         \
    using namespace glm;     \
    using glsl_rt::atomicAdd; \
    static glm::uvec3 gl_GlobalInvocationID;

// clang-format off
namespace s2_reset { GLSL_PRELUDE
#include "2d_reset.inc"
}
namespace s2_p2g { GLSL_PRELUDE
#include "2d_p2g.inc"
}
namespace s2_grid { GLSL_PRELUDE
#include "2d_grid_update.inc"
}
namespace s2_g2p { GLSL_PRELUDE
#include "2d_g2p.inc"
}
namespace s3_reset { GLSL_PRELUDE
#include "3d_reset.inc"
}
namespace s3_p2g { GLSL_PRELUDE
#include "3d_p2g.inc"
}
namespace s3_grid { GLSL_PRELUDE
#include "3d_grid_update.inc"
}
namespace s3_g2p { GLSL_PRELUDE
#include "3d_g2p.inc"
}
// clang-format on

extern "C" {
typedef struct {
    int32_t dim, width, height, depth;
    float border_margin, delta_time, gravity, friction, theta_c, theta_s, xi, mu, lambda;
} sr_params;
}

namespace {

template <typename M, int D> M to_glm(const float* a) {  // row-major D x D -> glm
    M m(0.f);
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) m[c][r] = a[r * D + c];
    return m;
}
template <typename M, int D> void from_glm(const M& m, float* a) {
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) a[r * D + c] = m[c][r];
}

// Uniforms of one shader namespace (the ones it declares).
#define SET_GRID_UNIFORMS(ns, p)            \
    ns::gWidth = (p).width;                 \
    ns::gHeight = (p).height

void run2(const sr_params& p, int64_t n, float* x, float* v, float* B, float* Fe, float* Fp, const float* mass,
          const float* vol, int nsteps) {
    using glm::mat2;
    using glm::vec2;
    const int64_t nodes = int64_t(p.width + 1) * (p.height + 1);
    std::vector<vec2> pos(n), vel(n), gcol(nodes), gfric(nodes);
    std::vector<mat2> fe(n), fp(n), bp(n);
    std::vector<float> ms(mass, mass + n), vo(vol, vol + n), gm(nodes, 0.f), gx(nodes, 0.f), gy(nodes, 0.f);
    for (int64_t i = 0; i < n; ++i) {
        pos[i] = vec2(x[2 * i], x[2 * i + 1]);
        vel[i] = vec2(v[2 * i], v[2 * i + 1]);
        bp[i] = to_glm<mat2, 2>(B + 4 * i);
        fe[i] = to_glm<mat2, 2>(Fe + 4 * i);
        fp[i] = to_glm<mat2, 2>(Fp + 4 * i);
    }
    // buffers (bindings as in GPUSolver::InitBuffers)
    s2_p2g::pos = pos.data(); s2_p2g::vel = vel.data(); s2_p2g::mass = ms.data(); s2_p2g::vol = vo.data();
    s2_p2g::fe = fe.data(); s2_p2g::fp = fp.data(); s2_p2g::bp = bp.data();
    s2_p2g::gMass = gm.data(); s2_p2g::gVelX = gx.data(); s2_p2g::gVelY = gy.data();
    s2_grid::gMass = gm.data(); s2_grid::gVelX = gx.data(); s2_grid::gVelY = gy.data();
    s2_grid::gVelCol = gcol.data(); s2_grid::gVelFric = gfric.data();
    s2_g2p::pos = pos.data(); s2_g2p::vel = vel.data(); s2_g2p::fe = fe.data(); s2_g2p::fp = fp.data();
    s2_g2p::bp = bp.data(); s2_g2p::gVelCol = gcol.data(); s2_g2p::gVelFric = gfric.data();
    s2_reset::gMass = gm.data(); s2_reset::gVelX = gx.data(); s2_reset::gVelY = gy.data();
    s2_reset::gVelCol = gcol.data(); s2_reset::gVelFric = gfric.data();
    // uniforms
    s2_p2g::numParticles = int(n); SET_GRID_UNIFORMS(s2_p2g, p);
    s2_p2g::XI = p.xi; s2_p2g::MU = p.mu; s2_p2g::LAMBDA = p.lambda; s2_p2g::DELTA_TIME = p.delta_time;
    SET_GRID_UNIFORMS(s2_grid, p);
    s2_grid::borderMargin = p.border_margin; s2_grid::DELTA_TIME = p.delta_time;
    s2_grid::GRAVITY = p.gravity; s2_grid::FRICTION = p.friction;
    s2_g2p::numParticles = int(n); SET_GRID_UNIFORMS(s2_g2p, p);
    s2_g2p::DELTA_TIME = p.delta_time; s2_g2p::THETA_C = p.theta_c; s2_g2p::THETA_S = p.theta_s;
    SET_GRID_UNIFORMS(s2_reset, p);
    for (int st = 0; st < nsteps; ++st) {
        for (int64_t i = 0; i < n; ++i) { s2_p2g::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s2_p2g::shader_main(); }
        for (int64_t i = 0; i < nodes; ++i) { s2_grid::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s2_grid::shader_main(); }
        for (int64_t i = 0; i < n; ++i) { s2_g2p::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s2_g2p::shader_main(); }
        for (int64_t i = 0; i < nodes; ++i) { s2_reset::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s2_reset::shader_main(); }
    }
    for (int64_t i = 0; i < n; ++i) {
        x[2 * i] = pos[i].x; x[2 * i + 1] = pos[i].y;
        v[2 * i] = vel[i].x; v[2 * i + 1] = vel[i].y;
        from_glm<mat2, 2>(bp[i], B + 4 * i);
        from_glm<mat2, 2>(fe[i], Fe + 4 * i);
        from_glm<mat2, 2>(fp[i], Fp + 4 * i);
    }
}

void run3(const sr_params& p, int64_t n, float* x, float* v, float* B, float* Fe, float* Fp, const float* mass,
          const float* vol, int nsteps) {
    using glm::mat3;
    using glm::mat4;
    using glm::vec4;
    const int64_t nodes = int64_t(p.width + 1) * (p.height + 1) * (p.depth + 1);
    std::vector<vec4> pos(n), vel(n), gcol(nodes, vec4(0.f)), gfric(nodes, vec4(0.f));
    std::vector<mat4> fe(n), fp(n), bp(n);
    std::vector<float> ms(mass, mass + n), vo(vol, vol + n), gm(nodes, 0.f), gx(nodes, 0.f), gy(nodes, 0.f),
        gz(nodes, 0.f);
    for (int64_t i = 0; i < n; ++i) {
        pos[i] = vec4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.f);
        vel[i] = vec4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.f);
        bp[i] = mat4(to_glm<mat3, 3>(B + 9 * i));
        fe[i] = mat4(to_glm<mat3, 3>(Fe + 9 * i));
        fp[i] = mat4(to_glm<mat3, 3>(Fp + 9 * i));
    }
    s3_p2g::pos = pos.data(); s3_p2g::vel = vel.data(); s3_p2g::mass = ms.data(); s3_p2g::vol = vo.data();
    s3_p2g::fe = fe.data(); s3_p2g::fp = fp.data(); s3_p2g::bp = bp.data();
    s3_p2g::gMass = gm.data(); s3_p2g::gVelX = gx.data(); s3_p2g::gVelY = gy.data(); s3_p2g::gVelZ = gz.data();
    s3_grid::gMass = gm.data(); s3_grid::gVelX = gx.data(); s3_grid::gVelY = gy.data(); s3_grid::gVelZ = gz.data();
    s3_grid::gVelCol = gcol.data(); s3_grid::gVelFric = gfric.data();
    s3_g2p::pos = pos.data(); s3_g2p::vel = vel.data(); s3_g2p::fe = fe.data(); s3_g2p::fp = fp.data();
    s3_g2p::bp = bp.data(); s3_g2p::gVelCol = gcol.data(); s3_g2p::gVelFric = gfric.data();
    s3_reset::gMass = gm.data(); s3_reset::gVelX = gx.data(); s3_reset::gVelY = gy.data(); s3_reset::gVelZ = gz.data();
    s3_reset::gVelCol = gcol.data(); s3_reset::gVelFric = gfric.data();
    s3_p2g::numParticles = int(n); SET_GRID_UNIFORMS(s3_p2g, p); s3_p2g::gDepth = p.depth;
    s3_p2g::XI = p.xi; s3_p2g::MU = p.mu; s3_p2g::LAMBDA = p.lambda; s3_p2g::DELTA_TIME = p.delta_time;
    SET_GRID_UNIFORMS(s3_grid, p); s3_grid::gDepth = p.depth;
    s3_grid::borderMargin = p.border_margin; s3_grid::DELTA_TIME = p.delta_time;
    s3_grid::GRAVITY = p.gravity; s3_grid::FRICTION = p.friction;
    s3_g2p::numParticles = int(n); SET_GRID_UNIFORMS(s3_g2p, p); s3_g2p::gDepth = p.depth;
    s3_g2p::DELTA_TIME = p.delta_time; s3_g2p::THETA_C = p.theta_c; s3_g2p::THETA_S = p.theta_s;
    SET_GRID_UNIFORMS(s3_reset, p); s3_reset::gDepth = p.depth;
    for (int st = 0; st < nsteps; ++st) {
        for (int64_t i = 0; i < n; ++i) { s3_p2g::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s3_p2g::shader_main(); }
        for (int64_t i = 0; i < nodes; ++i) { s3_grid::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s3_grid::shader_main(); }
        for (int64_t i = 0; i < n; ++i) { s3_g2p::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s3_g2p::shader_main(); }
        for (int64_t i = 0; i < nodes; ++i) { s3_reset::gl_GlobalInvocationID = glm::uvec3(unsigned(i), 0u, 0u); s3_reset::shader_main(); }
    }
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) { x[3 * i + k] = pos[i][k]; v[3 * i + k] = vel[i][k]; }
        from_glm<mat3, 3>(mat3(bp[i]), B + 9 * i);
        from_glm<mat3, 3>(mat3(fe[i]), Fe + 9 * i);
        from_glm<mat3, 3>(mat3(fp[i]), Fp + 9 * i);
    }
}

}  // namespace

extern "C" {

// nsteps of the reference's shader pipeline on the given state (in place).
int sr_run(const sr_params* p, int64_t n, float* x, float* v, float* B, float* Fe, float* Fp, const float* mass,
           const float* vol, int32_t nsteps) {
    if (!p || n < 0 || nsteps < 0 || (p->dim != 2 && p->dim != 3)) return 1;
    if (p->dim == 2) run2(*p, n, x, v, B, Fe, Fp, mass, vol, nsteps);
    else run3(*p, n, x, v, B, Fe, Fp, mass, vol, nsteps);
    return 0;
}

// The shaders' own svd (2d/common.glsl:2-37, 3d/common.glsl:57-105) on a
// row-major matrix; U, V row-major, S the singular values (last one carries the
// reflection sign).
void sr_svd(int32_t dim, const float* M, float* U, float* S, float* V) {
    if (dim == 2) {
        glm::mat2 u, vv;
        glm::vec2 sg;
        s2_p2g::svd(to_glm<glm::mat2, 2>(M), u, sg, vv);
        from_glm<glm::mat2, 2>(u, U);
        from_glm<glm::mat2, 2>(vv, V);
        S[0] = sg.x; S[1] = sg.y;
    } else {
        glm::mat3 u, vv;
        glm::vec3 sg;
        s3_p2g::svd(to_glm<glm::mat3, 3>(M), u, sg, vv);
        from_glm<glm::mat3, 3>(u, U);
        from_glm<glm::mat3, 3>(vv, V);
        S[0] = sg.x; S[1] = sg.y; S[2] = sg.z;
    }
}

// The shaders' cubic B-spline N and N_grad (3d/common.glsl:111-137; the 2D
// file holds the same text).
void sr_bspline(int32_t dim, float x, float* n, float* dn) {
    if (dim == 2) { *n = s2_p2g::N(x); *dn = s2_p2g::N_grad(x); }
    else { *n = s3_p2g::N(x); *dn = s3_p2g::N_grad(x); }
}

// The shaders' wall response of one node (2d/grid_update.glsl:17-80,
// 3d/grid_update.glsl:19-86).
void sr_collide(const sr_params* p, const float* loc, const float* vel, float* vcol, float* vfric) {
    if (p->dim == 2) {
        SET_GRID_UNIFORMS(s2_grid, *p);
        s2_grid::borderMargin = p->border_margin; s2_grid::DELTA_TIME = p->delta_time;
        s2_grid::GRAVITY = p->gravity; s2_grid::FRICTION = p->friction;
        glm::vec2 vc, vf;
        s2_grid::detectCollisions(glm::vec2(loc[0], loc[1]), glm::vec2(vel[0], vel[1]), vc, vf);
        vcol[0] = vc.x; vcol[1] = vc.y; vfric[0] = vf.x; vfric[1] = vf.y;
    } else {
        SET_GRID_UNIFORMS(s3_grid, *p); s3_grid::gDepth = p->depth;
        s3_grid::borderMargin = p->border_margin; s3_grid::DELTA_TIME = p->delta_time;
        s3_grid::GRAVITY = p->gravity; s3_grid::FRICTION = p->friction;
        glm::vec3 vc, vf;
        s3_grid::detectCollisions(glm::vec3(loc[0], loc[1], loc[2]), glm::vec3(vel[0], vel[1], vel[2]), vc, vf);
        for (int k = 0; k < 3; ++k) { vcol[k] = vc[k]; vfric[k] = vf[k]; }
    }
}

}  // extern "C"
