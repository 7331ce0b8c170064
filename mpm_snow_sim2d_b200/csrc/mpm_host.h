// Host-side set-up shared by the single-scene solver and the batched scenes:
// parameter validation, per-scene step constants, fixed-point scales.
#pragma once

#include <cmath>
#include <string>

#include "mpm/mpm.h"
#include "mpm_kernels.cuh"

namespace mpm {

inline mpm_status validate_params(const mpm_params* p, std::string& why) {
    if (!p) { why = "params is NULL"; return MPM_ERR_INVALID_ARGUMENT; }
    if (p->dim != 2 && p->dim != 3) { why = "dim must be 2 or 3"; return MPM_ERR_INVALID_ARGUMENT; }
    if (p->width < 1 || p->height < 1 || (p->dim == 3 && p->depth < 1)) { why = "grid extent must be >= 1 cell"; return MPM_ERR_INVALID_ARGUMENT; }
    const double nodes = double(p->width + 1) * (p->height + 1) * (p->dim == 3 ? p->depth + 1 : 1);
    if (nodes > 2.0e9) { why = "grid too large"; return MPM_ERR_INVALID_ARGUMENT; }
    if (p->dim == 3 && (p->width > 2000000 || p->height > 2000000 || p->depth > 2000000)) {
        why = "3D grid extents are limited to 2,000,000 cells per axis";  // 21-bit stencil keys in P2G
        return MPM_ERR_INVALID_ARGUMENT;
    }
    if (!(p->delta_time > 0.f) || !std::isfinite(p->delta_time)) { why = "delta_time must be > 0"; return MPM_ERR_INVALID_ARGUMENT; }
    if (p->formulation != MPM_FORMULATION_MLS && p->formulation != MPM_FORMULATION_CLASSIC &&
        p->formulation != MPM_FORMULATION_MLS_QUADRATIC) { why = "unknown formulation"; return MPM_ERR_INVALID_ARGUMENT; }
    if (p->formulation == MPM_FORMULATION_CLASSIC && p->dim != 2) { why = "the CLASSIC (reference CPU) formulation is 2D only"; return MPM_ERR_UNSUPPORTED; }
    if (p->boundary != MPM_BOUNDARY_FRICTION && p->boundary != MPM_BOUNDARY_STICKY) { why = "unknown boundary"; return MPM_ERR_INVALID_ARGUMENT; }
    if (p->border_margin < 0) { why = "border_margin must be >= 0"; return MPM_ERR_INVALID_ARGUMENT; }
    if (!(p->nu > -1.f && p->nu < 0.5f)) { why = "nu must be in (-1, 0.5)"; return MPM_ERR_INVALID_ARGUMENT; }
    return MPM_OK;
}

// Grid extents and material constants of one scene (scales left unset).
inline StepConsts step_consts(const mpm_params& p, int dim) {
    StepConsts C{};
    C.W = p.width; C.H = p.height; C.Dp = dim == 3 ? p.depth : 0;
    C.nx = p.width + 1; C.ny = p.height + 1; C.nz = dim == 3 ? p.depth + 1 : 1;
    C.nodes = (long long)C.nx * C.ny * C.nz;
    C.dt = p.delta_time; C.gravity = p.gravity; C.friction = p.friction;
    C.theta_c = p.theta_c; C.theta_s = p.theta_s; C.xi = p.xi;
    // Lame parameters as in src/shared/Parameters.h:82-84, evaluated in double.
    const double E = p.youngs, nu = p.nu;
    C.mu0 = (float)(E / (2.0 * (1.0 + nu)));
    C.la0 = (float)((E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu)));
    C.margin = (float)p.border_margin;
    C.boundary = p.boundary;
    return C;
}

// Power-of-two fixed-point scales: no node sum can exceed 2^62 for a total
// mass `total_mass` and node speeds up to v_cap = 16 cells per step (faster
// nodes raise MPM_FLAG_OVERFLOW). log2 of the mass, momentum, force scales
// into l2[0..2].
inline void fixed_point_scales(const mpm_params& p, double total_mass, StepConsts& C, int* l2) {
    const double v_cap = 16.0 / p.delta_time;
    const double mt = total_mass > 0 ? total_mass * 1.125 : 1.0;
    int lm = (int)std::floor(62.0 - std::log2(mt));
    int lp = (int)std::floor(62.0 - std::log2(mt * v_cap));
    lm = lm > 100 ? 100 : (lm < -100 ? -100 : lm);
    lp = lp > 100 ? 100 : (lp < -100 ? -100 : lp);
    if (p.fixed_point_log2_mass != 0) lm = p.fixed_point_log2_mass;
    if (p.fixed_point_log2_momentum != 0) lp = p.fixed_point_log2_momentum;
    const int lf = lp + (int)std::floor(std::log2((double)p.delta_time));
    l2[0] = lm;
    l2[1] = lp;
    l2[2] = lf;
    C.sm = std::ldexp(1.0f, lm);
    C.sp = std::ldexp(1.0f, lp);
    C.sf = std::ldexp(1.0f, lf);
    C.inv_sm = std::ldexp(1.0f, -lm);
    C.inv_sp = std::ldexp(1.0f, -lp);
    C.inv_sf = std::ldexp(1.0f, -lf);
    C.v_cap = (float)v_cap;
}

}  // namespace mpm
