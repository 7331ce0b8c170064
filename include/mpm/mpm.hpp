// mpm.hpp — C++ drop-in for the reference's Solver alias.
//
// The reference selects its solver at compile time (src/main.cpp:23-29):
//     using Solver = GPUSolver;   // or CPUSolver
// and calls Solver(), Step() and GetParticlePositions() (src/gpu/GPUSolver.h:
// 11-16). mpm::BasicSolver<Vec> keeps those three calls over the C ABI in
// mpm.h, with Vec any standard-layout vector of `dim` floats (glm::vec2 /
// glm::vec3 in the reference):
//     using Solver = mpm::BasicSolver<Vec>;
// Where the reference reads its scene from the global SHAPES inside the
// constructor (src/gpu/GPUSolver.cpp:95-159), this constructor takes the
// particle arrays that loop builds. Errors throw std::runtime_error carrying
// the mpm_status text, as the reference throws on shader failures
// (src/gpu/GPUSolver.cpp:39-49).
#ifndef MPM_B200_MPM_HPP
#define MPM_B200_MPM_HPP

#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "mpm.h"

namespace mpm {

inline void check(mpm_status st, const mpm_solver* s = nullptr) {
    if (st == MPM_OK) return;
    std::string what = mpm_status_string(st);
    if (s) {
        const char* detail = mpm_last_error(s);
        if (detail && *detail) what += std::string(": ") + detail;
    }
    throw std::runtime_error("mpm: " + what);
}

template <typename Vec> class BasicSolver {
    static_assert(std::is_standard_layout<Vec>::value, "Vec must be a plain vector of floats");

public:
    // positions / velocities in grid units (one Vec per particle), volumes per
    // particle, optional masses (default: volume * RHO / 100, src/cpu/Particles.cpp:18).
    BasicSolver(const mpm_params& params, const std::vector<Vec>& positions, const std::vector<Vec>& velocities,
                const std::vector<float>& volumes, const std::vector<float>* masses = nullptr)
        : dim_(params.dim) {
        if (sizeof(Vec) != sizeof(float) * static_cast<size_t>(params.dim))
            throw std::invalid_argument("mpm: sizeof(Vec) must equal dim floats");
        if (velocities.size() != positions.size() || volumes.size() != positions.size() ||
            (masses && masses->size() != positions.size()))
            throw std::invalid_argument("mpm: particle arrays differ in length");
        mpm_particles_init init{};
        init.count = static_cast<int64_t>(positions.size());
        init.position = reinterpret_cast<const float*>(positions.data());
        init.velocity = reinterpret_cast<const float*>(velocities.data());
        init.volume = volumes.data();
        init.mass = masses ? masses->data() : nullptr;
        check(mpm_create(&params, &init, &solver_));
        cached_.resize(positions.size());
    }
    ~BasicSolver() {
        if (solver_) mpm_destroy(solver_);
    }
    BasicSolver(const BasicSolver&) = delete;
    BasicSolver& operator=(const BasicSolver&) = delete;

    // One time step (asynchronous on the solver's stream), GPUSolver::Step.
    void Step(int nsteps = 1) { check(mpm_step(solver_, nsteps), solver_); }

    // Synchronises and returns the positions in creation order,
    // GPUSolver::GetParticlePositions.
    const std::vector<Vec>& GetParticlePositions() {
        check(mpm_get_positions(solver_, reinterpret_cast<float*>(cached_.data()), cached_.size() * dim_), solver_);
        return cached_;
    }

    mpm_solver* handle() { return solver_; }

private:
    int dim_;
    mpm_solver* solver_ = nullptr;
    std::vector<Vec> cached_;
};

}  // namespace mpm

#endif  // MPM_B200_MPM_HPP
