// Test infrastructure (oracle build only): shadow of src/shared/Parameters.h.
//
// The reference keeps every knob as a compile-time `static const` in
// src/shared/Parameters.h:6-84 and the scene in the global `SHAPES`
// (:49-52). To drive src/cpu/Grid.cpp and src/cpu/Particles.cpp unmodified on
// seeded scenes, this header is found first on the include path and turns the
// knobs into runtime globals with the same names and types. The arithmetic the
// reference performs on them is unchanged (float operands, same expressions);
// the values are set by refcpu_driver.cpp before any step. SHAPES is empty:
// particles are injected through Particles::GetParticles().
#pragma once

#include <vector>
#include "Shapes.h"

using Vec = glm::vec2;
using Mat = glm::mat2;
using VecGPU = glm::vec2;
using MatGPU = glm::mat2;
static constexpr int DIM = 2;

extern int WIDTH, HEIGHT, BORDER_MARGIN;
extern int NUM_PARTICLES;
extern std::vector<SHAPE*> SHAPES;
extern int MAX_FRAMES;
extern float GRAVITY, FRICTION;
extern float DELTA_TIME, SAVE_FPS;
extern float PARTICLE_SIZE, THETA_C, THETA_S, XI, NU, E, RHO;
extern float MU, LAMBDA;
