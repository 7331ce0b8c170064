// Test infrastructure: a headless driver for the reference's own CPU MPM path.
//
// Links src/cpu/Grid.cpp and src/cpu/Particles.cpp, compiled unmodified from the
// reference tree (see oracle/build_oracle.py), against the shadow Parameters.h
// and the Eigen/Dense stand-in under oracle/refcpu/shadow. It mirrors what
// CPUSolver (src/cpu/CPUSolver.h:12-16) does: build a Grid(WIDTH, HEIGHT,
// BORDER_MARGIN) and a Particles(grid), then call Particles::Solver() once per
// step. Particles come from an input file instead of SHAPES (which is empty):
// each is created with the public Particle(pos, vel, vol) constructor
// (src/cpu/Particles.cpp:7-19), so mass = vol * RHO / 100 exactly as there.
//
// Usage: refcpu_driver IN OUT [--replicas R] [--timeout S]
//   IN  : binary scene (see read_scene)
//   OUT : binary dumps of (step, pos, vel, B_p, F_E, F_P) every `dump_every`
//         steps and after the last step; matrices row-major, float32.
// With --replicas R > 1 the same scene is stepped by R independent solvers on
// R threads (aggregate throughput of the single-threaded reference) and only
// replica 0 is dumped. Prints one JSON line with the step-loop wall time.
//
// The reference spins forever on a NaN stress (src/cpu/Particles.cpp:50-61);
// an alarm() bounds every run and exits with status 3 instead.
#include <chrono>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>
#include <unistd.h>

#include "Parameters.h"
#include "Grid.h"
#include "Particles.h"

// Definitions of the knobs that the shadow Parameters.h declares.
int WIDTH = 200, HEIGHT = 100, BORDER_MARGIN = 2;
int NUM_PARTICLES = 3000;
std::vector<SHAPE*> SHAPES;
int MAX_FRAMES = 200;
float GRAVITY = -9.81f, FRICTION = 0.3f;
float DELTA_TIME = 1e-3f, SAVE_FPS = 30.f;
float PARTICLE_SIZE = 1.f, THETA_C = 2.0e-2f, THETA_S = 6.0e-3f, XI = 10.f, NU = 2.0e-1f, E = 1.4e5f,
      RHO = 400.f;
float MU = 0.f, LAMBDA = 0.f;

namespace {

struct Scene {
    int32_t nsteps = 0, dump_every = 0;
    int64_t n = 0;
    std::vector<float> pos, vel, vol;
};

[[noreturn]] void die(const char* msg) {
    std::fprintf(stderr, "refcpu_driver: %s\n", msg);
    std::exit(2);
}

template <typename T> void rd(FILE* f, T* p, size_t count) {
    if (count && std::fread(p, sizeof(T), count, f) != count) die("short read");
}

// Layout: "RCPU" | i32 version=1 | i32 W, H, margin, nsteps, dump_every |
//         f32 dt, gravity, friction, theta_c, theta_s, xi, nu, E, rho |
//         i64 n | f32 pos[2n] | f32 vel[2n] | f32 vol[n]
Scene read_scene(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) die("cannot open input");
    char magic[4];
    rd(f, magic, 4);
    if (std::memcmp(magic, "RCPU", 4) != 0) die("bad magic");
    int32_t ver, ints[5];
    rd(f, &ver, 1);
    if (ver != 1) die("bad version");
    rd(f, ints, 5);
    float fl[9];
    rd(f, fl, 9);
    Scene s;
    WIDTH = ints[0];
    HEIGHT = ints[1];
    BORDER_MARGIN = ints[2];
    s.nsteps = ints[3];
    s.dump_every = ints[4];
    DELTA_TIME = fl[0];
    GRAVITY = fl[1];
    FRICTION = fl[2];
    THETA_C = fl[3];
    THETA_S = fl[4];
    XI = fl[5];
    NU = fl[6];
    E = fl[7];
    RHO = fl[8];
    // Same float expressions as src/shared/Parameters.h:82-84.
    MU = E / (2.f * (1.f + NU));
    LAMBDA = (E * NU) / ((1.f + NU) * (1.f - (2.f * NU)));
    rd(f, &s.n, 1);
    if (s.n < 0 || s.n > (int64_t(1) << 31)) die("bad particle count");
    s.pos.resize(2 * s.n);
    s.vel.resize(2 * s.n);
    s.vol.resize(s.n);
    rd(f, s.pos.data(), s.pos.size());
    rd(f, s.vel.data(), s.vel.size());
    rd(f, s.vol.data(), s.vol.size());
    std::fclose(f);
    return s;
}

struct Replica {
    Grid grid;
    Particles particles;
    explicit Replica(const Scene& s) : grid(WIDTH, HEIGHT, BORDER_MARGIN), particles(grid) {
        auto& ps = particles.GetParticles();
        ps.reserve(s.n);
        for (int64_t i = 0; i < s.n; ++i)
            ps.emplace_back(glm::vec2(s.pos[2 * i], s.pos[2 * i + 1]), glm::vec2(s.vel[2 * i], s.vel[2 * i + 1]),
                            s.vol[i]);
    }
};

void dump(FILE* f, int32_t step, Particles& particles) {
    auto& ps = particles.GetParticles();
    const int64_t n = (int64_t)ps.size();
    std::vector<float> buf;
    buf.reserve(n * 16);
    std::fwrite(&step, sizeof(step), 1, f);
    // glm matrices are column-major: m[col][row]; written row-major.
    auto put_mat = [&](const glm::mat2& m) {
        buf.push_back(m[0][0]);
        buf.push_back(m[1][0]);
        buf.push_back(m[0][1]);
        buf.push_back(m[1][1]);
    };
    buf.clear();
    for (auto& p : ps) { buf.push_back(p.GetPosition().x); buf.push_back(p.GetPosition().y); }
    for (auto& p : ps) { buf.push_back(p.GetVelocity().x); buf.push_back(p.GetVelocity().y); }
    for (auto& p : ps) put_mat(p.GetBp());
    for (auto& p : ps) put_mat(p.GetElasticForce());
    for (auto& p : ps) put_mat(p.GetPlasticForce());
    std::fwrite(buf.data(), sizeof(float), buf.size(), f);
}

void on_alarm(int) {
    const char msg[] = "refcpu_driver: timeout (the reference spins on a NaN stress)\n";
    ssize_t r = write(2, msg, sizeof(msg) - 1);
    (void)r;
    _exit(3);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) die("usage: refcpu_driver IN OUT [--replicas R] [--timeout S]");
    int replicas = 1;
    int timeout_s = 600;
    for (int i = 3; i + 1 < argc; i += 2) {
        if (!std::strcmp(argv[i], "--replicas")) replicas = std::atoi(argv[i + 1]);
        else if (!std::strcmp(argv[i], "--timeout")) timeout_s = std::atoi(argv[i + 1]);
        else die("unknown option");
    }
    if (replicas < 1) replicas = 1;
    std::signal(SIGALRM, on_alarm);
    alarm((unsigned)timeout_s);

    Scene scene = read_scene(argv[1]);
    std::vector<std::unique_ptr<Replica>> reps;
    for (int r = 0; r < replicas; ++r) reps.emplace_back(new Replica(scene));

    FILE* out = std::fopen(argv[2], "wb");
    if (!out) die("cannot open output");

    double loop_seconds = 0.0;
    if (replicas == 1) {
        Replica& rep = *reps[0];
        for (int32_t s = 1; s <= scene.nsteps; ++s) {
            auto t0 = std::chrono::steady_clock::now();
            rep.particles.Solver();
            loop_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if ((scene.dump_every > 0 && s % scene.dump_every == 0) || s == scene.nsteps)
                dump(out, s, rep.particles);
        }
        if (scene.nsteps == 0) dump(out, 0, rep.particles);
    } else {
        auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> th;
        for (int r = 0; r < replicas; ++r)
            th.emplace_back([&, r] {
                for (int32_t s = 0; s < scene.nsteps; ++s) reps[r]->particles.Solver();
            });
        for (auto& t : th) t.join();
        loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        dump(out, scene.nsteps, reps[0]->particles);
    }
    std::fclose(out);
    std::printf("{\"particles\": %lld, \"steps\": %d, \"replicas\": %d, \"loop_seconds\": %.6f}\n",
                (long long)scene.n, scene.nsteps, replicas, loop_seconds);
    return 0;
}
