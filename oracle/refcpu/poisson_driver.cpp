// TEST INFRASTRUCTURE — runs the reference's own Poisson-disk samplers
// (PoissonDiskCircle / PoissonDiskSphere, src/shared/Shapes.h, included where
// it lies in the reference tree) on one snowball and prints the sample count
// and the smallest pairwise distance as JSON. Built by oracle/build_oracle.py
// into the git-ignored oracle/_ref/; 2D without SIM_3D, 3D with it.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "Shapes.h"

int main(int argc, char** argv) {
#ifdef SIM_3D
    if (argc < 6) { std::fprintf(stderr, "usage: cx cy cz radius min_dist\n"); return 2; }
    const glm::vec3 c((float)std::atof(argv[1]), (float)std::atof(argv[2]), (float)std::atof(argv[3]));
    const float r = (float)std::atof(argv[4]), md = (float)std::atof(argv[5]);
    const auto s = PoissonDiskSphere(c, r, md);
#else
    if (argc < 5) { std::fprintf(stderr, "usage: cx cy radius min_dist\n"); return 2; }
    const glm::vec2 c((float)std::atof(argv[1]), (float)std::atof(argv[2]));
    const float r = (float)std::atof(argv[3]), md = (float)std::atof(argv[4]);
    const auto s = PoissonDiskCircle(c, r, md);
#endif
    double mind = 1e30;
    for (size_t i = 0; i < s.size(); ++i)
        for (size_t j = i + 1; j < s.size(); ++j) mind = std::fmin(mind, (double)glm::length(s[i] - s[j]));
    std::printf("{\"count\": %zu, \"min_dist\": %.9g}\n", s.size(), mind);
    return 0;
}
