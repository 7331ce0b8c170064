// Test infrastructure (oracle build only): stand-in for src/shared/helpers.h.
//
// src/cpu/Particles.cpp:4 includes "helpers.h", which in the reference tree sits
// next to the real Parameters.h and would pull it in; this copy of the three
// helpers is found first on the include path instead, so that the shadow
// Parameters.h is used. Same names, signatures and semantics as
// src/shared/helpers.h:8-32:
//   VectorOuterProduct(v, d) = v d^T (glm column-major, so col j = v * d[j]);
//   GLMToEigen / EigenToGLM   = transpose of storage order between glm (m[col][row])
//                               and Eigen (m(row, col)).
#pragma once

#include "Parameters.h"

#include <glm/glm.hpp>
#include <Eigen/Dense>

inline glm::mat2 VectorOuterProduct(glm::vec2 v, glm::vec2 d) {
    glm::mat2 r;
    for (int col = 0; col < 2; ++col)
        for (int row = 0; row < 2; ++row) r[col][row] = v[row] * d[col];
    return r;
}

inline Eigen::Matrix2f GLMToEigen(glm::mat2 a) {
    Eigen::Matrix2f r;
    for (int row = 0; row < 2; ++row)
        for (int col = 0; col < 2; ++col) r(row, col) = a[col][row];
    return r;
}

inline glm::mat2 EigenToGLM(Eigen::Matrix2f a) {
    glm::mat2 r;
    for (int row = 0; row < 2; ++row)
        for (int col = 0; col < 2; ++col) r[col][row] = a(row, col);
    return r;
}
