// Node coordinates of the reference Mesh on one rank, shared by the metric
// tables (nova_capi.cu) and the EnSight geometry writer (nova_io.cu).
#pragma once

#include "nova_gpu.h"

#include <cmath>

namespace nova {

// coefficient of the hyperbolic-tangent stretching (src/Mesh/Mesh.cpp:57-61)
inline double mesh_hyp_b(const nova_mesh_desc &m)
{
    double b = 1.0;
    if (m.hyperbolic_z) {
        const int globN = m.N[2] + 1;
        for (int i = 1; i < 10000; i++) b = std::asinh(b / ((globN - 1) * std::pow(m.s1 * m.s2, 0.5)));
    }
    return b;
}

// Mesh::z (src/Mesh/Mesh.cpp:373-407) of the ghosted index k (h ghosts)
inline double mesh_z(const nova_mesh_desc &m, int h, double bcoef, int k)
{
    const double dz = m.L[2] / m.N[2];
    if (m.hyperbolic_z) {
        const double A = std::pow(m.s1 / m.s2, 0.5);
        const int globK = k - h + (int)(long)m.origin[2];
        const int globN = m.N[2] + 1;
        const double R = (double)globK / (double)(globN - 1) - 0.5;
        const double U = 1.0 + std::tanh(bcoef * R) / std::tanh(bcoef / 2.0);
        return U / (2.0 * A + (1 - A) * U) * m.L[2];
    }
    return (k - h) * dz + m.origin[2];
}

}  // namespace nova
