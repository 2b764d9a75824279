// Host-side mesh import (reference layout -> solver layout) and geometry.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

struct mc_mesh_view;

namespace mcb {

struct HostPhysics {
    double density;
};

// Solver-side mesh on the host before upload (see mc_internal.h for layout).
struct HostMesh {
    int N = 0, F = 0;
    int btype[6];
    int last_bface[6];
    std::vector<int> fc0, fc1, nbr, sface, col, outlet_faces;
    std::vector<double> area, lam, rl, S, xf, xc, vol, rho;  // S, xf, xc: [.][3]
};

int build_host_mesh(const mc_mesh_view *mv, const HostPhysics &hp, HostMesh &hm, std::string &err);
double inlet_effective_viscosity(double mu, double u_in);

} // namespace mcb
