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

// Reverse Cuthill-McKee order of the cells over the internal-face graph
// (cell_n2o[new] = old): each connected component starts from a
// pseudo-peripheral cell of least degree, neighbours are queued by increasing
// degree (ties by id), and the whole order is reversed.
void rcm_cell_order(const HostMesh &hm, std::vector<int> &cell_n2o);

// Renumber the cells by cell_n2o and the faces by first touch when walking
// the renumbered cells, each cell's faces in reference face order
// (face_n2o[new] = old).  Every per-face and per-cell array is permuted; the
// slot orders (cell_faces order for nbr, reference face order for sface and
// col) are unchanged, so every gather sums in the same order as before.
int apply_reorder(HostMesh &hm, const std::vector<int> &cell_n2o, std::vector<int> &face_n2o, std::string &err);
double inlet_effective_viscosity(double mu, double u_in);

} // namespace mcb
