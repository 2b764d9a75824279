// Device side of the flow/particle exchange: particle rows summed into their
// cells (the flow side of update_flow_field, FlowSolver.inl:496-736) and the
// flow state interpolated to mesh nodes (get_neighbour_cells and
// interpolate_to_nodes, :293-494).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace mcb {

// Keys (cell << 32 | row) of n rows, padded with UINT64_MAX to n2 (a power of
// two, at least 2048), then sorted ascending in place: the rows of a cell end
// up together and in arrival order.
void particle_keys(cudaStream_t s, int n, int n2, const int *cells, uint64_t *keys);
void sort_keys(cudaStream_t s, uint64_t *keys, int n2);
// src[k][o2n[cell]] = the sum, in arrival order, of the cell's rows [n][5]
// (src must be zero; o2n null: identity).
void particle_sums(cudaStream_t s, int n, const uint64_t *keys, const double *rows, const int *o2n, int N,
                   double *src);

struct NodeArgs {
    const double *U, *V, *W, *P, *T;          // fields, handle order
    const double *gU[3], *gV[3], *gW[3], *gP[3], *gT[3];
    const double *xc, *yc, *zc;               // cell centres, handle order
    const double *px, *py, *pz;               // node coordinates
    const int *pc_off, *pc_cells;             // node -> its cells (handle ids, ascending caller id)
    double u_ref, p_ref, t_ref;               // reference gas state
};

// Distinct nodes of the requested cells (caller ids) in ascending node id:
// flag[P] must be zero on entry and is left zero; block_counts needs
// ceil(P / 1024) + 1 ints; count receives the number of nodes.
void mark_nodes(cudaStream_t s, int n_req, const int *req, const int *cell_nodes, unsigned char *flag);
void compact_nodes(cudaStream_t s, int P, unsigned char *flag, int *block_counts, int *nodes, int *count);
// out[i][5] = {vel.x, vel.y, vel.z, pressure, temp} at nodes[i].
void node_values(cudaStream_t s, int n, const int *nodes, const NodeArgs &a, double *out);

} // namespace mcb
