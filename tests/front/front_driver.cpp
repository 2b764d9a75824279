// Driver for the reference-side front (include/flow_b200/FlowSolver.inl): the
// flow branch of the reference's src/minicombust.cpp (:142-174 set-up,
// :219-227 main loop) on one flow rank, with the mesh built by the
// reference's own load_mesh (src/examples/mesh_examples.cpp:120).
//
//   front_driver ex ey ez lx ly lz timesteps fields.bin [vtk_prefix]
//
// Writes the 13 fields (phi_vector member order, cells + 6 values each,
// float64) after `timesteps` calls of FlowSolver::timestep() to fields.bin,
// and with vtk_prefix also calls output_data.  Test infrastructure: built
// by oracle/Makefile (target front) against the reference's headers and the
// single-rank MPI shim; run by tests/test_front.py.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mpi.h"
#include "utils/utils.hpp"
#include "geometry/Mesh.hpp"
#include "examples/mesh_examples.hpp"
#include "flow_b200/FlowSolver.inl"

using namespace minicombust::flow;

int main(int argc, char **argv)
{
    if (argc < 9) {
        std::fprintf(stderr, "usage: %s ex ey ez lx ly lz timesteps fields.bin [vtk_prefix]\n", argv[0]);
        return 2;
    }
    MPI_Init(&argc, &argv);
    MPI_Config c;
    std::memset(&c, 0, sizeof(c));
    c.world = MPI_COMM_WORLD;
    MPI_Comm_rank(c.world, &c.rank);
    MPI_Comm_size(c.world, &c.world_size);
    const int flow_ranks = 1;
    c.solver_type = (c.rank >= flow_ranks);
    MPI_Comm_split(c.world, c.solver_type, c.rank, &c.particle_flow_world);
    MPI_Comm_rank(c.particle_flow_world, &c.particle_flow_rank);
    MPI_Comm_size(c.particle_flow_world, &c.particle_flow_world_size);
    MPI_Type_contiguous(sizeof(flow_aos<double>) / sizeof(double), MPI_DOUBLE, &c.MPI_FLOW_STRUCTURE);
    MPI_Type_contiguous(sizeof(vec<double>) / sizeof(double), MPI_DOUBLE, &c.MPI_VEC_STRUCTURE);
    MPI_Type_contiguous(sizeof(particle_aos<double>) / sizeof(double), MPI_DOUBLE, &c.MPI_PARTICLE_STRUCTURE);
    MPI_Type_commit(&c.MPI_FLOW_STRUCTURE);
    MPI_Type_commit(&c.MPI_PARTICLE_STRUCTURE);
    c.one_flow_rank = (int *)calloc(flow_ranks, sizeof(int));
    c.every_one_flow_rank = (int *)calloc(flow_ranks, sizeof(int));
    c.one_flow_world_size = (int *)calloc(flow_ranks, sizeof(int));
    c.every_one_flow_world_size = (int *)calloc(flow_ranks, sizeof(int));
    c.one_flow_world = (MPI_Comm *)calloc(flow_ranks, sizeof(MPI_Comm));
    c.every_one_flow_world = (MPI_Comm *)calloc(flow_ranks, sizeof(MPI_Comm));
    c.alias_rank = (int *)calloc(flow_ranks, sizeof(int));

    vec<uint64_t> elements = {(uint64_t)atoll(argv[1]), (uint64_t)atoll(argv[2]), (uint64_t)atoll(argv[3])};
    vec<double> box = {atof(argv[4]), atof(argv[5]), atof(argv[6])};
    const int timesteps = atoi(argv[7]);
    FILE *log = fopen("/dev/null", "w");
    Mesh<double> *mesh = load_mesh(&c, box, elements, flow_ranks, log);
    int status = 0;
    try {
        FlowSolver<double> flow_solver(&c, mesh, 1.0e-5, log);
        for (int t = 0; t < timesteps; t++) {
            flow_solver.timestep();
            if (argc > 9) flow_solver.output_data(t + 1);
        }
        flow_solver.print_logger_stats(timesteps, 0.0);
        const size_t n = mesh->mesh_size + 6;
        std::vector<double> buf(n);
        FILE *out = fopen(argv[8], "wb");
        if (!out) throw std::runtime_error("cannot open output");
        for (int f = 0; f < 13; f++) {
            flow_solver.get_field(f, buf.data());
            fwrite(buf.data(), sizeof(double), n, out);
        }
        fclose(out);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "front_driver: %s\n", e.what());
        status = 1;
    }
    fclose(log);
    MPI_Finalize();
    return status;
}
