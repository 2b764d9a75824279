/*
 * flow_b200/FlowSolver.inl -- the reference's flow-solver class over this
 * library's C ABI (minicombust_flow.h), for the reference's own driver.
 *
 * It is compiled inside the reference's tree in place of its CPU or GPU
 * back-end: src/minicombust.cpp includes "flow/FlowSolver.inl" (CPU) or
 * "flow/gpu/FlowSolver.inl" (GPU) at :15-48 and uses exactly the members
 * declared here -- the constructor (:174), timestep() (:221),
 * output_data(t) (:226), print_logger_stats (:249), compute_time (:277-282)
 * and AMGX_free() (:322, GPU build).  The class keeps the reference's name,
 * namespace and signatures (include/flow/FlowSolver.hpp:147, 1003-1048;
 * include/flow/gpu/FlowSolver.hpp:274), takes the reference's Mesh<T> as
 * load_mesh builds it, and runs every pass on the GPU through one mc_flow
 * handle.  Needs the reference's include/ directory on the include path (for
 * Mesh<T>, MPI_Config and the vec/particle types) and this repository's
 * include/; link with -lmcflow.
 *
 * Status codes become exceptions (std::runtime_error with the library's
 * message) where the reference would have exited; a Krylov solve that
 * stops at max_iters is reported on output_file and the run continues, as
 * the reference prints and continues (FlowSolver.inl:1355-1360, 2255-2260).
 */
#pragma once

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "geometry/Mesh.hpp"
#include "utils/utils.hpp"

#include "minicombust_flow.h"

namespace minicombust::flow
{
template <class T>
class FlowSolver
{
    static_assert(std::is_same<T, double>::value, "the B200 flow solver computes in double precision");

  public:
    MPI_Config *mpi_config;
    double compute_time = 0.0;

    // FlowSolver(MPI_Config*, Mesh<T>*, double delta, FILE*): the reference's
    // constructor (FlowSolver.hpp:147).  params: the library's settings; by
    // default the reference's constants and control flow (MC_MODE_COMPAT).
    FlowSolver(MPI_Config *mpi_config, Mesh<T> *mesh, double delta, FILE *output_file,
               const mc_flow_params *params = nullptr)
        : mpi_config(mpi_config), mesh(mesh), output_file(output_file)
    {
        if (mesh->mesh_size != mesh->local_mesh_size)
            throw std::runtime_error("the B200 flow solver takes one flow block per rank (mesh_size == local_mesh_size)");
        mc_mesh_view mv{};
        mv.cells = mesh->mesh_size;
        mv.faces = mesh->faces_size;
        mv.points = mesh->points_size;
        mv.points_xyz = &mesh->points[0].x;          // vec<double>: three doubles
        mv.cell_nodes = mesh->cells;
        mv.face_cells = &mesh->faces[0].cell0;       // Face<uint64_t>: two uint64_t
        mv.cell_faces = mesh->cell_faces;
        mv.cell_neighbours = mesh->cell_neighbours;
        mv.cell_centers = &mesh->cell_centers[0].x;
        for (int s = 0; s < 6; s++) mv.boundary_types[s] = mesh->boundary_types[s];
        mc_flow_params p;
        if (params) {
            p = *params;
        } else {
            mc_flow_default_params(&p, MC_MODE_COMPAT);
        }
        p.delta = delta;
        check(mc_flow_create(&mv, &p, &h), "mc_flow_create");
    }

    FlowSolver(const FlowSolver &) = delete;
    FlowSolver &operator=(const FlowSolver &) = delete;
    ~FlowSolver()
    {
        if (h) mc_flow_destroy(h);
    }

    // FlowSolver::timestep (FlowSolver.inl:3148-3356): the particle source
    // terms the particle ranks left in mesh->particle_terms, then three
    // SIMPLE passes on the GPU.
    void timestep()
    {
        if (mpi_config->particle_flow_rank == 0 && output_file) fprintf(output_file, "\ntimestep %lu\n", (unsigned long)(count + 1));
        compute_time -= MPI_Wtime();
        if (mesh->particle_terms) check(mc_flow_set_sources(h, &mesh->particle_terms[0].momentum.x), "mc_flow_set_sources");
        const int rc = mc_flow_timestep(h, &stats);
        compute_time += MPI_Wtime();
        count++;
        if (rc == MC_ERR_NOT_CONVERGED) {
            if (output_file) fprintf(output_file, "flow solve reached max_iters: %s\n", mc_flow_last_error(h));
        } else {
            check(rc, "mc_flow_timestep");
        }
    }

    // FlowSolver::output_data (FlowSolver.inl:18-23): the VTK flow file.
    void output_data(uint64_t timestep)
    {
        check(mc_flow_write_vtk(h, "out/flow/minicombust", (int)timestep), "mc_flow_write_vtk");
    }

    void print_logger_stats(uint64_t timesteps, double runtime)
    {
        if (mpi_config->particle_flow_rank != 0 || !output_file) return;
        fprintf(output_file, "Flow solver (B200): %lu timesteps, runtime %.3f s, compute %.3f s\n",
                (unsigned long)timesteps, runtime, compute_time);
        fprintf(output_file, "  last pass: momentum iterations %d %d %d, pressure solves %d (%d iterations), "
                             "temperature iterations %d, mass imbalance %.3e\n",
                stats.momentum_iters[0], stats.momentum_iters[1], stats.momentum_iters[2], stats.pressure_solves,
                stats.pressure_iters_total, stats.temperature_iters, stats.mass_imbalance);
    }

    void AMGX_free() {}  // the GPU build's driver calls it; nothing to release here

    // Access for drivers that compare or post-process: a field (cells + 6
    // values, phi_vector member order) and the handle itself.
    void get_field(int which, T *out) { check(mc_flow_get_field(h, which, out), "mc_flow_get_field"); }
    void set_field(int which, const T *in) { check(mc_flow_set_field(h, which, in), "mc_flow_set_field"); }
    mc_flow *handle() { return h; }
    const mc_iter_stats &last_stats() const { return stats; }

  private:
    void check(int rc, const char *what)
    {
        if (rc == MC_OK) return;
        std::string msg = std::string(what) + ": " + mc_status_string(rc);
        if (h && mc_flow_last_error(h)[0]) msg += std::string(" (") + mc_flow_last_error(h) + ")";
        throw std::runtime_error(msg);
    }

    Mesh<T> *mesh;
    FILE *output_file;
    mc_flow *h = nullptr;
    mc_iter_stats stats{};
    uint64_t count = 0;
};
} // namespace minicombust::flow
