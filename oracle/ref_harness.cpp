// Harness around the reference's own CPU flow solver, compiled unmodified from
// its sources (include/flow/FlowSolver.{hpp,inl}, include/geometry/Mesh.hpp,
// src/examples/mesh_examples.cpp, include/utils/utils.hpp) against the
// single-rank MPI and PETSc shims in ref_shim/.  Test infrastructure only: it
// is built into oracle/_ref/ and used to pin the oracle restatement and to
// produce golden vectors; the product never links it.
//
// Members are made reachable with `#define private public` in this TU only, so
// the harness can read phi, gradients, face fluxes and the assembled matrices
// and can run single SIMPLE passes.
#include <algorithm>
#include <cinttypes>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <bitset>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "mpi.h"
#include "petscksp.h"

#define private public
#include "utils/utils.hpp"
#include "geometry/Mesh.hpp"
#include "performance/PerformanceLogger.hpp"
#include "particles/Particle.hpp"
using namespace minicombust::performance;
using namespace minicombust::particles;
#include "visit/VisitWriter.hpp"
#include "examples/mesh_examples.hpp"
using namespace minicombust::visit;
#include "flow/FlowSolver.inl"
#undef private

using namespace minicombust::flow;

namespace {

struct RefHandle {
    MPI_Config mpi;
    Mesh<double> *mesh = nullptr;
    FlowSolver<double> *solver = nullptr;
    FILE *log = nullptr;
    int pass_in_step = 0;  // loop index i of FlowSolver::timestep (FlowSolver.inl:3188)
};

// Single flow rank configuration, following minicombust.cpp:96-117 and :142-148.
void init_mpi_config(MPI_Config &c)
{
    memset(&c, 0, sizeof(c));
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
}

double *phi_ptr(FlowSolver<double> *s, int which)
{
    phi_vector<double> &p = s->phi;
    double *a[13] = {p.U, p.V, p.W, p.P, p.PP, p.TE, p.ED, p.TP, p.TEM, p.FUL, p.PRO, p.VARF, p.VARP};
    return (which >= 0 && which < 13) ? a[which] : nullptr;
}

vec<double> *grad_ptr(FlowSolver<double> *s, int which)
{
    phi_vector<vec<double>> &g = s->phi_grad;
    // TP has no gradient array in the reference (FlowSolver.hpp:228-239).
    vec<double> *a[13] = {g.U, g.V, g.W, g.P, g.PP, g.TE, g.ED, nullptr, g.TEM, g.FUL, g.PRO, g.VARF, g.VARP};
    return (which >= 0 && which < 13) ? a[which] : nullptr;
}

uint64_t phi_len(RefHandle *h) { return h->mesh->local_mesh_size + h->solver->nhalos + h->mesh->boundary_cells_size; }

} // namespace

extern "C" {

// Build the reference box mesh (load_mesh, mesh_examples.cpp:120) and the
// reference FlowSolver (FlowSolver.hpp:147) for one flow rank.
void *mcref_create(uint64_t ex, uint64_t ey, uint64_t ez, double lx, double ly, double lz, double delta)
{
    RefHandle *h = new RefHandle();
    init_mpi_config(h->mpi);
    h->log = fopen("/dev/null", "w");
    vec<double> box_dim = {lx, ly, lz};
    vec<uint64_t> elements = {ex, ey, ez};
    h->mesh = load_mesh(&h->mpi, box_dim, elements, 1, h->log);
    h->solver = new FlowSolver<double>(&h->mpi, h->mesh, delta, h->log);
    return h;
}

void mcref_destroy(void *vh)
{
    RefHandle *h = (RefHandle *)vh;
    // The reference FlowSolver has no destructor; its buffers are released with
    // the process.  Only the object itself (which holds the 800 MB FGM table)
    // is returned here.
    ::operator delete((void *)h->solver);
    if (h->log) fclose(h->log);
    delete h;
}

void mcref_sizes(void *vh, uint64_t *cells, uint64_t *faces, uint64_t *points, uint64_t *phi_length)
{
    RefHandle *h = (RefHandle *)vh;
    *cells = h->mesh->mesh_size;
    *faces = h->mesh->faces_size;
    *points = h->mesh->points_size;
    *phi_length = phi_len(h);
}

// Mesh arrays exactly as the reference lays them out (Mesh.hpp:86-106).
void mcref_get_mesh(void *vh, double *points, uint64_t *cells, uint64_t *faces, uint64_t *cell_faces,
                    uint64_t *cell_neighbours, double *cell_centers, uint64_t *boundary_types)
{
    RefHandle *h = (RefHandle *)vh;
    Mesh<double> *m = h->mesh;
    if (points) memcpy(points, m->points, m->points_size * sizeof(vec<double>));
    if (cells) memcpy(cells, m->cells, m->mesh_size * m->cell_size * sizeof(uint64_t));
    if (faces)
        for (uint64_t f = 0; f < m->faces_size; f++) {
            faces[2 * f] = m->faces[f].cell0;
            faces[2 * f + 1] = m->faces[f].cell1;
        }
    if (cell_faces) memcpy(cell_faces, m->cell_faces, m->mesh_size * m->faces_per_cell * sizeof(uint64_t));
    if (cell_neighbours) memcpy(cell_neighbours, m->cell_neighbours, m->mesh_size * m->faces_per_cell * sizeof(uint64_t));
    if (cell_centers) memcpy(cell_centers, m->cell_centers, m->mesh_size * sizeof(vec<double>));
    if (boundary_types) memcpy(boundary_types, m->boundary_types, 6 * sizeof(uint64_t));
}

void mcref_set_tolerances(double bcgs_rtol, double cg_rtol, int max_iters) { mcshim_set_tolerances(bcgs_rtol, cg_rtol, max_iters); }

int mcref_get_field(void *vh, int which, double *out)
{
    RefHandle *h = (RefHandle *)vh;
    double *p = phi_ptr(h->solver, which);
    if (!p) return -1;
    memcpy(out, p, phi_len(h) * sizeof(double));
    return 0;
}

int mcref_set_field(void *vh, int which, const double *in)
{
    RefHandle *h = (RefHandle *)vh;
    double *p = phi_ptr(h->solver, which);
    if (!p) return -1;
    memcpy(p, in, phi_len(h) * sizeof(double));
    return 0;
}

int mcref_get_grad(void *vh, int which, double *out)
{
    RefHandle *h = (RefHandle *)vh;
    vec<double> *g = grad_ptr(h->solver, which);
    if (!g) return -1;
    memcpy(out, g, h->mesh->local_mesh_size * sizeof(vec<double>));
    return 0;
}

// which: 0..2 A_phi.U/V/W, 3..5 S_phi.U/V/W, 6 volumes, 7 densities (length N).
int mcref_get_cell_array(void *vh, int which, double *out)
{
    RefHandle *h = (RefHandle *)vh;
    FlowSolver<double> *s = h->solver;
    double *a[8] = {s->A_phi.U, s->A_phi.V, s->A_phi.W, s->S_phi.U, s->S_phi.V, s->S_phi.W, s->cell_volumes, s->cell_densities};
    if (which < 0 || which >= 8) return -1;
    memcpy(out, a[which], h->mesh->local_mesh_size * sizeof(double));
    return 0;
}

// which: 0 mass flux, 1 area, 2 lambda, 3 rlencos, 4 face_fields (2/face),
// 5 normals (3/face), 6 centres (3/face).
int mcref_get_face_array(void *vh, int which, double *out)
{
    RefHandle *h = (RefHandle *)vh;
    FlowSolver<double> *s = h->solver;
    const uint64_t F = h->mesh->faces_size;
    switch (which) {
    case 0: memcpy(out, s->face_mass_fluxes, F * sizeof(double)); return 0;
    case 1: memcpy(out, s->face_areas, F * sizeof(double)); return 0;
    case 2: memcpy(out, s->face_lambdas, F * sizeof(double)); return 0;
    case 3: memcpy(out, s->face_rlencos, F * sizeof(double)); return 0;
    case 4:
        for (uint64_t f = 0; f < F; f++) {
            out[2 * f] = s->face_fields[f].cell0;
            out[2 * f + 1] = s->face_fields[f].cell1;
        }
        return 0;
    case 5: memcpy(out, s->face_normals, F * sizeof(vec<double>)); return 0;
    case 6: memcpy(out, s->face_centers, F * sizeof(vec<double>)); return 0;
    default: return -1;
    }
}

// Assembled matrices as CSR with ascending columns.  which: 0 the shared
// momentum/scalar matrix A, 1 Pressure_A.  Pass NULL arrays to query sizes.
int mcref_get_csr(void *vh, int which, int *n, int *nnz, int *row_ptr, int *col, double *val)
{
    RefHandle *h = (RefHandle *)vh;
    Mat A = which == 0 ? h->solver->A : h->solver->Pressure_A;
    mcshim_mat_csr(A, n, nnz, row_ptr, col, val);
    return 0;
}

// which: 0 b, 1 Pressure_b, 2 u (last solution).
int mcref_get_vec(void *vh, int which, double *out)
{
    RefHandle *h = (RefHandle *)vh;
    Vec v = which == 0 ? h->solver->b : (which == 1 ? h->solver->Pressure_b : h->solver->u);
    int n = 0;
    mcshim_vec_values(v, &n, out);
    return n;
}

// One full reference timestep (FlowSolver.inl:3148-3356): three SIMPLE passes.
void mcref_timestep(void *vh)
{
    RefHandle *h = (RefHandle *)vh;
    h->solver->timestep();
    h->pass_in_step = 0;
}

// One SIMPLE pass: the body of the loop at FlowSolver.inl:3188-3268 with the
// loop index the reference would have, so that 3 passes equal one timestep()
// (timestep_count advances after the third pass, FlowSolver.inl:3355).
void mcref_pass(void *vh)
{
    RefHandle *h = (RefHandle *)vh;
    FlowSolver<double> *s = h->solver;
    const int i = h->pass_in_step;
    const int comms_timestep = 1;
    s->exchange_phi_halos();
    s->get_phi_gradients();
    if (FLOW_SOLVER_LIMIT_GRAD) s->limit_phi_gradients();
    s->exchange_grad_halos();
    if (s->timestep_count == 0 && i == 0) {
        s->set_up_field();
        s->set_up_fgm_table();
    }
    if (((s->timestep_count % comms_timestep) == 0) && i == 2) s->update_flow_field();
    s->calculate_UVW();
    s->exchange_phi_halos();
    s->calculate_pressure();
    s->Scalar_solve(TERBTE, s->phi.TE, s->phi_grad.TE);
    s->Scalar_solve(TERBED, s->phi.ED, s->phi_grad.ED);
    s->Scalar_solve(TEMP, s->phi.TEM, s->phi_grad.TEM);
    s->Scalar_solve(FUEL, s->phi.FUL, s->phi_grad.FUL);
    s->Scalar_solve(PROG, s->phi.PRO, s->phi_grad.PRO);
    s->Scalar_solve(VARFU, s->phi.VARF, s->phi_grad.VARF);
    s->Scalar_solve(VARPR, s->phi.VARP, s->phi_grad.VARP);
    s->FGM_loop_up();
    h->pass_in_step++;
    if (h->pass_in_step == 3) {
        h->pass_in_step = 0;
        s->timestep_count++;
    }
}

// Individual stages, for stage-by-stage comparison.
void mcref_stage_gradients(void *vh) { ((RefHandle *)vh)->solver->get_phi_gradients(); }
void mcref_stage_set_up_field(void *vh) { ((RefHandle *)vh)->solver->set_up_field(); }
void mcref_stage_calculate_uvw(void *vh) { ((RefHandle *)vh)->solver->calculate_UVW(); }
void mcref_stage_calculate_pressure(void *vh) { ((RefHandle *)vh)->solver->calculate_pressure(); }
void mcref_stage_scalar_temperature(void *vh)
{
    FlowSolver<double> *s = ((RefHandle *)vh)->solver;
    s->Scalar_solve(TEMP, s->phi.TEM, s->phi_grad.TEM);
}
// Scalar_solve for one transported field (phi_vector member index:
// 5 TE, 6 ED, 8 TEM, 9 FUL, 10 PRO, 11 VARF, 12 VARP).
int mcref_stage_scalar(void *vh, int field)
{
    FlowSolver<double> *s = ((RefHandle *)vh)->solver;
    switch (field) {
    case 5: s->Scalar_solve(TERBTE, s->phi.TE, s->phi_grad.TE); return 0;
    case 6: s->Scalar_solve(TERBED, s->phi.ED, s->phi_grad.ED); return 0;
    case 8: s->Scalar_solve(TEMP, s->phi.TEM, s->phi_grad.TEM); return 0;
    case 9: s->Scalar_solve(FUEL, s->phi.FUL, s->phi_grad.FUL); return 0;
    case 10: s->Scalar_solve(PROG, s->phi.PRO, s->phi_grad.PRO); return 0;
    case 11: s->Scalar_solve(VARFU, s->phi.VARF, s->phi_grad.VARF); return 0;
    case 12: s->Scalar_solve(VARPR, s->phi.VARP, s->phi_grad.VARP); return 0;
    default: return -1;
    }
}
// The flow side of the flow/particle exchange (FlowSolver::update_flow_field,
// FlowSolver.inl:496-736) with the messages staged in the MPI shim
// (mcshim_inject_rank): particle terms summed into mesh->particle_terms and
// node values sent back to each rank (mcshim_outbox_*).
void mcref_update_flow_field(void *vh) { ((RefHandle *)vh)->solver->update_flow_field(); }
void mcref_get_particle_terms(void *vh, double *out)
{
    RefHandle *h = (RefHandle *)vh;
    std::memcpy(out, h->mesh->particle_terms, h->mesh->local_mesh_size * sizeof(particle_aos<double>));
}

// FlowSolver::output_data's writer (VisitWriter<T>::write_flow,
// VisitWriter.hpp:127-234) on the current fields.
void mcref_write_flow(void *vh, const char *prefix, int id)
{
    RefHandle *h = (RefHandle *)vh;
    VisitWriter<double> w(h->mesh, &h->mpi);
    w.write_flow(prefix, id, &h->solver->phi);
}
int mcref_first_pressure(void *vh) { return ((RefHandle *)vh)->solver->first_pressure ? 1 : 0; }
uint64_t mcref_timestep_count(void *vh) { return ((RefHandle *)vh)->solver->timestep_count; }
double mcref_inlet_effective_viscosity(void *vh) { return ((RefHandle *)vh)->solver->inlet_effective_viscosity; }
void mcref_last_solve(int *iters, double *relres, int *kind) { mcshim_last_solve(iters, relres, kind); }
void mcref_solve_counts(long *bcgs, long *cg) { mcshim_solve_counts(bcgs, cg); }

} // extern "C"
