/*
 * minicombust_flow.h -- C ABI of the B200 (sm_100a) flow-solver SIMPLE pass.
 *
 * This is the drop-in boundary for miniCOMBUST's flow solver.  It replaces:
 *   - the reference CPU solver's per-pass work (include/flow/FlowSolver.inl,
 *     timestep loop :3188-3268, stages cited per entry point below), and
 *   - the reference GPU back-end's launch shims (include/flow/gpu/gpu_kernels.cuh:11-82,
 *     "void C_kernel_*(int block_count, int thread_count, device pointers...)")
 *     together with the AmgX calls of include/flow/gpu/FlowSolver.inl:644-1025.
 * Those shims take raw device pointers, return nothing and exit() on error
 * (gpu_kernels.cu:24-32).  Here a handle owns every device buffer, inputs and
 * outputs are host arrays in the reference layout, every call returns a status
 * code and nothing exits the process.
 *
 * Layout contract (the reference's, Mesh.hpp:86-106 and utils.hpp:158-174):
 *   - cells are indexed 0..cells-1; a face is {cell0, cell1} with cell0 < cell1;
 *     a boundary face has cell1 = cells + d, d = 0..5 the boundary side
 *     FRONT, BACK, LEFT, RIGHT, DOWN, UP, whose type is boundary_types[d]
 *     (1 wall, 2 inlet, 3 outlet);
 *   - a field is an array of cells + 6 doubles: interior values, then the
 *     value of each boundary side at index cells + d;
 *   - particle source terms are particle_aos<double> per cell:
 *     {momentum.x, momentum.y, momentum.z, energy, fuel (mass)}.
 *
 * Threading: one host thread per handle at a time; each handle owns one CUDA
 * stream on the device chosen at creation.  Calls are synchronous unless noted.
 */
#ifndef MINICOMBUST_FLOW_H
#define MINICOMBUST_FLOW_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MC_FLOW_ABI_VERSION 2

typedef enum mc_status {
    MC_OK = 0,
    MC_ERR_ARG = -1,            /* bad argument or handle */
    MC_ERR_CUDA = -2,           /* a CUDA call failed; see mc_flow_last_error */
    MC_ERR_NOT_CONVERGED = -3,  /* a Krylov solve reached max_iters */
    MC_ERR_NONFINITE = -4,      /* a residual or reduction became NaN/Inf */
    MC_ERR_MESH = -5,           /* mesh arrays inconsistent */
    MC_ERR_NOMEM = -6,          /* device or host allocation failed */
    MC_ERR_UNSUPPORTED = -7,    /* option not available in this build */
    MC_ERR_TIMEOUT = -8         /* a bounded device-side wait gave up (tensor-core kernels) */
} mc_status;

enum { MC_MODE_COMPAT = 0, MC_MODE_SIMPLE = 1 };
enum { MC_PSOLVER_PCG_JACOBI = 0, MC_PSOLVER_PCG_AMG = 1 };
enum { MC_PRECISION_FP64 = 0, MC_PRECISION_FP32_REFINED = 1 };
enum { MC_GUESS_ZERO = 0, MC_GUESS_PREVIOUS = 1, MC_GUESS_LEARNED = 2 };
/* Cell order inside the handle.  Inputs and outputs of every call stay in the
 * caller's (reference) numbering; MC_REORDER_RCM renumbers cells by reverse
 * Cuthill-McKee and faces by first touch in that order, on the device only. */
enum { MC_REORDER_NONE = 0, MC_REORDER_RCM = 1 };

/* Field ids: the member order of phi_vector<T> (utils.hpp:158-174). */
enum {
    MC_FIELD_U = 0, MC_FIELD_V = 1, MC_FIELD_W = 2, MC_FIELD_P = 3, MC_FIELD_PP = 4,
    MC_FIELD_TE = 5, MC_FIELD_ED = 6, MC_FIELD_TP = 7, MC_FIELD_TEM = 8,
    MC_FIELD_FUL = 9, MC_FIELD_PRO = 10, MC_FIELD_VARF = 11, MC_FIELD_VARP = 12
};

/* Linear systems readable with mc_flow_get_csr.  MC_SYSTEM_TEMPERATURE is the
 * scalar-transport system assembled last: T, or with transport_scalars the
 * last of TE, ED, TEM, FUL, PRO, VARF, VARP that ran (they share storage, as
 * they share the reference's A/b, FlowSolver.inl:2885-2960). */
enum { MC_SYSTEM_MOMENTUM = 0, MC_SYSTEM_PRESSURE = 1, MC_SYSTEM_TEMPERATURE = 2 };

/* Mesh in the reference layout (Mesh<T> public arrays, Mesh.hpp:86-106). */
typedef struct mc_mesh_view {
    uint64_t cells;                  /* Mesh::mesh_size */
    uint64_t faces;                  /* Mesh::faces_size */
    uint64_t points;                 /* Mesh::points_size */
    const double *points_xyz;        /* [points][3]  Mesh::points */
    const uint64_t *cell_nodes;      /* [cells][8]   Mesh::cells, vertex order A..H */
    const uint64_t *face_cells;      /* [faces][2]   Mesh::faces */
    const uint64_t *cell_faces;      /* [cells][6]   Mesh::cell_faces */
    const uint64_t *cell_neighbours; /* [cells][6]   Mesh::cell_neighbours (UINT64_MAX on the boundary) */
    const double *cell_centers;      /* [cells][3]   Mesh::cell_centers */
    uint64_t boundary_types[6];      /* Mesh::boundary_types */
} mc_mesh_view;

/* Physics and solver settings.  mc_flow_default_params fills the reference's
 * constants (FlowSolver.hpp:296,342; Mesh.hpp:114-116; FlowSolver.inl:1731,
 * 1871, 2425, 2939-2946; minicombust.cpp:120) for MC_MODE_COMPAT and the
 * benchmark physics for MC_MODE_SIMPLE. */
typedef struct mc_flow_params {
    int mode;                 /* MC_MODE_COMPAT: the reference's control flow and quirks;
                                 MC_MODE_SIMPLE: corrected SIMPLE pass (see below) */
    double delta;             /* time step */
    double density;
    double viscosity;
    double inlet_u;           /* inlet velocity (x); v = w = 0 */
    double pressure0;         /* initial and boundary pressure */
    double temperature0;      /* initial, inlet and buoyancy-reference temperature */
    double urf_momentum;
    double urf_pressure;
    double urf_temperature;
    double flux_corr;         /* non-orthogonal flux-correction factor */
    double u_rtol;            /* momentum and temperature BiCGStab: ||r|| <= u_rtol ||b|| */
    double p_rtol;            /* pressure-correction PCG: ||r|| <= p_rtol ||b|| */
    int max_iters;            /* per Krylov solve */
    int pressure_solver;      /* MC_PSOLVER_* */
    int precision;            /* MC_PRECISION_* */
    int initial_guess;        /* MC_GUESS_* for the first pressure correction of a pass (later ones start at 0) */
    int device;               /* CUDA device ordinal */
    int amg_sweeps;           /* MC_PSOLVER_PCG_AMG: damped-Jacobi sweeps before and after the coarse correction */
    double amg_omega;         /* Jacobi damping (every sweep, when amg_cheb_ratio is 0) */
    double amg_alpha;         /* coarse-correction scaling */
    double ir_inner_rtol;     /* MC_PRECISION_FP32_REFINED: each inner FP32 pressure solve reduces its
                                 residual by the factor still missing to p_rtol (with a margin of 2), but
                                 by no less than this: the smallest relative tolerance asked of it */
    int reorder;              /* MC_REORDER_* */
    double ir_inner_rtol_bicg; /* the same floor for the inner FP32 BiCGStab solves of momentum and
                                  temperature (their target is u_rtol) */
    double amg_cheb_ratio;    /* MC_PSOLVER_PCG_AMG: > 1 gives the amg_sweeps sweeps the damping of a
                                 Chebyshev smoother on [2 / ratio, 2] (a different damping per sweep,
                                 the reciprocal roots of the polynomial); 0: every sweep damps by
                                 amg_omega */
    int transport_scalars;    /* 0: a pass transports u, v, w, p and T only (none of them depends on
                                 the other scalars); 1: it also solves the reference's other scalar
                                 transports -- turbulent kinetic energy and dissipation (k-epsilon
                                 with wall functions), mixture fraction, progress variable and their
                                 two variances -- in the reference's order TE, ED, TEM, FUL, PRO,
                                 VARF, VARP (FlowSolver.inl:3229-3261).  Default: 1 in
                                 MC_MODE_COMPAT, 0 in MC_MODE_SIMPLE. */
    int ir_line_steps;        /* MC_PRECISION_FP32_REFINED, momentum and temperature: k > 0 makes each inner
                                 FP32 solve k steps of an x-line sweep (the splitting that keeps the
                                 diagonal and the upwind -x couplings, solved along each line) on meshes
                                 whose cells run x-fastest along whole lines; 0, or another mesh: inner
                                 BiCGStab.  Default 2. */
} mc_flow_params;

/* Per-pass statistics. */
typedef struct mc_iter_stats {
    int momentum_iters[3];
    int temperature_iters;
    int pressure_solves;
    int pressure_iters_total;
    int pressure_iters_first;
    double pressure_correction_max_first;
    double pressure_rel_residual;    /* max over the pass's pressure solves of ||r|| / ||b_1||, b_1 the
                                        first solve's right-hand side (later correctors stop on
                                        p_rtol ||b_1||) */
    double mass_imbalance;           /* max over cells |div(mdot) - mass source| after the pass */
    int guess_choice_first;          /* initial guess of the first pressure solve: -1 zero, 2 the
                                        residual-minimising combination of the previous correction and
                                        (MC_GUESS_LEARNED) the network's prediction */
    double guess_rel_residual_first; /* ||b - A x0|| / ||b|| of that guess (1 for zero) */
    double pressure_rel_residual_first; /* ||r|| / ||b|| at the end of the first pressure solve */
    int scalar_iters[6];             /* transport_scalars: BiCGStab iterations of TE, ED, FUL, PRO,
                                        VARF, VARP (0 when not run) */
} mc_iter_stats;

typedef struct mc_flow mc_flow;

/* Fill params with the defaults of a mode. */
void mc_flow_default_params(mc_flow_params *params, int mode);

/* Replaces the FlowSolver constructor (FlowSolver.hpp:147-539; GPU back-end
 * gpu/FlowSolver.hpp:274-1118): face geometry, cell volumes, initial fields,
 * matrix pattern, device buffers.  The mesh is copied; the caller keeps it. */
int mc_flow_create(const mc_mesh_view *mesh, const mc_flow_params *params, mc_flow **out);
int mc_flow_destroy(mc_flow *flow);

/* Field access, cells + 6 doubles (FlowSolver::phi).  Without
 * transport_scalars, fields outside the coupled set U, V, W, P, PP, TEM
 * return MC_ERR_UNSUPPORTED; with it all 13 fields are held. */
int mc_flow_set_field(mc_flow *flow, int field, const double *host_values);
int mc_flow_get_field(mc_flow *flow, int field, double *host_values);
/* Least-squares gradient of U, V, W, P, PP or TEM (and, with
 * transport_scalars, TE, ED, FUL, PRO, VARF, VARP), [cells][3]. */
int mc_flow_get_gradient(mc_flow *flow, int field, double *host_values);
/* Particle source terms, [cells][5] particle_aos<double> (Mesh::particle_terms). */
int mc_flow_set_sources(mc_flow *flow, const double *host_particle_terms);
/* The same from device memory the caller owns: terms_soa[5][cells] (component
 * k of cell i at k * cells + i, caller's numbering) on the handle's device.
 * The copy and the total mass source are formed on the handle's stream (the
 * data must be ready on it); nothing crosses to the host, so time-varying
 * sources can be updated every pass.  No reference counterpart. */
int mc_flow_set_sources_device(mc_flow *flow, const double *terms_soa);
/* Face arrays in reference face order.  which: 0 mass flux [faces], 1 area,
 * 2 lambda, 3 rlencos, 4 face_fields [faces][2], 5 normals [faces][3], 6 centres [faces][3]. */
int mc_flow_get_face_array(mc_flow *flow, int which, double *host_values);
/* Particle-to-cell source terms, the flow side of the flow/particle
 * exchange (FlowSolver::update_flow_field, FlowSolver.inl:496-736; GPU
 * back-end gpu_kernels.cu:131-149): `rows` rows from the particle ranks in
 * arrival order, each a cell id (caller's numbering) and a particle_aos<double>
 * {momentum.x, momentum.y, momentum.z, energy, fuel}.  They replace the
 * handle's sources as mc_flow_set_sources does: every cell is zeroed and each
 * row added to its cell, a cell's rows in arrival order, so the sums equal
 * the reference's sequential loop bit for bit.  A cell id >= cells returns
 * MC_ERR_ARG; more than 2^29 rows in one call, MC_ERR_UNSUPPORTED. */
int mc_flow_ingest_particles(mc_flow *flow, int64_t rows, const uint64_t *cells, const double *terms);
/* The handle's particle source terms, [cells][5] particle_aos<double>. */
int mc_flow_get_sources(mc_flow *flow, double *terms);
/* Flow state at mesh nodes for the particle side (get_neighbour_cells and
 * interpolate_to_nodes, FlowSolver.inl:293-494; gpu_kernels.cu:2132-2198):
 * for every distinct node of the n_cells given cells (caller ids), in
 * ascending node id, the velocity, pressure and temperature interpolated
 * from the cells around the node -- (8 - n_c)/8 of the reference gas state
 * (inlet_u, 0, 0; pressure0; temperature0) for the n_c < 8 cells a boundary
 * node lacks, plus, for each cell c sharing the node in ascending cell id,
 * (phi_c + grad phi_c . (x_node - x_c)) / 8, with the current fields and the
 * gradients of the last gradient stage.  node_ids[n] and node_fields[n][5] =
 * flow_aos<double> {vel.x, vel.y, vel.z, pressure, temp}; *n_nodes receives n.
 * With node_ids and node_fields NULL only n is computed; otherwise n above
 * max_nodes returns MC_ERR_ARG.  The reference sums each node's cells in
 * hash-set order, so its values differ from these in the last bits only. */
int mc_flow_interpolate_nodes(mc_flow *flow, int64_t n_cells, const uint64_t *cells, int64_t max_nodes,
                              int64_t *n_nodes, uint64_t *node_ids, double *node_fields);

/* Flow-field output for visualisation, the file the reference's
 * VisitWriter<T>::write_flow writes (include/visit/VisitWriter.hpp:127-234,
 * called by FlowSolver::output_data, FlowSolver.inl:18-23): legacy-VTK
 * POLYDATA at the cell centres, file "<prefix>_flow0_timestep<id>.vtk", with
 * the velocity vector and the scalar blocks in the reference's order, labels
 * and number formatting (the blocks labelled flow_ful and flow_pro carry the
 * progress variable and the mixture fraction, as the reference writes them).
 * Scalars the handle does not transport are written as zeros. */
int mc_flow_write_vtk(mc_flow *flow, const char *prefix, int id);
/* Checkpoint and resume.  No reference counterpart (the reference restarts
 * from its initial state).  The file holds the state a pass carries to the
 * next -- every field with its boundary slots, face mass fluxes, the
 * pressure-correction system (reused across passes in compat mode), sources,
 * the previous correction, the timestep counters -- in the handle's own cell
 * order, behind a 128-byte header ("MCCKPT01").  It can be read into a handle
 * created with the same mesh and the same mode, reorder, precision, pressure
 * solver and transport_scalars (MC_ERR_ARG otherwise); continuing from it
 * gives the passes the uninterrupted run would have given. */
int mc_flow_checkpoint_write(mc_flow *flow, const char *path);
int mc_flow_checkpoint_read(mc_flow *flow, const char *path);

/* The handle's cell order: cell_new_to_old[i] = caller's id of the handle's
 * i-th cell (the identity without reordering).  No reference counterpart. */
int mc_flow_get_cell_order(mc_flow *flow, int *cell_new_to_old);

/* Parameters of the learned pressure-correction guess (MC_GUESS_LEARNED);
 * the layout is that of mc_gnn_get_params (minicombust_gnn.h).  Required
 * before the first pass with MC_GUESS_LEARNED.  No reference counterpart. */
int mc_flow_set_guess_params(mc_flow *flow, const float *params, int count);

/* Snapshot dataset writer: after every pressure-correction solve, append one
 * record of four float32 arrays of `cells` values in the caller's numbering
 * -- the right-hand side projected to mean zero, the matrix diagonal, the
 * previous converged correction and the converged correction -- to `path`,
 * until max_records have been written.  File: a 64-byte header (magic
 * "MCSNAP01", uint32 version 1, uint32 cells, uint32 fields 4, uint32 dtype 0
 * = float32, uint64 records, zero padding), then the records.  The record
 * count is written on close.  No reference counterpart. */
int mc_flow_snapshot_open(mc_flow *flow, const char *path, int max_records);
int mc_flow_snapshot_close(mc_flow *flow);
/* which: 0 A_phi.U (momentum diagonal after under-relaxation), 1 pressure
 * diagonal, 2 cell volumes, 3 cell densities; [cells]. */
int mc_flow_get_cell_array(mc_flow *flow, int which, double *host_values);
/* Assembled system as CSR with ascending columns (the PETSc AIJ pattern the
 * reference builds, FlowSolver.inl:1186-1297 and 2106-2201) and its right-hand
 * side.  Pass NULL arrays to query n and nnz. */
int mc_flow_get_csr(mc_flow *flow, int system, int *n, int *nnz, int *row_ptr, int *col, double *val, double *rhs);

/* One SIMPLE pass: the body of FlowSolver::timestep's loop (FlowSolver.inl:3188-3268)
 * for the coupled fields u, v, w, p, T.  stats may be NULL. */
int mc_flow_simple_iteration(mc_flow *flow, mc_iter_stats *stats);
/* FlowSolver::timestep (FlowSolver.inl:3148-3356): three SIMPLE passes. */
int mc_flow_timestep(mc_flow *flow, mc_iter_stats *stats);

/* The stages of a pass, callable one at a time (same order as in a pass). */
int mc_flow_stage_gradients(mc_flow *flow);   /* get_phi_gradients, FlowSolver.inl:917-1063 */
int mc_flow_stage_set_up_field(mc_flow *flow);/* set_up_field, FlowSolver.inl:1106-1113 */
int mc_flow_stage_momentum(mc_flow *flow, mc_iter_stats *stats);    /* calculate_UVW, :1655-1810 */
int mc_flow_stage_pressure(mc_flow *flow, mc_iter_stats *stats);    /* calculate_pressure, :2317-2514 */
int mc_flow_stage_temperature(mc_flow *flow, mc_iter_stats *stats); /* Scalar_solve(TEMP), :2885-3076 */
/* Scalar_solve for one transported scalar (FlowSolver.inl:2885-3076, with
 * FluxScalar :2516-2744 and solveTurbulenceModels :2746-2883): field is
 * MC_FIELD_TE, _ED, _TEM, _FUL, _PRO, _VARF or _VARP.  The fields other than
 * TEM need transport_scalars (MC_ERR_UNSUPPORTED otherwise). */
int mc_flow_stage_scalar(mc_flow *flow, int field, mc_iter_stats *stats);

/* Kernel timing on the handle's stream (CUDA events around each launch).
 * While enabled, passes run without graph replay.  Times accumulate until
 * reset; ids are dense from 0 to mc_flow_kernel_count()-1. */
int mc_flow_set_timing(mc_flow *flow, int enable);
int mc_flow_kernel_count(void);
const char *mc_flow_kernel_name(int id);
int mc_flow_get_kernel_times(mc_flow *flow, double *total_ms, long *launches);
int mc_flow_reset_kernel_times(mc_flow *flow);
/* The handle's cudaStream_t, for callers that time around it. */
void *mc_flow_stream(mc_flow *flow);
/* Number of this library's kernel launches since creation. */
long mc_flow_launch_count(mc_flow *flow);

const char *mc_flow_last_error(mc_flow *flow);
const char *mc_status_string(int status);

/* Allocation-free solve.  No counterpart in the reference: it is offered to
 * callers that must not allocate device memory -- hosts that hand all device
 * memory to their own pool or fixed budget at start-up (a cudaMalloc from a
 * library would fail there, or take memory the host has promised elsewhere),
 * and callers inside a time-critical loop, where cudaMalloc and cudaFree can
 * synchronise the device and stall the host's other streams.
 *
 * Solves A x = b with the BiCGStab kernels the temperature stage uses (zero
 * initial guess, ||b - A x|| <= rtol ||b||), on a 7-point system the caller
 * owns on the current device, given in the ELL layout of this library:
 * diag[n], off[6][n], col[6][n] (an unused slot has col = its row, off = 0).
 * All pointers are device pointers; x receives the solution.  Work goes on
 * `stream` (a cudaStream_t, may be NULL); the call returns when it is done.
 * Nothing is allocated: the Krylov vectors, partial sums and status live in
 * one file-scope device array sized for MC_SOLVE_NOALLOC_MAX_ROWS rows (about
 * 16 MB, held by every device that loads the library until the process
 * exits).  n above that limit returns MC_ERR_ARG.  All calls share the array,
 * which keeps the last call's contents (each call clears what must start at
 * zero), so calls that overlap on the GPU race.  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress, once per device, with
 * that device current).  iterations (may be NULL) receives the count. */
#define MC_SOLVE_NOALLOC_MAX_ROWS 262144
int mc_solve_bicgstab_noalloc(int n, const double *diag, const double *off, const int *col, const double *b,
                              double *x, double rtol, int max_iters, void *stream, int *iterations);

/* Box mesh in the reference layout: load_mesh for one flow rank
 * (src/examples/mesh_examples.cpp:120-571), x-min inlet, x-max outlet, walls
 * elsewhere.  Arrays are allocated by the library; release them with
 * mc_mesh_box_destroy. */
int mc_mesh_box_create(uint64_t ex, uint64_t ey, uint64_t ez, double lx, double ly, double lz, mc_mesh_view *out);
void mc_mesh_box_destroy(mc_mesh_view *mesh);

/* Validate a mesh and write the reverse Cuthill-McKee cell order that
 * MC_REORDER_RCM uses (cell_new_to_old[i] = caller's id of the i-th cell).
 * Host only.  No reference counterpart. */
int mc_mesh_rcm_order(const mc_mesh_view *mesh, int *cell_new_to_old);

#ifdef __cplusplus
}
#endif
#endif /* MINICOMBUST_FLOW_H */
