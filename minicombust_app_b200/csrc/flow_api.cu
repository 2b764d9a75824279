// C ABI of the B200 flow solver (include/minicombust_flow.h): handle
// lifetime, device memory arena, the SIMPLE pass orchestration and the host
// side of the Krylov solves (batched iterations captured in CUDA graphs, one
// status read per batch).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <new>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "amg.h"
#include "exchange.cuh"
#include "flow_kernels.cuh"
#include "gnn.cuh"
#include "krylov.cuh"
#include "mc_internal.h"
#include "mc_reduce.cuh"
#include "mesh_setup.h"
#include "minicombust_flow.h"

using namespace mcb;

namespace {

enum KernelId {
    K_GRAD5, K_GRAD1, K_PRECOMP_AU, K_MOMENTUM, K_MASS_FLUX, K_OUTLET_FIX, K_PRESSURE_ROWS, K_PP_FACES,
    K_PP_CELLS, K_P_BOUNDARY, K_PP_MAX, K_TEMPERATURE, K_IMBALANCE, K_PCG_MEAN, K_PCG_INIT, K_PCG_ITER1,
    K_PCG_ITER2, K_PCG_XMEAN, K_PCG_SUBMEAN, K_BICG3_INIT, K_BICG3_1, K_BICG3_2, K_BICG3_3, K_BICG1_INIT,
    K_BICG1_1, K_BICG1_2, K_BICG1_3, K_AMG_SETUP, K_PCG_INIT_AMG, K_PCG_ITER2_AMG, K_AMG_VCYCLE,
    K_IR, K_PCG_INIT_AMG32, K_PCG_ITER1_32, K_PCG_ITER2_AMG32, K_AMG_VCYCLE32, K_PERMUTE, K_GUESS, K_GNN,
    K_SNAPSHOT, K_BIR, K_ROUND_ELL, K_BICG3_INIT32, K_BICG3_1_32, K_BICG3_2_32, K_BICG3_3_32, K_BICG1_INIT32,
    K_BICG1_1_32, K_BICG1_2_32, K_BICG1_3_32, K_GRAD6, K_SCALAR, K_SCALAR_CLIP, K_EXCHANGE, K_LINE3, K_LINE1,
    K_GNN_LAYERS, K_COUNT
};

const char *kKernelNames[K_COUNT] = {
    "lsq_gradients_uvwpt", "lsq_gradient_single", "precomp_au", "momentum_assemble", "mass_flux",
    "outlet_fix", "pressure_rows", "pp_correct_faces", "pp_correct_cells", "update_p_boundary", "pp_max",
    "temperature_assemble", "mass_imbalance", "pcg_mean", "pcg_init", "pcg_iter1_spmv", "pcg_iter2_update",
    "pcg_xmean", "pcg_sub_xmean", "bicg3_init", "bicg3_1_spmv", "bicg3_2_spmv", "bicg3_3_update",
    "bicg1_init", "bicg1_1_spmv", "bicg1_2_spmv", "bicg1_3_update", "amg_setup_galerkin_factor",
    "pcg_init_amg", "pcg_iter2_amg_update", "amg_vcycle", "ir_fp64_residual_update", "pcg32_init_amg",
    "pcg32_iter1_spmv", "pcg32_iter2_amg_update", "amg32_vcycle", "permute", "guess_select", "gnn_encode_decode",
    "snapshot_pack", "bicg_refine_fp64_residual", "round_fp32", "bicg3_32_init", "bicg3_32_1_spmv",
    "bicg3_32_2_spmv", "bicg3_32_3_update", "bicg1_32_init", "bicg1_32_1_spmv", "bicg1_32_2_spmv",
    "bicg1_32_3_update", "lsq_gradients_scalars", "scalar_assemble", "scalar_clip_negative", "particle_exchange",
    "line_sweep3_32", "line_sweep1_32", "gnn_layers"};

constexpr int PCG_BATCH = 16;   // iterations per status read (even: ping-pong buffers)
constexpr int PCG_AMG_BATCH = 4;
constexpr int BICG_BATCH = 8;

// One cudaMalloc carved into aligned sub-buffers.
struct Arena {
    char *base = nullptr;
    size_t size = 0, used = 0;
    size_t reserve(size_t bytes)
    {
        const size_t off = used;
        used += (bytes + 255) & ~(size_t)255;
        return off;
    }
};

struct Timing {
    bool on = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ids;
    size_t used = 0;
    double total_ms[K_COUNT] = {0};
    long count[K_COUNT] = {0};
};

} // namespace

struct mc_flow {
    mc_flow_params prm{};
    int N = 0, F = 0;
    int dev = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    Physics ph{};
    MeshArgs margs{};
    Arena arena;
    std::vector<int> hcol;   // ELL columns with -1 on boundary slots (CSR export)
    uint32_t *dcode = nullptr;  // direction codes of the ELL columns (used when dc.code is set)
    DirCodes dc;
    // FP64 momentum, temperature and scalar rows stored by direction
    // (rows.code set; see RowStore) and the codes the solvers read them with;
    // hcode: the direction codes on the host (CSR export)
    double *ir_x2 = nullptr;  // the refined pressure solve's second FP64 solution buffer
    RowStore rows;
    DirCodes dc_rows;
    std::vector<uint32_t> hcode;
    // the solvers' copy of the pressure-correction matrix stored by direction
    // (DirCodes::dia; with dc_pdir.sym in the half form of a symmetric
    // matrix), written with the slot-order rows; null: the solvers read those
    double *p_dir64 = nullptr;
    DirCodes dc_pdir;
    // cell/face renumbering (reorder == MC_REORDER_RCM); host and device copies
    bool reordered = false;
    std::vector<int> cell_n2o, cell_o2n, face_o2n;
    int *d_cell_n2o = nullptr, *d_cell_o2n = nullptr, *d_face_o2n = nullptr;
    double *stage = nullptr;  // max(F, N + 6) doubles, staging for permuted copies

    // mesh
    int *fc0, *fc1, *nbr, *sface, *col, *outlet_faces;
    uint8_t *sown;  // [N] bit k: the cell is cell0 of its slot-k face
    double *area, *lam, *rl, *Sx, *Sy, *Sz, *xf, *yf, *zf, *xc, *yc, *zc, *vol, *rho;
    // fields and gradients (G_U..G_T x 3 components)
    double *phi[G_NFIELDS];
    double *grad[G_NFIELDS][3];
    double *mdot, *ff0, *ff1, *fcorr;
    double *AU, *off_m, *b_m;
    double *off_p, *diag_p, *b_p;
    double *off_t, *diag_t, *b_t;
    double *src;
    // reductions
    double *partials;
    unsigned int *counter;
    FluxBalance *balance;
    double *scalars;   // [0] max|PP|, [1] mass imbalance, [2] max |diag| of the pressure rows (FP16 level 0)
    // Krylov
    PcgVectors pv{};
    BicgVectors<3> b3{};
    BicgVectors<1> b1{};
    PcgState *h_pcg = nullptr;         // pinned
    BicgState<3> *h_b3 = nullptr;      // pinned
    BicgState<1> *h_b1 = nullptr;      // pinned
    double *h_scalars = nullptr;       // pinned
    cudaGraphExec_t g_pcg = nullptr, g_b3 = nullptr, g_b1 = nullptr, g_pcg_amg = nullptr;
    // lagged coarsest inverse: formed on a side stream while the pass runs,
    // used from the next pass on
    cudaStream_t side = nullptr;
    cudaEvent_t ev_levels = nullptr, ev_inverse = nullptr;
    bool inverse_ready = false, inverse_pending = false, inverse_deferred = false;
    bool p32_written = false;  // the pressure kernel wrote the FP32 level 0 since the last AMG setup
    // device-side loops (conditional WHILE graphs) of the same solves
    cudaGraphExec_t l_pcg = nullptr, l_b3 = nullptr, l_b1 = nullptr, l_pcg_amg = nullptr;
    cudaGraphExec_t l_pcg_amg32 = nullptr, l_b3_32 = nullptr, l_b1_32 = nullptr;
    bool loops_failed = false;   // a loop graph could not be built: host-driven batches
    // aggregation AMG (pressure_solver == MC_PSOLVER_PCG_AMG)
    bool use_amg = false;
    AmgHierarchy amg;
    char *amg_mem = nullptr;
    // FP32-refined pressure solve (precision == MC_PRECISION_FP32_REFINED)
    bool refined = false;
    PcgVectorsT<float> pv32{};   // inner FP32 PCG: x = correction, b = outer residual in FP32
    float *r32 = nullptr;
    PcgState *h_pcg_inner = nullptr;  // pinned
    cudaGraphExec_t g_pcg_amg32 = nullptr;
    // FP32-refined momentum and temperature solves
    float *m32_diag = nullptr, *m32_off = nullptr, *t32_diag = nullptr, *t32_off = nullptr;
    BicgVectorsT<float, 3> bi3{};
    BicgVectorsT<float, 1> bi1{};
    BirVectors<3> bo3{};
    BirVectors<1> bo1{};
    BicgState<3> *h_bi3 = nullptr;   // pinned
    BicgState<1> *h_bi1 = nullptr;
    BirState<3> *h_bo3 = nullptr;
    BirState<1> *h_bo1 = nullptr;
    cudaGraphExec_t g_b3_32 = nullptr, g_b1_32 = nullptr;
    char *bir_mem = nullptr;
    // x-line sweep inner solves (ir_line_steps > 0 on a box whose cells run
    // x-fastest): line length, the two systems and a scratch iterate
    int line_ex = 0;
    LineSystem line3{}, line1{};
    float *line_scratch = nullptr;
    // initial guess of the pressure correction
    double *pp_prev = nullptr;        // previous converged correction [N]
    GuessState *gs = nullptr;
    GuessState *h_gs = nullptr;       // pinned
    double *x0_learned = nullptr;     // [N]
    GnnGraph gnn_g{};
    GnnWork gnn_w;
    float *gnn_p = nullptr;
    __nv_bfloat16 *gnn_pk = nullptr;
    char *gnn_mem = nullptr;
    bool gnn_loaded = false;
    int guess_choice = -1;
    int corrector = 1;                // pressure-correction solve within the pass (1 = first)
    bool guess_used = false;          // the last pressure solve started from a guess
    double guess_rel = 1.0;
    // snapshot dataset writer
    FILE *snap = nullptr;
    int snap_max = 0, snap_count = 0;
    float *snap_dev = nullptr;        // [4][N] device staging (inside gnn_mem or its own allocation)
    float *snap_host = nullptr;       // pinned [4][N]
    char *snap_mem = nullptr;

    // the other scalar transports (transport_scalars): TE, ED, TP, FUL, PRO,
    // VARF, VARP fields and the gradients of all but TP, by MC_FIELD id
    bool has_scalars = false;
    char *scal_mem = nullptr;
    double *sfield[MC_FIELD_VARP + 1] = {};
    double *sgrad[MC_FIELD_VARP + 1][3] = {};
    double *xs = nullptr;             // a scalar solve's solution, copied into its field
    BicgVectors<1> bs{};              // the single-system BiCGStab buffers with x = xs
    cudaGraphExec_t g_bs = nullptr, l_bs = nullptr;
    int *neg_list = nullptr;          // negative k / epsilon cells after a solve
    unsigned int *neg_count = nullptr;

    // flow/particle exchange: the mesh's nodes (host copies taken at create;
    // device tables built on the first node interpolation) and grow-on-demand
    // buffers for the rows and requests of a call
    int P = 0;
    std::vector<int> h_cell_nodes;    // [N][8], caller order
    std::vector<double> h_points;     // [P][3]
    char *node_mem = nullptr;
    int *d_cell_nodes = nullptr, *pc_off = nullptr, *pc_cells = nullptr, *node_list = nullptr;
    int *node_counts = nullptr, *node_count = nullptr;
    double *px = nullptr, *py = nullptr, *pz = nullptr, *node_out = nullptr;
    unsigned char *node_flag = nullptr;
    char *xin_mem = nullptr;
    size_t xin_bytes = 0;

    // state of the reference's control flow
    int first_pressure = 1;
    uint64_t timestep_count = 0;
    int pass_in_step = 0;
    int sources_set = 0;
    double mass_source_total = 0.0;
    bool mass_source_on_device = false;  // sources set from device memory: total in scalars[2]
    double p_bnorm_ref = 0.0;
    long launches = 0;
    Timing timing;
    bool gp_stale = false;   // grad[G_P] is older than the corrected pressure (see ensure_pressure_gradient)
};

namespace {

int fail(mc_flow *h, int code, const std::string &msg)
{
    if (h) h->err = msg;
    return code;
}

#define CUDA_TRY(h, call)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail((h), MC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
    } while (0)

// Kernel launch with launch counting and optional event timing.
template <typename Fn>
void launch(mc_flow *h, int kid, Fn &&fn)
{
    Timing &t = h->timing;
    if (t.on) {
        if (t.used * 2 + 2 > t.ev.size()) {
            for (int i = 0; i < 64; i++) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                t.ev.push_back(e);
            }
        }
        cudaEventRecord(t.ev[2 * t.used], h->stream);
        fn();
        cudaEventRecord(t.ev[2 * t.used + 1], h->stream);
        t.ids.push_back(kid);
        t.used++;
    } else {
        fn();
    }
    h->launches++;
}

void flush_timing(mc_flow *h)
{
    Timing &t = h->timing;
    if (!t.on || t.used == 0) return;
    cudaStreamSynchronize(h->stream);
    for (size_t i = 0; i < t.used; i++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.ev[2 * i], t.ev[2 * i + 1]);
        t.total_ms[t.ids[i]] += ms;
        t.count[t.ids[i]] += 1;
    }
    t.used = 0;
    t.ids.clear();
}

int check_launch(mc_flow *h)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, MC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return MC_OK;
}

inline int blocks_for(int n) { return std::max(1, (n + MCB_THREADS - 1) / MCB_THREADS); }

int grad_index(int field)
{
    switch (field) {
    case MC_FIELD_U: return G_U;
    case MC_FIELD_V: return G_V;
    case MC_FIELD_W: return G_W;
    case MC_FIELD_P: return G_P;
    case MC_FIELD_PP: return G_PP;
    case MC_FIELD_TEM: return G_T;
    default: return -1;
    }
}

// The six scalar fields with a gradient, and TP, held only with transport_scalars.
constexpr int kScalarFields[7] = {MC_FIELD_TE, MC_FIELD_ED, MC_FIELD_TP, MC_FIELD_FUL, MC_FIELD_PRO, MC_FIELD_VARF,
                                  MC_FIELD_VARP};
constexpr int kClipCap = 4096;

bool is_scalar_field(int field)
{
    for (int f : kScalarFields)
        if (f == field) return true;
    return false;
}

// Device array of a field (cells + 6), or null when the handle does not hold it.
double *field_ptr(mc_flow *h, int field)
{
    const int g = grad_index(field);
    if (g >= 0) return h->phi[g];
    return (h->has_scalars && is_scalar_field(field)) ? h->sfield[field] : nullptr;
}

// Device gradient component d of a field, or null.
double *grad_ptr(mc_flow *h, int field, int d)
{
    const int g = grad_index(field);
    if (g >= 0) return h->grad[g][d];
    return (h->has_scalars && is_scalar_field(field) && field != MC_FIELD_TP) ? h->sgrad[field][d] : nullptr;
}

Ell momentum_matrix(mc_flow *h) { return Ell{h->N, h->AU, h->off_m, h->col, h->rows.code ? h->dc_rows : h->dc}; }
Ell pressure_matrix(mc_flow *h)
{
    if (h->p_dir64) return Ell{h->N, h->diag_p, h->p_dir64, h->col, h->dc_pdir};
    return Ell{h->N, h->diag_p, h->off_p, h->col, h->dc};
}
Ell temperature_matrix(mc_flow *h) { return Ell{h->N, h->diag_t, h->off_t, h->col, h->rows.code ? h->dc_rows : h->dc}; }

// ------------------------------------------------------------ Krylov drivers

int krylov_status_to_mc(int s)
{
    return s == KRYLOV_OK ? MC_OK : (s == KRYLOV_NONFINITE ? MC_ERR_NONFINITE : MC_ERR_NOT_CONVERGED);
}

// Graph of one batch of iterations, captured on first use.
template <typename Body>
int run_batch(mc_flow *h, cudaGraphExec_t *exec, int kernels_in_batch, Body &&body)
{
    if (h->timing.on) {
        body();
        return check_launch(h);
    }
    if (!*exec) {
        cudaGraph_t g;
        CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const long before = h->launches;
        body();
        h->launches = before;
        CUDA_TRY(h, cudaStreamEndCapture(h->stream, &g));
        CUDA_TRY(h, cudaGraphInstantiate(exec, g, 0));
        cudaGraphDestroy(g);
    }
    CUDA_TRY(h, cudaGraphLaunch(*exec, h->stream));
    h->launches += kernels_in_batch;
    return MC_OK;
}

// Device side of a loop graph: repeat the body while the solve is not done.
__global__ void k_loop_continue(cudaGraphConditionalHandle hc, const int *__restrict__ done)
{
    cudaGraphSetConditional(hc, *done ? 0u : 1u);
}

// MC_LOOP_GRAPHS=0 keeps the host-driven batches.
bool loop_graphs_enabled()
{
    static int v = -1;
    if (v < 0) {
        const char *e = std::getenv("MC_LOOP_GRAPHS");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

bool use_loops(const mc_flow *h) { return !h->timing.on && !h->loops_failed && loop_graphs_enabled(); }

constexpr int LOOP_ITERS = 2;  // iterations per loop body (even: ping-pong buffers)

// A whole solve as one graph launch: a kernel tests *done, a conditional
// WHILE node repeats `body` (LOOP_ITERS iterations whose kernels return
// early once *done is set) and the body ends with the same test, so the
// iterations run back to back on the device with no status read between
// them.  The device ends the loop at the solve's max_iters.  Returns false
// (nothing launched) when the graph cannot be built.
template <typename Body>
bool run_loop(mc_flow *h, cudaGraphExec_t *exec, const int *done, Body &&body)
{
    if (!*exec) {
        cudaGraph_t g = nullptr;
        bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
        cudaGraphConditionalHandle hc{};
        ok = ok && cudaGraphConditionalHandleCreate(&hc, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraphNode_t test = nullptr, loop = nullptr;
        if (ok) {
            void *args[] = {&hc, &done};
            cudaKernelNodeParams kp{};
            kp.func = reinterpret_cast<void *>(k_loop_continue);
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(1);
            kp.kernelParams = args;
            ok = cudaGraphAddKernelNode(&test, g, nullptr, 0, &kp) == cudaSuccess;
        }
        cudaGraphNodeParams cp{};
        if (ok) {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = hc;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            ok = cudaGraphAddNode(&loop, g, &test, 1, &cp) == cudaSuccess;
        }
        if (ok) {
            ok = cudaStreamBeginCaptureToGraph(h->stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                const long before = h->launches;
                body();
                k_loop_continue<<<1, 1, 0, h->stream>>>(hc, done);
                h->launches = before;
                cudaGraph_t captured = nullptr;
                ok = cudaStreamEndCapture(h->stream, &captured) == cudaSuccess;
            }
        }
        ok = ok && cudaGraphInstantiate(exec, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        if (!ok) {
            *exec = nullptr;
            cudaGetLastError();
            h->loops_failed = true;
            return false;
        }
    }
    if (cudaGraphLaunch(*exec, h->stream) != cudaSuccess) {
        cudaGetLastError();
        h->loops_failed = true;
        return false;
    }
    return true;
}

// Kernels a loop graph launched for `iters` iterations of `per_iter` kernels.
long loop_launches(int iters, int per_iter)
{
    const long bodies = (iters + LOOP_ITERS - 1) / LOOP_ITERS;
    return 1 + bodies * (LOOP_ITERS * per_iter + 1);
}

// Snapshot record [4][N] float32 in the caller's numbering (idx = old -> new
// or nullptr): b - mean, diagonal, previous correction, correction.
__global__ void k_snapshot_pack(int N, const double *__restrict__ b, const PcgState *__restrict__ st,
                                const double *__restrict__ diag, const double *__restrict__ prev,
                                const double *__restrict__ x, const int *__restrict__ idx, float *__restrict__ out)
{
    const double mean = st->mean;
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < N; o += gridDim.x * blockDim.x) {
        const int i = idx ? idx[o] : o;
        out[o] = (float)(b[i] - mean);
        out[(size_t)N + o] = (float)diag[i];
        out[(size_t)2 * N + o] = (float)prev[i];
        out[(size_t)3 * N + o] = (float)x[i];
    }
}

// Initial guess of a pressure-correction solve (after pcg_mean): the
// previous converged correction and, with MC_GUESS_LEARNED, the network's
// prediction compete with the zero guess on ||b' - A x0||; the winner is
// written into x.  Returns 1 when x holds the guess (0: start from zero).
// With fuse set the guess is not written to x here: A xa and A xb are kept
// (in the FP64 PCG's r and q, unused by the refined solve) and ir_init
// applies the combination (guess_ir).
int select_guess(mc_flow *h, const Ell &A, const double *b, const PcgState *st, double *x, bool fuse = false)
{
    // Only the first corrector of a pass starts from a guess: the later ones
    // solve for the small non-orthogonal remainder, which on the benchmark box
    // converges at the initial residual check, so a guess there is pure cost
    // (the reference starts every corrector from PP = 0).
    if (h->prm.initial_guess == MC_GUESS_ZERO || h->corrector > 1) return 0;
    const bool learned = h->prm.initial_guess == MC_GUESS_LEARNED;
    if (learned) {
        // the network's layers are timed apart from its encoder and decoder
        const GnnInput<double> in{b, &st->mean, A.diag, h->pp_prev};
        for (const int part : {GNN_FWD_BEGIN, GNN_FWD_LAYERS, GNN_FWD_END})
            launch(h, part == GNN_FWD_LAYERS ? K_GNN_LAYERS : K_GNN, [&] {
                gnn_forward<double>(h->stream, h->gnn_g, in, h->gnn_p, h->gnn_pk, h->gnn_w, h->x0_learned, part);
            });
        h->launches -= 2;
        CUDA_TRY(h, cudaMemcpyAsync(&h->gs->net_status, h->gnn_w.status, sizeof(int), cudaMemcpyDeviceToDevice,
                                    h->stream));
        h->launches += gnn_forward_launches() - 1;
    }
    launch(h, K_GUESS, [&] {
        guess_residuals(h->stream, A, b, st, h->pp_prev, learned ? h->x0_learned : nullptr, h->gs, h->partials,
                        h->counter, fuse ? h->pv.r : nullptr, fuse ? h->pv.q : nullptr);
    });
    if (!fuse)
        launch(h, K_GUESS,
               [&] { guess_apply(h->stream, h->N, x, h->pp_prev, learned ? h->x0_learned : nullptr, h->gs); });
    CUDA_TRY(h, cudaMemcpyAsync(h->h_gs, h->gs, sizeof(GuessState), cudaMemcpyDeviceToHost, h->stream));
    return 1;
}

// After a solve: append a snapshot record, then keep the correction as the
// next solve's previous correction.
int after_pressure_solve(mc_flow *h)
{
    if (h->prm.initial_guess != MC_GUESS_ZERO && h->corrector == 1) {
        const GuessState &g = *h->h_gs;  // the copy was ordered before the solve's final synchronisation
        if (h->prm.initial_guess == MC_GUESS_LEARNED && g.net_status)
            return fail(h, MC_ERR_TIMEOUT, "learned-guess layer kernel gave up waiting (prediction zeroed)");
        h->guess_choice = g.choice;
        h->guess_rel = g.bb > 0 ? std::sqrt((g.choice < 0 ? g.bb : g.rc) / g.bb) : 1.0;
    }
    if (h->snap && h->snap_count < h->snap_max) {
        launch(h, K_SNAPSHOT, [&] {
            k_snapshot_pack<<<blocks_for(h->N), MCB_THREADS, 0, h->stream>>>(
                h->N, h->pv.b, h->pv.st, pressure_matrix(h).diag, h->pp_prev, h->phi[G_PP],
                h->reordered ? h->d_cell_o2n : nullptr, h->snap_dev);
        });
        const size_t bytes = (size_t)4 * h->N * sizeof(float);
        CUDA_TRY(h, cudaMemcpyAsync(h->snap_host, h->snap_dev, bytes, cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        if (std::fwrite(h->snap_host, 1, bytes, h->snap) != bytes) return fail(h, MC_ERR_ARG, "snapshot write failed");
        h->snap_count++;
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->pp_prev, h->phi[G_PP], (size_t)h->N * 8, cudaMemcpyDeviceToDevice, h->stream));
    return MC_OK;
}

int launch_deferred_inverse(mc_flow *h);

int solve_pressure(mc_flow *h, double abs_floor, int *iters, double *relres, double *bnorm)
{
    const Ell A = pressure_matrix(h);
    PcgVectors v = h->pv;
    const bool amg = h->use_amg;
    launch(h, K_PCG_MEAN, [&] { pcg_mean(h->stream, A, v); });
    const int use_x0 = select_guess(h, A, v.b, v.st, v.x);
    h->guess_used = use_x0 != 0;
    if (const int rl = launch_deferred_inverse(h)) return rl;
    if (amg) {
        launch(h, K_PCG_INIT_AMG,
               [&] { pcg_init_amg(h->stream, A, v, h->prm.p_rtol, abs_floor, h->prm.max_iters, 1, use_x0); });
        launch(h, K_AMG_VCYCLE,
               [&] { amg_vcycle<double>(h->stream, h->amg, v.r, v.zp[0], v.st, v.partials, v.counter, 1); });
        h->launches += amg_kernels_per_vcycle(h->amg, false) - 1;
    } else {
        launch(h, K_PCG_INIT,
               [&] { pcg_init(h->stream, A, v, h->prm.p_rtol, abs_floor, h->prm.max_iters, use_x0, 1); });
    }
    int rc = check_launch(h);
    if (rc) return rc;
    // The device marks the solve done at max_iters; the host bound is a second guard.
    const int batch_iters = amg ? PCG_AMG_BATCH : PCG_BATCH;
    const long max_batches = h->prm.max_iters / batch_iters + 2;
    const int per_iter = amg ? 2 + amg_kernels_per_vcycle(h->amg, false) : PCG_KERNELS_PER_ITER;
    auto iterations = [&](int count) {
        for (int it = 0; it < count; it++) {
            const int pin = it & 1;
            launch(h, K_PCG_ITER1, [&] { pcg_iter1(h->stream, A, v, pin); });
            if (amg) {
                launch(h, K_PCG_ITER2_AMG, [&] { pcg_iter2_amg(h->stream, A, v, pin ^ 1); });
                launch(h, K_AMG_VCYCLE, [&] {
                    amg_vcycle<double>(h->stream, h->amg, v.r, v.zp[pin ^ 1], v.st, v.partials, v.counter, 0);
                });
                h->launches += amg_kernels_per_vcycle(h->amg, false) - 1;
            } else {
                launch(h, K_PCG_ITER2, [&] { pcg_iter2(h->stream, A, v, pin ^ 1); });
            }
        }
    };
    const bool looped = use_loops(h) &&
                        run_loop(h, amg ? &h->l_pcg_amg : &h->l_pcg, &v.st->done, [&] { iterations(LOOP_ITERS); });
    for (long batch = 0;; batch++) {
        CUDA_TRY(h, cudaMemcpyAsync(h->h_pcg, v.st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        flush_timing(h);
        if (h->h_pcg->done) break;
        if (looped) return fail(h, MC_ERR_CUDA, "pressure solve loop ended before convergence");
        if (batch > max_batches) return fail(h, MC_ERR_NOT_CONVERGED, "pressure solve state did not advance");
        rc = run_batch(h, amg ? &h->g_pcg_amg : &h->g_pcg, batch_iters * per_iter, [&] { iterations(batch_iters); });
        if (rc) return rc;
    }
    if (looped) h->launches += loop_launches(h->h_pcg->iter, per_iter);
    // a solve that stopped at its initial check from x = 0 left x = 0, whose
    // mean removal changes nothing
    if (h->h_pcg->iter > 0 || use_x0) {
        launch(h, K_PCG_XMEAN, [&] { pcg_xmean(h->stream, h->N, v); });
        launch(h, K_PCG_SUBMEAN, [&] { pcg_sub_xmean(h->stream, h->N, v); });
    }
    rc = check_launch(h);
    if (rc) return rc;
    const PcgState &s = *h->h_pcg;
    *iters = s.iter;
    *bnorm = std::sqrt(s.bb);
    *relres = s.bb > 0 ? std::sqrt(s.rr / s.bb) : 0.0;
    return krylov_status_to_mc(s.status);
}

// FP32-refined pressure solve: FP64 outer iterative refinement (true
// residual, norms, solution accumulation) around inner PCG solves whose
// matrix, vectors and AMG V-cycle are FP32 (dot products summed in FP64).
int solve_pressure_refined(mc_flow *h, double abs_floor, int *iters, double *relres, double *bnorm)
{
    const Ell A = pressure_matrix(h);
    const EllT<float> A32{h->N, h->amg.lv32[0].diag, h->amg.lv32[0].off, h->col, h->amg.lv32[0].dc};
    PcgVectors o = h->pv;
    PcgVectorsT<float> in = h->pv32;
    constexpr int kMaxOuter = 50;
    launch(h, K_PCG_MEAN, [&] { pcg_mean(h->stream, A, o); });
    const int use_x0 = select_guess(h, A, o.b, o.st, o.x, true);
    h->guess_used = use_x0 != 0;
    if (const int rl = launch_deferred_inverse(h)) return rl;
    IrGuess g{};
    if (use_x0)
        g = IrGuess{h->gs, h->pp_prev,
                    h->prm.initial_guess == MC_GUESS_LEARNED ? h->x0_learned : nullptr, h->pv.r, h->pv.q};
    launch(h, K_IR, [&] {
        ir_init(h->stream, A, o.b, o.x, nullptr, h->r32, o.st, o.partials, o.counter, h->prm.p_rtol, abs_floor, kMaxOuter,
                0, g);
    });
    int rc = check_launch(h);
    if (rc) return rc;
    const int per_iter = 2 + amg_kernels_per_vcycle(h->amg, true);
    const long max_batches = h->prm.max_iters / PCG_AMG_BATCH + 2;
    int inner_total = 0, worst = MC_OK;
    double *xcur = o.x;  // the FP64 solution alternates between o.x and ir_x2
    int outers = 0;      // outer iterations that ran an inner solve
    // A device-looped inner solve is followed at once by the outer update;
    // its state is read together with the next outer check (one
    // synchronisation per outer iteration).
    bool inner_pending = false;
    auto account_inner = [&](bool looped) -> int {
        if (looped) {
            if (!h->h_pcg_inner->done) return fail(h, MC_ERR_CUDA, "inner solve loop ended before convergence");
            h->launches += loop_launches(h->h_pcg_inner->iter, per_iter);
        }
        inner_total += h->h_pcg_inner->iter;
        if (h->h_pcg_inner->status == KRYLOV_NONFINITE) return fail(h, MC_ERR_NONFINITE, "inner FP32 solve");
        return MC_OK;
    };
    for (int outer = 0;; outer++) {
        CUDA_TRY(h, cudaMemcpyAsync(h->h_pcg, o.st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        if (inner_pending)
            CUDA_TRY(h, cudaMemcpyAsync(h->h_pcg_inner, in.st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        flush_timing(h);
        if (inner_pending) {
            inner_pending = false;
            if ((rc = account_inner(true))) return rc;
        }
        if (h->h_pcg->done) break;
        if (outer > kMaxOuter) return fail(h, MC_ERR_NOT_CONVERGED, "refinement state did not advance");
        // each inner solve asks for the reduction still missing (with a
        // margin of 2), but never for less than ir_inner_rtol
        const PcgState &os = *h->h_pcg;
        outers++;
        double inner_rtol = os.rr > 0 ? 0.5 * std::sqrt(os.tol2 / os.rr) : h->prm.ir_inner_rtol;
        inner_rtol = std::min(0.5, std::max(h->prm.ir_inner_rtol, inner_rtol));
        launch(h, K_PCG_INIT_AMG32,
               [&] { pcg_init_amg<float>(h->stream, A32, in, inner_rtol, 0.0, h->prm.max_iters, 0); });
        launch(h, K_AMG_VCYCLE32,
               [&] { amg_vcycle<float>(h->stream, h->amg, in.r, in.zp[0], in.st, in.partials, in.counter, 1); });
        h->launches += amg_kernels_per_vcycle(h->amg, true) - 1;
        rc = check_launch(h);
        if (rc) return rc;
        auto iterations = [&](int count) {
            for (int it = 0; it < count; it++) {
                const int pin = it & 1;
                launch(h, K_PCG_ITER1_32, [&] { pcg_iter1<float>(h->stream, A32, in, pin); });
                launch(h, K_PCG_ITER2_AMG32, [&] { pcg_iter2_amg<float>(h->stream, A32, in, pin ^ 1); });
                launch(h, K_AMG_VCYCLE32, [&] {
                    amg_vcycle<float>(h->stream, h->amg, in.r, in.zp[pin ^ 1], in.st, in.partials, in.counter, 0);
                });
                h->launches += amg_kernels_per_vcycle(h->amg, true) - 1;
            }
        };
        if (use_loops(h) && run_loop(h, &h->l_pcg_amg32, &in.st->done, [&] { iterations(LOOP_ITERS); })) {
            inner_pending = true;
        } else {
            for (long batch = 0;; batch++) {
                CUDA_TRY(h, cudaMemcpyAsync(h->h_pcg_inner, in.st, sizeof(PcgState), cudaMemcpyDeviceToHost,
                                            h->stream));
                CUDA_TRY(h, cudaStreamSynchronize(h->stream));
                flush_timing(h);
                if (h->h_pcg_inner->done) break;
                if (batch > max_batches) return fail(h, MC_ERR_NOT_CONVERGED, "inner solve state did not advance");
                rc = run_batch(h, &h->g_pcg_amg32, PCG_AMG_BATCH * per_iter, [&] { iterations(PCG_AMG_BATCH); });
                if (rc) return rc;
            }
            if ((rc = account_inner(false))) return rc;
        }
        // x + e and the new FP64 residual in one pass, into the other buffer
        double *const xn = (xcur == o.x) ? h->ir_x2 : o.x;
        launch(h, K_IR, [&] {
            ir_residual(h->stream, A, o.b, xcur, nullptr, h->r32, o.st, o.partials, o.counter, in.x, xn);
        });
        xcur = xn;
        rc = check_launch(h);
        if (rc) return rc;
    }
    if (xcur != o.x) CUDA_TRY(h, cudaMemcpyAsync(o.x, xcur, (size_t)h->N * 8, cudaMemcpyDeviceToDevice, h->stream));
    // a solve that stopped at its initial check from x = 0 left x = 0, whose
    // mean removal changes nothing
    if (xcur != o.x || outers > 0 || use_x0) {
        launch(h, K_PCG_XMEAN, [&] { pcg_xmean(h->stream, h->N, o); });
        launch(h, K_PCG_SUBMEAN, [&] { pcg_sub_xmean(h->stream, h->N, o); });
    }
    rc = check_launch(h);
    if (rc) return rc;
    const PcgState &st = *h->h_pcg;
    *iters = inner_total;
    *bnorm = std::sqrt(st.bb);
    *relres = st.bb > 0 ? std::sqrt(st.rr / st.bb) : 0.0;
    const int s = krylov_status_to_mc(st.status);
    return s != MC_OK ? s : worst;
}

template <int R>
int solve_bicg(mc_flow *h, const Ell &A, const BicgVectors<R> &v, BicgState<R> *hs, cudaGraphExec_t *exec,
               cudaGraphExec_t *loop, int kid_init, int kid1, int iters_out[R])
{
    launch(h, kid_init, [&] { bicg_init<R>(h->stream, A, v, h->prm.u_rtol, h->prm.max_iters); });
    int rc = check_launch(h);
    if (rc) return rc;
    const long max_batches = h->prm.max_iters / BICG_BATCH + 2;
    auto iterations = [&](int count) {
        for (int it = 0; it < count; it++) {
            const int pin = it & 1;
            launch(h, kid1, [&] { bicg_1<R>(h->stream, A, v, pin); });
            launch(h, kid1 + 1, [&] { bicg_2<R>(h->stream, A, v, pin ^ 1); });
            launch(h, kid1 + 2, [&] { bicg_3<R>(h->stream, A, v, pin ^ 1); });
        }
    };
    const bool looped = use_loops(h) && run_loop(h, loop, &v.st->all_done, [&] { iterations(LOOP_ITERS); });
    for (long batch = 0;; batch++) {
        CUDA_TRY(h, cudaMemcpyAsync(hs, v.st, sizeof(BicgState<R>), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        flush_timing(h);
        if (hs->all_done) break;
        if (looped) return fail(h, MC_ERR_CUDA, "BiCGStab loop ended before convergence");
        if (batch > max_batches) return fail(h, MC_ERR_NOT_CONVERGED, "BiCGStab state did not advance");
        rc = run_batch(h, exec, BICG_BATCH * BICG_KERNELS_PER_ITER, [&] { iterations(BICG_BATCH); });
        if (rc) return rc;
    }
    if (looped) h->launches += loop_launches(*std::max_element(hs->iter, hs->iter + R), BICG_KERNELS_PER_ITER);
    int worst = MC_OK;
    for (int j = 0; j < R; j++) {
        iters_out[j] = hs->iter[j];
        const int s = krylov_status_to_mc(hs->status[j]);
        if (s == MC_ERR_NONFINITE || worst == MC_OK) worst = (s != MC_OK) ? s : worst;
    }
    return worst;
}

// FP64 iterative refinement around FP32 BiCGStab solves (momentum, R = 3;
// temperature, R = 1): each inner solve works on the row-scaled system
// D^-1 A e = D^-1 r (FP32 copies from round_ell, D = diag A) and asks for
// the reduction still missing (margin 2, floor ir_inner_rtol_bicg); the
// outer loop stops on the FP64 true residual, ||b - A x|| <= u_rtol ||b||
// per system.
template <int R>
int solve_bicg_refined(mc_flow *h, const Ell &A, const EllT<float> &A32, const BicgVectorsT<float, R> &in,
                       const BirVectors<R> &out, BicgState<R> *hin, BirState<R> *hout, cudaGraphExec_t *exec,
                       cudaGraphExec_t *loop, int kid_init32, int kid1_32, int iters_out[R])
{
    constexpr int kMaxOuter = 30;
    const LineSystem *line = nullptr;
    if (h->prm.ir_line_steps > 0 && h->line_ex > 0) line = (R == 3) ? &h->line3 : &h->line1;
    launch(h, K_BIR, [&] { bir_init<R>(h->stream, A, out, h->prm.u_rtol, kMaxOuter); });
    int rc = check_launch(h);
    if (rc) return rc;
    for (int j = 0; j < R; j++) iters_out[j] = 0;
    const long max_batches = h->prm.max_iters / BICG_BATCH + 2;
    // as in the refined pressure solve: a device-looped inner solve's state
    // is read together with the next outer check
    bool inner_pending = false;
    auto account_inner = [&](bool looped) -> int {
        if (looped) {
            if (!hin->all_done) return fail(h, MC_ERR_CUDA, "BiCGStab loop ended before convergence");
            h->launches += loop_launches(*std::max_element(hin->iter, hin->iter + R), BICG_KERNELS_PER_ITER);
        }
        for (int j = 0; j < R; j++) {
            iters_out[j] += hin->iter[j];
            if (hin->status[j] == KRYLOV_NONFINITE) return fail(h, MC_ERR_NONFINITE, "inner FP32 BiCGStab");
        }
        return MC_OK;
    };
    for (int outer = 0;; outer++) {
        CUDA_TRY(h, cudaMemcpyAsync(hout, out.st, sizeof(BirState<R>), cudaMemcpyDeviceToHost, h->stream));
        if (inner_pending)
            CUDA_TRY(h, cudaMemcpyAsync(hin, in.st, sizeof(BicgState<R>), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        flush_timing(h);
        if (inner_pending) {
            inner_pending = false;
            if ((rc = account_inner(true))) return rc;
        }
        if (hout->all_done) break;
        if (outer > kMaxOuter) return fail(h, MC_ERR_NOT_CONVERGED, "refinement state did not advance");
        if (line) {
            // x-line sweep steps on the row-scaled FP32 system; the last step
            // writes the inner solution out.e.  A step reduces the residual by
            // about 10^3 on the flows this is meant for, so when every open
            // system is within 10^3 of its tolerance one step is taken (a slower
            // step only costs another outer iteration)
            double need = 1.0;
            for (int j = 0; j < R; j++)
                if (!hout->done[j] && hout->rr[j] > 0) need = std::min(need, std::sqrt(hout->tol2[j] / hout->rr[j]));
            const int K = need >= 1e-3 ? 1 : h->prm.ir_line_steps;
            float *E[2] = {const_cast<float *>(out.e), h->line_scratch};
            // the last step adds its result to x (the refinement update)
            for (int k = 1; k <= K; k++) {
                float *dst = E[(K - k) % 2];
                const float *prev = E[(K - k + 1) % 2];
                launch(h, R == 3 ? K_LINE3 : K_LINE1, [&] {
                    line_step<R>(h->stream, *line, out.r32, prev, dst, k == 1 ? 1 : 0, k == K ? &out : nullptr);
                });
            }
            for (int j = 0; j < R; j++)
                if (!hout->done[j]) iters_out[j] += K;
            launch(h, K_BIR, [&] { bir_residual<R>(h->stream, A, out); });
            rc = check_launch(h);
            if (rc) return rc;
            continue;
        }
        double inner_rtol = 0.5;
        for (int j = 0; j < R; j++)
            if (!hout->done[j] && hout->rr[j] > 0)
                inner_rtol = std::min(inner_rtol, 0.5 * std::sqrt(hout->tol2[j] / hout->rr[j]));
        inner_rtol = std::max(inner_rtol, h->prm.ir_inner_rtol_bicg);
        launch(h, kid_init32, [&] { bicg_init_t<float, R>(h->stream, A32, in, inner_rtol, h->prm.max_iters); });
        auto iterations = [&](int count) {
            for (int it = 0; it < count; it++) {
                const int pin = it & 1;
                launch(h, kid1_32, [&] { bicg_1_t<float, R>(h->stream, A32, in, pin); });
                launch(h, kid1_32 + 1, [&] { bicg_2_t<float, R>(h->stream, A32, in, pin ^ 1); });
                launch(h, kid1_32 + 2, [&] { bicg_3_t<float, R>(h->stream, A32, in, pin ^ 1); });
            }
        };
        if (use_loops(h) && run_loop(h, loop, &in.st->all_done, [&] { iterations(LOOP_ITERS); })) {
            inner_pending = true;
        } else {
            for (long batch = 0;; batch++) {
                CUDA_TRY(h, cudaMemcpyAsync(hin, in.st, sizeof(BicgState<R>), cudaMemcpyDeviceToHost, h->stream));
                CUDA_TRY(h, cudaStreamSynchronize(h->stream));
                flush_timing(h);
                if (hin->all_done) break;
                if (batch > max_batches) return fail(h, MC_ERR_NOT_CONVERGED, "BiCGStab state did not advance");
                rc = run_batch(h, exec, BICG_BATCH * BICG_KERNELS_PER_ITER, [&] { iterations(BICG_BATCH); });
                if (rc) return rc;
            }
            if ((rc = account_inner(false))) return rc;
        }
        launch(h, K_BIR, [&] { bir_add<R>(h->stream, A.N, out); });
        launch(h, K_BIR, [&] { bir_residual<R>(h->stream, A, out); });
        rc = check_launch(h);
        if (rc) return rc;
    }
    int worst = MC_OK;
    for (int j = 0; j < R; j++) {
        const int st = krylov_status_to_mc(hout->status[j]);
        if (st == MC_ERR_NONFINITE || worst == MC_OK) worst = (st != MC_OK) ? st : worst;
    }
    return worst;
}

// -------------------------------------------------------------- SIMPLE stages

void launch_gradients5(mc_flow *h)
{
    h->gp_stale = false;
    GradArgs<5> a{};
    const int fields[5] = {G_U, G_V, G_W, G_P, G_T};
    for (int k = 0; k < 5; k++) {
        a.phi[k] = h->phi[fields[k]];
        a.gx[k] = h->grad[fields[k]][0];
        a.gy[k] = h->grad[fields[k]][1];
        a.gz[k] = h->grad[fields[k]][2];
    }
    a.zero_boundary = 1u << 3;  // pressure: dphi = 0 on boundary faces (FlowSolver.inl:980)
    launch(h, K_GRAD5, [&] {
        launch_lsq_gradients5(h->stream, h->N, h->nbr, h->fc1, h->xc, h->yc, h->zc, h->xf, h->yf, h->zf, a);
    });
}

void launch_gradient_pressure(mc_flow *h, int g)
{
    GradArgs<1> a{};
    a.phi[0] = h->phi[g];
    a.gx[0] = h->grad[g][0];
    a.gy[0] = h->grad[g][1];
    a.gz[0] = h->grad[g][2];
    a.zero_boundary = 1u;
    launch(h, K_GRAD1, [&] {
        launch_lsq_gradients1(h->stream, h->N, h->nbr, h->fc1, h->xc, h->yc, h->zc, h->xf, h->yf, h->zf, a);
    });
}

// The pressure gradient of the corrected pressure, for readers between
// passes (get_phi_gradient(P) at the end of calculate_pressure,
// FlowSolver.inl:2454).
void ensure_pressure_gradient(mc_flow *h)
{
    if (!h->gp_stale) return;
    launch_gradient_pressure(h, G_P);
    h->gp_stale = false;
}

void launch_mass_flux(mc_flow *h)
{
    MassFluxArgs a{};
    a.U = h->phi[G_U];
    a.V = h->phi[G_V];
    a.W = h->phi[G_W];
    a.P = h->phi[G_P];
    a.AU = h->AU;
    for (int d = 0; d < 3; d++) {
        a.gU[d] = h->grad[G_U][d];
        a.gV[d] = h->grad[G_V][d];
        a.gW[d] = h->grad[G_W][d];
        a.gP[d] = h->grad[G_P][d];
    }
    a.mdot = h->mdot;
    a.ff0 = h->ff0;
    a.ff1 = h->ff1;
    a.partials = h->partials;
    a.counter = h->counter;
    a.balance = h->balance;
    a.mass_source_total = (h->prm.mode == MC_MODE_SIMPLE && h->sources_set) ? h->mass_source_total : 0.0;
    a.mass_source_dev = (h->prm.mode == MC_MODE_SIMPLE && h->sources_set && h->mass_source_on_device)
                            ? h->scalars + 2 : nullptr;
    const int grid = std::min(blocks_for(h->F), krylov_grid(h->F));
    launch(h, K_MASS_FLUX, [&] { k_mass_flux<<<grid, MCB_THREADS, 0, h->stream>>>(h->ph, h->margs, a); });
    if (h->margs.n_outlet > 0)
        launch(h, K_OUTLET_FIX, [&] {
            k_outlet_fix<<<blocks_for(h->margs.n_outlet), MCB_THREADS, 0, h->stream>>>(
                h->ph, h->margs, h->mdot, h->phi[G_U], h->phi[G_V], h->phi[G_W], h->balance);
        });
}

// Gradients of the six other scalars, with those of u, v, w, p, T at the
// start of a pass (get_phi_gradients computes all eleven, FlowSolver.inl:917-1063).
void launch_gradients_scalars(mc_flow *h)
{
    GradArgs<6> a{};
    const int fields[6] = {MC_FIELD_TE, MC_FIELD_ED, MC_FIELD_FUL, MC_FIELD_PRO, MC_FIELD_VARF, MC_FIELD_VARP};
    for (int k = 0; k < 6; k++) {
        a.phi[k] = h->sfield[fields[k]];
        a.gx[k] = h->sgrad[fields[k]][0];
        a.gy[k] = h->sgrad[fields[k]][1];
        a.gz[k] = h->sgrad[fields[k]][2];
    }
    a.zero_boundary = 0u;
    launch(h, K_GRAD6, [&] {
        launch_lsq_gradients6(h->stream, h->N, h->nbr, h->fc1, h->xc, h->yc, h->zc, h->xf, h->yf, h->zf, a);
    });
}

int stage_gradients(mc_flow *h)
{
    launch_gradients5(h);
    if (h->has_scalars) launch_gradients_scalars(h);
    return check_launch(h);
}

int stage_set_up_field(mc_flow *h)
{
    launch(h, K_PRECOMP_AU, [&] {
        k_precomp_au<<<blocks_for(h->N), MCB_THREADS, 0, h->stream>>>(h->ph, h->margs, h->mdot, h->AU);
    });
    launch_mass_flux(h);
    return check_launch(h);
}

// MC_AMG_LAGGED_INVERSE=0 forms the coarsest inverse on the critical path
// every pass.
bool lagged_inverse_enabled()
{
    static int v = -1;
    if (v < 0) {
        const char *e = std::getenv("MC_AMG_LAGGED_INVERSE");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

// AMG values for a new pressure matrix.  The coarse levels follow the matrix
// at once; the explicit inverse on the coarsest level (one block, about a
// quarter of a millisecond) is formed on a side stream from this pass's
// coarsest values and used from the next pass on, so the V-cycles of a pass
// use the inverse of the previous pass's coarsest matrix (the first pass
// forms its own in line).  The V-cycle stays one fixed symmetric operator
// within a solve.  The side launch is deferred until after the initial
// guess (launch_deferred_inverse): its block must not hold an SM while the
// network's persistent layer kernel wants every SM.
int setup_amg_values(mc_flow *h)
{
    AmgHierarchy &H = h->amg;
    const int nc = H.lv[H.levels - 1].n;
    if (h->inverse_pending) {  // the next-pass inverse formed during the previous pass
        CUDA_TRY(h, cudaStreamWaitEvent(h->stream, h->ev_inverse, 0));
        CUDA_TRY(h, cudaMemcpyAsync(H.dense, H.dense_next, (size_t)nc * nc * sizeof(double), cudaMemcpyDeviceToDevice,
                                    h->stream));
        h->inverse_pending = false;
    }
    if (h->refined)
        amg_setup_levels<float>(h->stream, H, h->p32_written, h->partials, h->counter, h->scalars + 2);
    else
        amg_setup_levels<double>(h->stream, H, false, h->partials, h->counter, h->scalars + 2);
    h->launches += h->refined ? H.levels - 1 : H.levels - 2;  // with the one the caller's launch() counts
    if (h->refined && H.lv32[0].off16) h->launches += h->p32_written ? 1 : 2;  // the FP16 level 0 (and its scale)
    h->p32_written = false;
    if (h->inverse_ready && h->side && lagged_inverse_enabled()) {
        h->inverse_deferred = true;
        return MC_OK;
    }
    if (h->refined)
        amg_coarsest_inverse<float>(h->stream, H, H.dense);
    else
        amg_coarsest_inverse<double>(h->stream, H, H.dense);
    h->launches += 1;
    h->inverse_ready = true;
    return MC_OK;
}

// The deferred coarsest inverse of this pass, on the side stream.
int launch_deferred_inverse(mc_flow *h)
{
    if (!h->inverse_deferred) return MC_OK;
    h->inverse_deferred = false;
    AmgHierarchy &H = h->amg;
    CUDA_TRY(h, cudaEventRecord(h->ev_levels, h->stream));
    CUDA_TRY(h, cudaStreamWaitEvent(h->side, h->ev_levels, 0));
    if (h->refined)
        amg_coarsest_inverse<float>(h->side, H, H.dense_next);
    else
        amg_coarsest_inverse<double>(h->side, H, H.dense_next);
    CUDA_TRY(h, cudaEventRecord(h->ev_inverse, h->side));
    h->launches += 1;
    h->inverse_pending = true;
    return MC_OK;
}

int stage_momentum(mc_flow *h, mc_iter_stats *st)
{
    MomentumArgs a{};
    a.U = h->phi[G_U];
    a.V = h->phi[G_V];
    a.W = h->phi[G_W];
    a.T = h->phi[G_T];
    for (int d = 0; d < 3; d++) {
        a.gU[d] = h->grad[G_U][d];
        a.gV[d] = h->grad[G_V][d];
        a.gW[d] = h->grad[G_W][d];
        a.gP[d] = h->grad[G_P][d];
    }
    a.mdot = h->mdot;
    a.src = h->sources_set ? h->src : nullptr;
    a.off = h->off_m;
    a.store = h->rows;
    a.AU = h->AU;
    a.b = h->b_m;
    const bool fused32 = h->bir_mem && h->dc.code;  // the FP32 copy written by the assembly itself
    if (fused32) a.f32 = Fp32Rows{h->m32_diag, h->m32_off, h->dc.code};
    launch(h, K_MOMENTUM, [&] { k_momentum_assemble<<<blocks_for(h->N), MCB_THREADS, 0, h->stream>>>(h->ph, h->margs, a); });
    int rc = check_launch(h);
    if (rc) return rc;
    int its[3] = {0, 0, 0};
    if (h->bir_mem) {
        if (!fused32)
            launch(h, K_ROUND_ELL,
                   [&] { round_ell(h->stream, h->N, h->AU, h->off_m, h->dc.code, h->m32_diag, h->m32_off); });
        const EllT<float> A32{h->N, h->m32_diag, h->m32_off, h->col, by_direction(h->dc)};
        rc = solve_bicg_refined<3>(h, momentum_matrix(h), A32, h->bi3, h->bo3, h->h_bi3, h->h_bo3, &h->g_b3_32,
                                   &h->l_b3_32, K_BICG3_INIT32, K_BICG3_1_32, its);
    } else {
        rc = solve_bicg<3>(h, momentum_matrix(h), h->b3, h->h_b3, &h->g_b3, &h->l_b3, K_BICG3_INIT, K_BICG3_1, its);
    }
    if (st)
        for (int j = 0; j < 3; j++) st->momentum_iters[j] = its[j];
    return rc;
}

int stage_pressure(mc_flow *h, mc_iter_stats *st)
{
    if (h->prm.initial_guess == MC_GUESS_LEARNED && !h->gnn_loaded)
        return fail(h, MC_ERR_ARG, "MC_GUESS_LEARNED needs mc_flow_set_guess_params first");
    const int simple = h->prm.mode == MC_MODE_SIMPLE;
    launch_mass_flux(h);
    if (simple || h->first_pressure) {
        PressureRowArgs a{};
        a.mdot = h->mdot;
        a.ff0 = h->ff0;
        a.ff1 = h->ff1;
        a.src = h->sources_set ? h->src : nullptr;
        a.off = h->off_p;
        a.diag = h->diag_p;
        a.b = h->b_p;
        h->p32_written = h->use_amg && h->refined;  // the FP32 level 0 of the hierarchy, written by the kernel
        if (h->p32_written) {
            const AmgLevelT<float> &L0 = h->amg.lv32[0];
            a.f32 = Fp32Rows{L0.diag, L0.off, L0.dc.dia ? h->dc.code : nullptr, 0};
            if (L0.off16) {  // the scale of its FP16 copy
                a.diag_max = h->scalars + 2;
                CUDA_TRY(h, cudaMemsetAsync(a.diag_max, 0, sizeof(double), h->stream));
            }
        }
        a.dir64 = h->p_dir64;
        a.dir64_sym = h->dc_pdir.sym;
        a.code = h->dc.code;
        launch(h, K_PRESSURE_ROWS, [&] {
            k_pressure_rows<<<blocks_for(h->N), MCB_THREADS, 0, h->stream>>>(h->ph, h->margs, a);
        });
        if (h->use_amg) {
            int rs = MC_OK;
            launch(h, K_AMG_SETUP, [&] { rs = setup_amg_values(h); });
            if (rs) return rs;
        }
    }
    int rc = check_launch(h);
    if (rc) return rc;
    int loop = 0, worst = MC_OK;
    double pc_ref = 0.0;
    for (;;) {
        loop++;
        int its = 0;
        double relres = 0.0, bnorm = 0.0;
        const double floor = (simple && loop > 1) ? h->prm.p_rtol * h->p_bnorm_ref : 0.0;
        h->corrector = loop;
        rc = h->refined ? solve_pressure_refined(h, floor, &its, &relres, &bnorm)
                        : solve_pressure(h, floor, &its, &relres, &bnorm);
        if (rc == MC_ERR_CUDA) return rc;
        if (rc != MC_OK && worst == MC_OK) worst = rc;
        if (loop == 1) h->p_bnorm_ref = bnorm;
        {
            const int rs = after_pressure_solve(h);
            if (rs) return rs;
        }
        if (st) {
            st->pressure_solves++;
            st->pressure_iters_total += its;
            if (loop == 1) {
                st->pressure_iters_first = its;
                st->guess_choice_first = h->guess_choice;
                st->guess_rel_residual_first = h->guess_rel;
                st->pressure_rel_residual_first = relres;
            }
            // every corrector's final residual against the first corrector's
            // right-hand side (the norm the later correctors' floor uses)
            const double rel_ref = h->p_bnorm_ref > 0 ? relres * bnorm / h->p_bnorm_ref : relres;
            st->pressure_rel_residual = std::max(st->pressure_rel_residual, rel_ref);
        }
        // A solve that met its tolerance at the initial check from the zero
        // guess leaves PP = 0 exactly: the corrections below would add zeros
        // (signed zeros aside) and max|PP| = 0 ends the loop, so skip them.
        if (rc == MC_OK && its == 0 && !h->guess_used) {
            if (!simple && h->first_pressure) h->first_pressure = 0;
            if (loop == 1 && st) st->pressure_correction_max_first = 0.0;
            break;
        }
        launch(h, K_PP_MAX, [&] {
            k_pp_max<<<krylov_grid(h->N), MCB_THREADS, 0, h->stream>>>(h->N, h->ph.cell0, h->phi[G_PP], h->partials,
                                                                       h->counter,
                                                                       h->scalars);
        });
        CUDA_TRY(h, cudaMemcpyAsync(h->h_scalars, h->scalars, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        launch_gradient_pressure(h, G_PP);
        CorrectArgs c{};
        c.PP = h->phi[G_PP];
        c.P = h->phi[G_P];
        c.U = h->phi[G_U];
        c.V = h->phi[G_V];
        c.W = h->phi[G_W];
        c.AU = h->AU;
        for (int d = 0; d < 3; d++) c.gPP[d] = h->grad[G_PP][d];
        c.ff0 = h->ff0;
        c.mdot = h->mdot;
        c.fcorr = h->fcorr;
        c.next_rhs = simple ? h->b_p : nullptr;
        const int grid_f = std::min(blocks_for(h->F), krylov_grid(h->F));
        launch(h, K_PP_FACES, [&] { k_pp_correct_faces<<<grid_f, MCB_THREADS, 0, h->stream>>>(h->ph, h->margs, c); });
        const int cell0 = (!simple && h->first_pressure) ? 1 : 0;
        launch(h, K_PP_CELLS, [&] {
            k_pp_correct_cells<<<blocks_for(h->N + 6), MCB_THREADS, 0, h->stream>>>(h->ph, h->margs, c, simple, cell0);
        });
        if (cell0) h->first_pressure = 0;
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        flush_timing(h);
        rc = check_launch(h);
        if (rc) return rc;
        const double pc_max = h->h_scalars[0];
        if (loop == 1) {
            pc_ref = pc_max;
            if (st) st->pressure_correction_max_first = pc_max;
        }
        if (!std::isfinite(pc_max)) return fail(h, MC_ERR_NONFINITE, "pressure correction is not finite");
        if (loop >= 4 || pc_max <= 0.25 * pc_ref) break;
    }
    // update_P needs the corrected pressure's gradient in six cells; the
    // whole field's gradient is formed only if something reads it before
    // the next pass's gradients replace it (ensure_pressure_gradient)
    launch(h, K_P_BOUNDARY, [&] {
        k_update_p_boundary<<<1, 32, 0, h->stream>>>(h->ph, h->margs, h->phi[G_P], h->grad[G_P][0], h->grad[G_P][1],
                                                     h->grad[G_P][2], h->nbr);
    });
    h->gp_stale = true;
    rc = check_launch(h);
    return rc ? rc : worst;
}

int stage_temperature(mc_flow *h, mc_iter_stats *st)
{
    ScalarArgs a{};
    a.phi = h->phi[G_T];
    for (int d = 0; d < 3; d++) a.g[d] = h->grad[G_T][d];
    a.mdot = h->mdot;
    a.src = h->sources_set ? h->src : nullptr;
    a.off = h->off_t;
    a.store = h->rows;
    a.diag = h->diag_t;
    a.b = h->b_t;
    a.imbalance = h->scalars + 1;
    CUDA_TRY(h, cudaMemsetAsync(a.imbalance, 0, sizeof(double), h->stream));
    const bool fused32 = h->bir_mem && h->dc.code;
    if (fused32) a.f32 = Fp32Rows{h->t32_diag, h->t32_off, h->dc.code};
    launch(h, K_TEMPERATURE, [&] {
        k_temperature_assemble<<<blocks_for(h->N), MCB_THREADS, 0, h->stream>>>(h->ph, h->margs, a);
    });
    int rc = check_launch(h);
    if (rc) return rc;
    int its[1] = {0};
    if (h->bir_mem) {
        if (!fused32)
            launch(h, K_ROUND_ELL,
                   [&] { round_ell(h->stream, h->N, h->diag_t, h->off_t, h->dc.code, h->t32_diag, h->t32_off); });
        const EllT<float> A32{h->N, h->t32_diag, h->t32_off, h->col, by_direction(h->dc)};
        rc = solve_bicg_refined<1>(h, temperature_matrix(h), A32, h->bi1, h->bo1, h->h_bi1, h->h_bo1, &h->g_b1_32,
                                   &h->l_b1_32, K_BICG1_INIT32, K_BICG1_1_32, its);
    } else {
        rc = solve_bicg<1>(h, temperature_matrix(h), h->b1, h->h_b1, &h->g_b1, &h->l_b1, K_BICG1_INIT, K_BICG1_1, its);
    }
    if (st) st->temperature_iters = its[0];
    return rc;
}

// Scalar_solve for TE, ED, FUL, PRO, VARF or VARP (FlowSolver.inl:2885-3076):
// assembly (with the k-epsilon sources), FP64 BiCGStab from zero into xs,
// the solution copied into the field, and for k and epsilon the
// replacement of negative values (:2956-2985).  TEM goes to the temperature
// stage.
int stage_scalar(mc_flow *h, int field, mc_iter_stats *st)
{
    if (field == MC_FIELD_TEM) return stage_temperature(h, st);
    int type = -1, slot = -1;
    switch (field) {
    case MC_FIELD_TE: type = SC_TERBTE; slot = 0; break;
    case MC_FIELD_ED: type = SC_TERBED; slot = 1; break;
    case MC_FIELD_FUL: type = SC_FUEL; slot = 2; break;
    case MC_FIELD_PRO: type = SC_PROG; slot = 3; break;
    case MC_FIELD_VARF: type = SC_VARFU; slot = 4; break;
    case MC_FIELD_VARP: type = SC_VARPR; slot = 5; break;
    default: return fail(h, MC_ERR_ARG, "not a transported scalar");
    }
    if (!h->has_scalars) return fail(h, MC_ERR_UNSUPPORTED, "transport_scalars is off");
    double *phi = h->sfield[field];
    ScalarArgs a{};
    a.phi = phi;
    for (int d = 0; d < 3; d++) a.g[d] = h->sgrad[field][d];
    a.mdot = h->mdot;
    a.src = nullptr;
    a.off = h->off_t;
    a.store = h->rows;
    a.diag = h->diag_t;
    a.b = h->b_t;
    TurbArgs t{};
    t.U = h->phi[G_U];
    t.V = h->phi[G_V];
    t.W = h->phi[G_W];
    for (int d = 0; d < 3; d++) {
        t.gU[d] = h->grad[G_U][d];
        t.gV[d] = h->grad[G_V][d];
        t.gW[d] = h->grad[G_W][d];
    }
    t.TE = h->sfield[MC_FIELD_TE];
    t.ED = h->sfield[MC_FIELD_ED];
    t.TP = h->sfield[MC_FIELD_TP];
    launch(h, K_SCALAR, [&] { launch_scalar_assemble(h->stream, type, h->ph, h->margs, a, t); });
    int rc = check_launch(h);
    if (rc) return rc;
    int its[1] = {0};
    const int solve_rc =
        solve_bicg<1>(h, temperature_matrix(h), h->bs, h->h_b1, &h->g_bs, &h->l_bs, K_BICG1_INIT, K_BICG1_1, its);
    if (solve_rc == MC_ERR_CUDA) return solve_rc;
    CUDA_TRY(h, cudaMemcpyAsync(phi, h->xs, (size_t)h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (type == SC_TERBTE || type == SC_TERBED) {
        ClipArgs c{};
        c.phi = phi;
        c.nbr = h->nbr;
        c.key = h->reordered ? h->d_cell_n2o : nullptr;
        c.o2n = h->reordered ? h->d_cell_o2n : nullptr;
        c.list = h->neg_list;
        c.count = h->neg_count;
        c.cap = kClipCap;
        launch(h, K_SCALAR_CLIP,
               [&] { k_scalar_negatives<<<krylov_grid(h->N), MCB_THREADS, 0, h->stream>>>(h->N, c); });
        launch(h, K_SCALAR_CLIP, [&] { k_scalar_clip<<<1, 1024, 0, h->stream>>>(h->N, c); });
    }
    rc = check_launch(h);
    if (rc) return rc;
    if (st) st->scalar_iters[slot] = its[0];
    return solve_rc;
}

// ------------------------------------------------------------------ create

// out[i] = in[idx[i]] for i < n, then `tail` values copied in place (the
// six boundary slots of a field).
__global__ void k_permute(int n, int tail, double *__restrict__ out, const double *__restrict__ in,
                          const int *__restrict__ idx)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + tail; i += gridDim.x * blockDim.x)
        out[i] = i < n ? in[idx[i]] : in[i];
}

void permute(mc_flow *h, double *out, const double *in, const int *idx, int n, int tail)
{
    launch(h, K_PERMUTE, [&] { k_permute<<<blocks_for(n + tail), MCB_THREADS, 0, h->stream>>>(n, tail, out, in, idx); });
}

int allocate(mc_flow *h)
{
    const size_t N = (size_t)h->N, F = (size_t)h->F, NB = N + 6;
    Arena &A = h->arena;
    const int G = krylov_grid(std::max(h->N, h->F));
    struct Item { void **p; size_t bytes; };
    std::vector<Item> items;
    auto add = [&](void *pp, size_t bytes) { items.push_back({(void **)pp, bytes}); };
    add(&h->fc0, F * 4); add(&h->fc1, F * 4);
    add(&h->nbr, 6 * N * 4); add(&h->sface, 6 * N * 4); add(&h->col, 6 * N * 4);
    add(&h->sown, N);
    add(&h->outlet_faces, std::max<size_t>(1, (size_t)h->margs.n_outlet) * 4);
    for (double **p : {&h->area, &h->lam, &h->rl, &h->Sx, &h->Sy, &h->Sz, &h->xf, &h->yf, &h->zf}) add(p, F * 8);
    for (double **p : {&h->xc, &h->yc, &h->zc, &h->vol, &h->rho}) add(p, N * 8);
    for (int g = 0; g < G_NFIELDS; g++) {
        add(&h->phi[g], NB * 8);
        for (int d = 0; d < 3; d++) add(&h->grad[g][d], N * 8);
    }
    for (double **p : {&h->mdot, &h->ff0, &h->ff1, &h->fcorr}) add(p, F * 8);
    add(&h->AU, N * 8); add(&h->off_m, 6 * N * 8); add(&h->b_m, 3 * N * 8);
    add(&h->off_p, 6 * N * 8); add(&h->diag_p, N * 8); add(&h->b_p, N * 8);
    add(&h->off_t, 6 * N * 8); add(&h->diag_t, N * 8); add(&h->b_t, N * 8);
    add(&h->src, 5 * N * 8);
    add(&h->partials, (size_t)G * 8 * 8 * 3);  // split BiCGStab launches use 3 x the blocks
    add(&h->counter, 256);
    add(&h->balance, sizeof(FluxBalance));
    add(&h->scalars, 8 * 8);
    // PCG
    add(&h->pv.r, N * 8); add(&h->pv.zp[0], N * 16); add(&h->pv.zp[1], N * 16);
    add(&h->pv.q, N * 8); add(&h->pv.st, sizeof(PcgState));
    // BiCGStab, three right-hand sides; the single-RHS solver shares the vectors
    double *bic[8];
    for (int k = 0; k < 8; k++) add(&bic[k], 3 * N * 8);
    add(&h->b3.st, sizeof(BicgState<3>));
    add(&h->b1.st, sizeof(BicgState<1>));
    add(&h->pp_prev, N * 8);
    add(&h->dcode, N * 4);
    add(&h->gs, sizeof(GuessState));
    if (h->reordered) {
        add(&h->d_cell_n2o, N * 4);
        add(&h->d_cell_o2n, N * 4);
        add(&h->d_face_o2n, F * 4);
        add(&h->stage, std::max(F, NB) * 8);
    }
    size_t total = 0;
    std::vector<size_t> offs;
    for (auto &it : items) offs.push_back(A.reserve(it.bytes));
    total = A.used;
    cudaError_t e = cudaMalloc((void **)&A.base, total);
    if (e != cudaSuccess) return fail(h, MC_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    A.size = total;
    for (size_t i = 0; i < items.size(); i++) *items[i].p = A.base + offs[i];
    CUDA_TRY(h, cudaMemsetAsync(A.base, 0, total, h->stream));
    h->pv.partials = h->partials;
    h->pv.counter = h->counter;
    h->b3.partials = h->b1.partials = h->partials;
    h->b3.counter = h->b1.counter = h->counter;
    h->b3.r = bic[0]; h->b3.r0 = bic[1]; h->b3.p[0] = bic[2]; h->b3.p[1] = bic[3];
    h->b3.v[0] = bic[4]; h->b3.v[1] = bic[5]; h->b3.s = bic[6]; h->b3.t = bic[7];
    h->b1.r = bic[0]; h->b1.r0 = bic[1]; h->b1.p[0] = bic[2]; h->b1.p[1] = bic[3];
    h->b1.v[0] = bic[4]; h->b1.v[1] = bic[5]; h->b1.s = bic[6]; h->b1.t = bic[7];
    h->b3.b = h->b_m;
    h->b3.x[0] = h->phi[G_U];
    h->b3.x[1] = h->phi[G_V];
    h->b3.x[2] = h->phi[G_W];
    h->b1.b = h->b_t;
    h->b1.x[0] = h->phi[G_T];
    h->pv.b = h->b_p;
    h->pv.x = h->phi[G_PP];
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_pcg, sizeof(PcgState)));
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_b3, sizeof(BicgState<3>)));
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_b1, sizeof(BicgState<1>)));
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_scalars, 8 * sizeof(double)));
    return MC_OK;
}

template <typename T>
int upload(mc_flow *h, T *dst, const T *src, size_t n)
{
    CUDA_TRY(h, cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    return MC_OK;
}

// Split [n][3] host data into three device arrays.
int upload3(mc_flow *h, double *x, double *y, double *z, const std::vector<double> &v, size_t n)
{
    std::vector<double> tmp(n);
    double *dst[3] = {x, y, z};
    for (int d = 0; d < 3; d++) {
        for (size_t i = 0; i < n; i++) tmp[i] = v[3 * i + d];
        CUDA_TRY(h, cudaMemcpy(dst[d], tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    }
    return MC_OK;
}

// Initial state of the FlowSolver constructor (FlowSolver.hpp:315-327 interior,
// :403-471 boundary slots).
int initial_fields(mc_flow *h, const int btype[6])
{
    const size_t NB = (size_t)h->N + 6;
    std::vector<double> v(NB);
    auto put = [&](int g, double interior, double inlet, double outlet, double wall) -> int {
        std::fill(v.begin(), v.begin() + h->N, interior);
        for (int s = 0; s < 6; s++) v[h->N + s] = btype[s] == INLET ? inlet : (btype[s] == OUTLET ? outlet : wall);
        CUDA_TRY(h, cudaMemcpy(h->phi[g], v.data(), NB * sizeof(double), cudaMemcpyHostToDevice));
        return MC_OK;
    };
    const mc_flow_params &p = h->prm;
    int rc = put(G_U, p.inlet_u, p.inlet_u, p.inlet_u, 0.0);
    rc = rc ? rc : put(G_V, 0.0, 0.0, 0.0, 0.0);
    rc = rc ? rc : put(G_W, 0.0, 0.0, 0.0, 0.0);
    rc = rc ? rc : put(G_P, p.pressure0, p.pressure0, p.pressure0, p.pressure0);
    rc = rc ? rc : put(G_PP, 0.0, 0.0, 0.0, 0.0);
    rc = rc ? rc : put(G_T, p.temperature0, p.temperature0, p.temperature0, p.temperature0);
    if (rc || !h->has_scalars) return rc;
    // the other scalars (FlowSolver.hpp:320-327 interior; :411-469 boundary
    // slots by type: inlet k and epsilon from the inlet speed)
    auto put_field = [&](int field, double interior, double inlet, double outlet, double wall) -> int {
        std::fill(v.begin(), v.begin() + h->N, interior);
        for (int s = 0; s < 6; s++) v[h->N + s] = btype[s] == INLET ? inlet : (btype[s] == OUTLET ? outlet : wall);
        CUDA_TRY(h, cudaMemcpy(h->sfield[field], v.data(), NB * sizeof(double), cudaMemcpyHostToDevice));
        return MC_OK;
    };
    const double te_in = h->ph.sc_inlet[SC_TERBTE], ed_in = h->ph.sc_inlet[SC_TERBED];
    rc = put_field(MC_FIELD_TE, 0.0001, te_in, 0.0001, 0.0001);
    rc = rc ? rc : put_field(MC_FIELD_ED, 0.0, ed_in, 0.0, 0.0);
    rc = rc ? rc : put_field(MC_FIELD_TP, 0.0, 0.0, 0.0, 0.0);
    rc = rc ? rc : put_field(MC_FIELD_FUL, 0.1, 0.1, 0.1, 0.0);
    rc = rc ? rc : put_field(MC_FIELD_PRO, 0.001, 0.0, 0.001, 0.0);
    rc = rc ? rc : put_field(MC_FIELD_VARF, 0.1, 0.1, 0.1, 0.0);
    rc = rc ? rc : put_field(MC_FIELD_VARP, 0.001, 0.0, 0.001, 0.0);
    return rc;
}

// Device storage of the other scalar transports: seven fields, eighteen
// gradient components, the solve's solution vector and the negative-cell list.
int setup_scalars(mc_flow *h)
{
    const size_t N = (size_t)h->N, NB = N + 6;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t bytes = 7 * al(NB * 8) + 18 * al(N * 8) + al(N * 8) + al(kClipCap * 4) + 256;
    CUDA_TRY(h, cudaMalloc((void **)&h->scal_mem, bytes));
    CUDA_TRY(h, cudaMemsetAsync(h->scal_mem, 0, bytes, h->stream));
    char *p = h->scal_mem;
    for (int f : kScalarFields) {
        h->sfield[f] = (double *)p;
        p += al(NB * 8);
        if (f == MC_FIELD_TP) continue;
        for (int d = 0; d < 3; d++) {
            h->sgrad[f][d] = (double *)p;
            p += al(N * 8);
        }
    }
    h->xs = (double *)p;
    p += al(N * 8);
    h->neg_list = (int *)p;
    p += al(kClipCap * 4);
    h->neg_count = (unsigned int *)p;
    h->bs = h->b1;
    h->bs.x[0] = h->xs;
    return MC_OK;
}

// FP32-refined momentum and temperature solves: FP32 matrix copies, the
// inner BiCGStab vectors (shared by the two solves, which never overlap) and
// the refinement state, in one device allocation.
int setup_bicg_refined(mc_flow *h)
{
    const size_t N = (size_t)h->N;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t m7 = al(7 * N * 4), v3 = al(3 * N * 4);
    const size_t total = 2 * m7 + 11 * v3 + 4 * al(512);
    const cudaError_t e = cudaMalloc((void **)&h->bir_mem, total);
    if (e != cudaSuccess) return fail(h, MC_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    CUDA_TRY(h, cudaMemset(h->bir_mem, 0, total));
    char *c = h->bir_mem;
    auto take = [&](size_t b) { char *p = c; c += b; return p; };
    h->m32_diag = reinterpret_cast<float *>(take(m7));
    h->m32_off = h->m32_diag + N;
    h->t32_diag = reinterpret_cast<float *>(take(m7));
    h->t32_off = h->t32_diag + N;
    float *vec[11];
    for (int k = 0; k < 11; k++) vec[k] = reinterpret_cast<float *>(take(v3));
    BicgState<3> *st3 = reinterpret_cast<BicgState<3> *>(take(al(512)));
    BicgState<1> *st1 = reinterpret_cast<BicgState<1> *>(take(al(512)));
    BirState<3> *bo3 = reinterpret_cast<BirState<3> *>(take(al(512)));
    BirState<1> *bo1 = reinterpret_cast<BirState<1> *>(take(al(512)));
    // vec: 0 e (inner solution), 1 r32 (inner right-hand side), 2 r, 3 r0, 4-5 p, 6-7 v, 8 s, 9 t
    for (int j = 0; j < 3; j++) h->bi3.x[j] = vec[0] + j * N;
    h->bi3.b = vec[1];
    h->bi3.r = vec[2];
    h->bi3.r0 = vec[3];
    h->bi3.p[0] = vec[4];
    h->bi3.p[1] = vec[5];
    h->bi3.v[0] = vec[6];
    h->bi3.v[1] = vec[7];
    h->bi3.s = vec[8];
    h->bi3.t = vec[9];
    h->bi3.partials = h->partials;
    h->bi3.counter = h->counter;
    h->bi3.st = st3;
    h->bi1.x[0] = vec[0];
    h->bi1.b = vec[1];
    h->bi1.r = vec[2];
    h->bi1.r0 = vec[3];
    h->bi1.p[0] = vec[4];
    h->bi1.p[1] = vec[5];
    h->bi1.v[0] = vec[6];
    h->bi1.v[1] = vec[7];
    h->bi1.s = vec[8];
    h->bi1.t = vec[9];
    h->bi1.partials = h->partials;
    h->bi1.counter = h->counter;
    h->bi1.st = st1;
    h->bo3 = BirVectors<3>{{h->phi[G_U], h->phi[G_V], h->phi[G_W]}, h->b_m, vec[1], vec[0], h->partials, h->counter,
                           bo3};
    h->bo1 = BirVectors<1>{{h->phi[G_T]}, h->b_t, vec[1], vec[0], h->partials, h->counter, bo1};
    if (h->line_ex > 0) {
        // the FP32 copies are stored by direction: slot d holds direction d
        LineSystem L;
        L.N = h->N;
        L.ex = h->line_ex;
        int q = 0;
        for (int d = 0; d < 6; d++) {
            if (h->dc.doff[d] == -1)
                L.dxm = d;
            else if (h->dc.doff[d] == 1)
                L.dxp = d;
            else {
                L.yz[q] = d;
                L.yzoff[q] = h->dc.doff[d];
                q++;
            }
        }
        h->line3 = L;
        h->line3.d = h->m32_diag;
        h->line3.off = h->m32_off;
        h->line1 = L;
        h->line1.d = h->t32_diag;
        h->line1.off = h->t32_off;
        h->line_scratch = vec[2];  // the inner BiCGStab's r, unused by the line solver
    }
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_bi3, sizeof(BicgState<3>)));
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_bi1, sizeof(BicgState<1>)));
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_bo3, sizeof(BirState<3>)));
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_bo1, sizeof(BirState<1>)));
    return MC_OK;
}

// Guess state (pinned copy) and, for MC_GUESS_LEARNED, the network's graph,
// parameters and inference scratch in one device allocation.
int setup_guess(mc_flow *h, const HostMesh &hm)
{
    CUDA_TRY(h, cudaMallocHost((void **)&h->h_gs, sizeof(GuessState)));
    memset(h->h_gs, 0, sizeof(GuessState));
    if (h->prm.initial_guess != MC_GUESS_LEARNED) return MC_OK;
    std::vector<int> col;
    std::vector<uint32_t> edge;
    std::vector<float> vhat;
    std::vector<uint8_t> mask;
    GnnGraph aff{};
    gnn_graph_host(hm, col, edge, vhat, aff, mask);
    const size_t N = (size_t)hm.N;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t eb = al(6 * N * 4), vb = al(N * 4), xb = al(N * 8), pb = al((size_t)GNN_NPARAM * 4),
                 kb = al((size_t)GNN_NPACK * 2), wb = gnn_work_bytes(hm.N, false), mb = al(mask.size()),
                 cb = al(6 * N * 4);
    const cudaError_t e = cudaMalloc((void **)&h->gnn_mem, eb + vb + xb + pb + kb + wb + mb + cb);
    if (e != cudaSuccess) return fail(h, MC_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    char *c = h->gnn_mem;
    CUDA_TRY(h, cudaMemcpy(c, edge.data(), 6 * N * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(c + eb, vhat.data(), N * 4, cudaMemcpyHostToDevice));
    int *dcol = reinterpret_cast<int *>(c + eb + vb + xb + pb + kb + wb + mb);
    CUDA_TRY(h, cudaMemcpy(dcol, col.data(), 6 * N * 4, cudaMemcpyHostToDevice));
    h->gnn_g.n = hm.N;
    h->gnn_g.col = dcol;
    h->gnn_g.edge = reinterpret_cast<const __nv_bfloat162 *>(c);
    h->gnn_g.vhat = reinterpret_cast<const float *>(c + eb);
    h->x0_learned = reinterpret_cast<double *>(c + eb + vb);
    h->gnn_p = reinterpret_cast<float *>(c + eb + vb + xb);
    h->gnn_pk = reinterpret_cast<__nv_bfloat16 *>(c + eb + vb + xb + pb);
    CUDA_TRY(h, cudaMemset(c + eb + vb + xb + pb + kb, 0, wb));
    gnn_work_carve(h->gnn_w, c + eb + vb + xb + pb + kb, hm.N, false);
    h->gnn_g.affine = aff.affine;
    for (int k = 0; k < 6; k++) {
        h->gnn_g.doff[k] = aff.doff[k];
        h->gnn_g.ebits[k] = aff.ebits[k];
    }
    h->gnn_g.mask = nullptr;
    if (aff.affine) {
        uint8_t *md = reinterpret_cast<uint8_t *>(c + eb + vb + xb + pb + kb + wb);
        CUDA_TRY(h, cudaMemcpy(md, mask.data(), mask.size(), cudaMemcpyHostToDevice));
        h->gnn_g.mask = md;
    }
    return MC_OK;
}

// MC_DIR_CODES=0 keeps the column lists even where direction codes apply
// (the tests use it to check both forms).
// Length of the x-lines when the rows form them: the -x and +x neighbours
// are row -/+ 1 (direction codes), every row at a multiple of ex lacks a -x
// neighbour and every other row has one, and likewise for +x at the line
// ends; 0 otherwise (or when a line would not fit one thread block).
int x_line_length(const std::vector<uint32_t> &code, const int doff[6], int N)
{
    int dxm = -1, dxp = -1, ex = 0;
    for (int d = 0; d < 6; d++) {
        if (doff[d] == -1) dxm = d;
        if (doff[d] == 1) dxp = d;
    }
    for (int d = 0; d < 6; d++)
        if (doff[d] > 1 && (ex == 0 || doff[d] < ex)) ex = doff[d];
    if (dxm < 0 || dxp < 0 || ex < 2 || ex > 1024 || N % ex != 0) return 0;
    for (int i = 0; i < N; i++) {
        bool m = false, p = false;
        for (int k = 0; k < 6; k++) {
            const unsigned d = (code[i] >> (3 * k)) & 7u;
            m = m || d == (unsigned)dxm;
            p = p || d == (unsigned)dxp;
        }
        if (m != (i % ex != 0) || p != (i % ex != ex - 1)) return 0;
    }
    return ex;
}

// Form of the pressure solvers' FP64 copy: 1 (default) the half form of the
// symmetric matrix, 2 all six directions, 0 none (the slot-order matrix);
// MC_PRESSURE_COPY overrides.  The FP32 level 0 keeps all six directions.
int pressure_copy_form()
{
    const char *v = std::getenv("MC_PRESSURE_COPY");
    return (v && *v) ? std::atoi(v) : 1;
}

bool dir_codes_disabled()
{
    const char *v = std::getenv("MC_DIR_CODES");
    return v && v[0] == '0';
}

bool amg_half_disabled()
{
    const char *v = std::getenv("MC_AMG_HALF");
    return v && v[0] == '0';
}

bool row_store_disabled()
{
    const char *v = std::getenv("MC_ROW_STORE");
    return v && v[0] == '0';
}

// Positions of the six directions in rows stored by direction (RowStore):
// an order in which the directions occur in the slots of every row, so that
// a row summed by position sums its terms in slot order.  False when the
// rows disagree (no such order).
bool row_direction_order(const std::vector<uint32_t> &code, uint32_t &pos)
{
    bool before[6][6] = {};
    std::unordered_map<uint32_t, int> seen;
    for (uint32_t cw : code) {
        if (seen.count(cw)) continue;
        seen[cw] = 1;
        int last[6], n = 0;
        for (int k = 0; k < 6; k++) {
            const unsigned d = (cw >> (3 * k)) & 7u;
            if (d < 6) last[n++] = (int)d;
        }
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++) before[last[a]][last[b]] = true;
    }
    bool placed[6] = {};
    pos = 0;
    for (int q = 0; q < 6; q++) {  // Kahn's order, ties by direction index
        int pick = -1;
        for (int d = 0; d < 6 && pick < 0; d++) {
            if (placed[d]) continue;
            bool free = true;
            for (int e = 0; e < 6; e++)
                if (!placed[e] && e != d && before[e][d]) free = false;
            if (free) pick = d;
        }
        if (pick < 0) return false;  // a cycle: the rows disagree
        placed[pick] = true;
        pos |= (uint32_t)q << (3 * pick);
    }
    return true;
}

// Direction codes of the ELL columns (DirCodes): slot k of row i holds the
// direction d with nbr[d][i] == col[k][i] (7: unused slot).  Returns false
// when some direction's neighbour offset is not the same for every row (RCM
// order, irregular meshes): the kernels then read the column list.
bool build_dir_codes(const HostMesh &hm, std::vector<uint32_t> &code, int doff[6])
{
    const int N = hm.N;
    bool seen[6] = {false, false, false, false, false, false};
    for (int d = 0; d < 6; d++) doff[d] = 0;
    code.assign(N, 0u);
    for (int i = 0; i < N; i++) {
        uint32_t cw = 0;
        for (int k = 0; k < 6; k++) {
            const int j = hm.col[(size_t)k * N + i];
            unsigned dsel = 7;
            if (j != i) {
                for (int d = 0; d < 6; d++)
                    if (hm.nbr[(size_t)d * N + i] == j) {
                        dsel = (unsigned)d;
                        break;
                    }
                if (dsel == 7) return false;
                if (!seen[dsel]) {
                    seen[dsel] = true;
                    doff[dsel] = j - i;
                } else if (doff[dsel] != j - i) {
                    return false;
                }
            }
            cw |= dsel << (3 * k);
        }
        code[i] = cw;
    }
    return true;
}

// Aggregation hierarchy for the pressure-correction system: pattern data on
// the host (amg.cu), one extra device allocation for all levels.
int build_amg(mc_flow *h, const HostMesh &hm)
{
    const int N = hm.N;
    std::vector<int> dn((size_t)6 * N);
    for (size_t i = 0; i < dn.size(); i++) dn[i] = hm.nbr[i] >= 0 ? hm.nbr[i] : -1;
    std::vector<AmgHostLevel> lv;
    std::string err;
    if (amg_build_host(N, hm.col, dn, lv, err) != 0) return fail(h, MC_ERR_MESH, err);
    const int L = (int)lv.size();
    if (L < 2) {  // the whole system is already at the coarsest size: plain Jacobi PCG
        h->use_amg = false;
        return MC_OK;
    }
    Arena ar;
    struct Item { void **p; size_t bytes; };
    std::vector<Item> items;
    auto add = [&](void *pp, size_t bytes) { items.push_back({(void **)pp, std::max<size_t>(bytes, 8)}); };
    AmgHierarchy &H = h->amg;
    H.levels = L;
    for (int l = 0; l < L; l++) H.lv[l].n = lv[l].n;
    amg_plan_fused(H);
    H.sweeps = h->prm.amg_sweeps;
    H.omega = h->prm.amg_omega;
    amg_set_damping(H, h->prm.amg_cheb_ratio);
    H.alpha = h->prm.amg_alpha;
    std::vector<int *> d_col(L), d_agg(L), d_mptr(L), d_mlist(L), d_gptr(L), d_gidx(L);
    for (int l = 0; l < L; l++) {
        const AmgHostLevel &a = lv[l];
        AmgLevel &d = H.lv[l];
        d.n = a.n;
        d.k = a.k;
        if (l > 0) {
            add(&d.diag, (size_t)a.n * 8);
            add(&d.off, (size_t)a.k * a.n * 8);
            add(&d_col[l], a.col.size() * 4);
            add(&d.r, (size_t)a.n * 8);
            add(&d_gptr[l], a.gptr.size() * 4);
            add(&d_gidx[l], a.gidx.size() * 4);
        }
        add(&d.e[0], (size_t)a.n * 8);
        add(&d.e[1], (size_t)a.n * 8);
        if (l + 1 < L) {
            add(&d_agg[l], a.agg.size() * 4);
            add(&d_mptr[l], a.mptr.size() * 4);
            add(&d_mlist[l], a.mlist.size() * 4);
        }
    }
    const int nc = lv[L - 1].n;
    add(&H.dense, (size_t)nc * nc * 8);
    add(&H.dense_next, (size_t)nc * nc * 8);
    const bool fp32 = h->prm.precision == MC_PRECISION_FP32_REFINED;
    PcgState *inner_state = nullptr;
    // the FP16 copy of the FP32 level 0 (values by direction) for the V-cycle
    const bool half0 = fp32 && h->dc.code && !amg_half_disabled();
    if (fp32) {
        for (int l = 0; l < L; l++) {
            AmgLevelT<float> &f = H.lv32[l];
            add(&f.diag, (size_t)lv[l].n * 4);
            add(&f.off, (size_t)lv[l].k * lv[l].n * 4);
            add(&f.r, (size_t)lv[l].n * 4);
            add(&f.e[0], (size_t)lv[l].n * 4);
            add(&f.e[1], (size_t)lv[l].n * 4);
            if (l == 0 && half0) {
                add(&f.off16, (size_t)6 * lv[l].n * 2);
                add(&f.scale16, 2 * sizeof(float));
            }
        }
        add(&h->pv32.x, (size_t)N * 4);
        add(&h->pv32.r, (size_t)N * 4);
        add(&h->pv32.q, (size_t)N * 4);
        add(&h->pv32.zp[0], (size_t)N * 8);
        add(&h->pv32.zp[1], (size_t)N * 8);
        add(&h->r32, (size_t)N * 4);
        add(&h->ir_x2, (size_t)N * 8);
        add(&inner_state, sizeof(PcgState));
    }
    std::vector<size_t> offs;
    for (auto &it : items) offs.push_back(ar.reserve(it.bytes));
    cudaError_t e = cudaMalloc((void **)&h->amg_mem, ar.used);
    if (e != cudaSuccess) return fail(h, MC_ERR_NOMEM, std::string("cudaMalloc (AMG): ") + cudaGetErrorString(e));
    CUDA_TRY(h, cudaMemset(h->amg_mem, 0, ar.used));
    for (size_t i = 0; i < items.size(); i++) *items[i].p = h->amg_mem + offs[i];
    auto put = [&](int *dst, const std::vector<int> &src) -> int {
        if (!src.empty()) CUDA_TRY(h, cudaMemcpy(dst, src.data(), src.size() * 4, cudaMemcpyHostToDevice));
        return MC_OK;
    };
    for (int l = 0; l < L; l++) {
        AmgLevel &d = H.lv[l];
        if (l == 0) {
            d.diag = h->diag_p;
            d.off = h->p_dir64 ? h->p_dir64 : h->off_p;
            d.col = h->col;
            d.dc = h->p_dir64 ? h->dc_pdir : h->dc;
            d.r = h->pv.r;
        } else {
            int rc = put(d_col[l], lv[l].col);
            rc = rc ? rc : put(d_gptr[l], lv[l].gptr);
            rc = rc ? rc : put(d_gidx[l], lv[l].gidx);
            if (rc) return rc;
            d.col = d_col[l];
            d.gptr = d_gptr[l];
            d.gidx = d_gidx[l];
            d.dc = DirCodes{};
            if (lv[l].dia) {  // values in direction order: the kernels compute the columns
                d.dc.dia = 1;
                for (int q = 0; q < 6; q++) d.dc.doff[q] = lv[l].doff[q];
            }
        }
        if (l + 1 < L) {
            int rc = put(d_agg[l], lv[l].agg);
            rc = rc ? rc : put(d_mptr[l], lv[l].mptr);
            rc = rc ? rc : put(d_mlist[l], lv[l].mlist);
            if (rc) return rc;
            d.agg = d_agg[l];
            d.mptr = d_mptr[l];
            d.mlist = d_mlist[l];
        }
    }
    H.g0 = H.lv[0];  // the slot-order level 0 (Galerkin lists, FP32 rounding)
    H.g0.off = h->off_p;
    H.g0.dc = h->dc;
    if (fp32) {
        for (int l = 0; l < L; l++) {
            AmgLevelT<float> &f = H.lv32[l];
            const AmgLevelT<double> &d = H.lv[l];
            f.n = d.n;
            f.k = d.k;
            f.col = d.col;
            f.dc = l == 0 ? by_direction(h->dc) : d.dc;  // FP32 level 0 values are stored by direction
            f.agg = d.agg;
            f.mptr = d.mptr;
            f.mlist = d.mlist;
            f.gptr = d.gptr;
            f.gidx = d.gidx;
        }
        h->pv32.b = h->r32;
        h->pv32.partials = h->partials;
        h->pv32.counter = h->counter;
        h->pv32.st = inner_state;
        CUDA_TRY(h, cudaMallocHost((void **)&h->h_pcg_inner, sizeof(PcgState)));
        H.has32 = true;
        h->refined = true;
    }
    h->use_amg = true;
    return MC_OK;
}

} // namespace

// =================================================================== C ABI

extern "C" {

void mc_flow_default_params(mc_flow_params *p, int mode)
{
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->mode = mode;
    p->delta = 1.0e-5;
    p->density = 1.2;
    p->inlet_u = 50.0;
    p->pressure0 = 4000.0;
    p->flux_corr = 0.8;
    p->urf_temperature = 0.95;
    p->max_iters = 10000;
    p->pressure_solver = MC_PSOLVER_PCG_JACOBI;
    p->precision = MC_PRECISION_FP64;
    p->initial_guess = MC_GUESS_ZERO;
    p->amg_sweeps = 3;
    p->amg_omega = 0.6667;
    p->amg_alpha = 2.0;
    p->ir_inner_rtol = 1e-5;
    p->ir_inner_rtol_bicg = 1e-4;
    p->amg_cheb_ratio = 4.0;
    p->reorder = MC_REORDER_NONE;
    p->transport_scalars = mode == MC_MODE_COMPAT ? 1 : 0;
    p->ir_line_steps = 2;
    if (mode == MC_MODE_COMPAT) {
        p->viscosity = 0.000014;
        p->temperature0 = 2000.0;
        p->urf_momentum = 0.5;
        p->urf_pressure = 0.2;
        p->u_rtol = 1e-13;
        p->p_rtol = 1e-13;
    } else {
        p->viscosity = 1.8e-5;
        p->temperature0 = 1500.0;
        p->urf_momentum = 0.7;
        p->urf_pressure = 0.3;
        p->u_rtol = 1e-8;
        p->p_rtol = 1e-8;
    }
}

int mc_flow_create(const mc_mesh_view *mesh, const mc_flow_params *params, mc_flow **out)
{
    if (!mesh || !params || !out) return MC_ERR_ARG;
    *out = nullptr;
    if (params->mode != MC_MODE_COMPAT && params->mode != MC_MODE_SIMPLE) return MC_ERR_ARG;
    if ((params->pressure_solver != MC_PSOLVER_PCG_JACOBI && params->pressure_solver != MC_PSOLVER_PCG_AMG) ||
        (params->precision != MC_PRECISION_FP64 && params->precision != MC_PRECISION_FP32_REFINED))
        return MC_ERR_UNSUPPORTED;
    if (params->initial_guess != MC_GUESS_ZERO && params->initial_guess != MC_GUESS_PREVIOUS &&
        params->initial_guess != MC_GUESS_LEARNED)
        return MC_ERR_ARG;
    if (params->reorder != MC_REORDER_NONE && params->reorder != MC_REORDER_RCM) return MC_ERR_ARG;
    if (params->precision == MC_PRECISION_FP32_REFINED &&
        (params->pressure_solver != MC_PSOLVER_PCG_AMG || !(params->ir_inner_rtol > 0) || params->ir_inner_rtol >= 1 ||
         !(params->ir_inner_rtol_bicg > 0) || params->ir_inner_rtol_bicg >= 1))
        return MC_ERR_UNSUPPORTED;
    if (params->pressure_solver == MC_PSOLVER_PCG_AMG &&
        (params->amg_sweeps < 1 || params->amg_sweeps > AMG_MAX_SWEEPS || !(params->amg_omega > 0) ||
         !(params->amg_alpha > 0) || !(params->amg_cheb_ratio == 0 || params->amg_cheb_ratio > 1)))
        return MC_ERR_ARG;
    if (params->ir_line_steps < 0 || params->ir_line_steps > 8) return MC_ERR_ARG;
    if (!(params->delta > 0) || !(params->urf_momentum > 0) || !(params->urf_temperature > 0) ||
        !(params->u_rtol > 0) || !(params->p_rtol > 0) || params->max_iters <= 0)
        return MC_ERR_ARG;
    mc_flow *h = new (std::nothrow) mc_flow();
    if (!h) return MC_ERR_NOMEM;
    h->prm = *params;
    int rc = MC_OK;
    {
        HostMesh hm;
        std::string err;
        HostPhysics hp{params->density};
        rc = build_host_mesh(mesh, hp, hm, err);
        if (!rc) {
            // the nodes, kept for the flow/particle exchange
            const uint64_t P64 = mesh->points;
            if (P64 == 0 || P64 >= (uint64_t)INT32_MAX) {
                err = "points out of range";
                rc = MC_ERR_MESH;
            } else {
                h->P = (int)P64;
                h->h_points.assign(mesh->points_xyz, mesh->points_xyz + 3 * P64);
                h->h_cell_nodes.resize((size_t)8 * mesh->cells);
                for (size_t i = 0; i < (size_t)8 * mesh->cells && !rc; i++) {
                    if (mesh->cell_nodes[i] >= P64) {
                        err = "cell_nodes refers to a point that does not exist";
                        rc = MC_ERR_MESH;
                    }
                    h->h_cell_nodes[i] = (int)mesh->cell_nodes[i];
                }
            }
        }
        if (!rc && params->reorder == MC_REORDER_RCM) {
            std::vector<int> face_n2o;
            rcm_cell_order(hm, h->cell_n2o);
            rc = apply_reorder(hm, h->cell_n2o, face_n2o, err);
            if (!rc) {
                h->reordered = true;
                h->cell_o2n.assign(hm.N, 0);
                for (int n = 0; n < hm.N; n++) h->cell_o2n[h->cell_n2o[n]] = n;
                h->face_o2n.assign(hm.F, 0);
                for (int n = 0; n < hm.F; n++) h->face_o2n[face_n2o[n]] = n;
            }
        }
        if (rc) {
            h->err = err;
            mc_flow_destroy(h);
            return rc;
        }
        cudaError_t e = cudaSetDevice(params->device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_levels, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_inverse, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            mc_flow_destroy(h);
            return MC_ERR_CUDA;
        }
        h->dev = params->device;
        h->N = hm.N;
        h->F = hm.F;
        h->margs.n_outlet = (int)hm.outlet_faces.size();
        rc = allocate(h);
        if (!rc) {
            const size_t N = hm.N, F = hm.F;
            rc = upload(h, h->fc0, hm.fc0.data(), F);
            rc = rc ? rc : upload(h, h->fc1, hm.fc1.data(), F);
            rc = rc ? rc : upload(h, h->nbr, hm.nbr.data(), 6 * N);
            rc = rc ? rc : upload(h, h->sface, hm.sface.data(), 6 * N);
            rc = rc ? rc : upload(h, h->col, hm.col.data(), 6 * N);
            // kept until the stream synchronisation below
            std::vector<uint8_t> own(N, 0);
            for (size_t c = 0; c < N; c++)
                for (int k = 0; k < 6; k++)
                    if (hm.fc0[hm.sface[(size_t)k * N + c]] == (int)c) own[c] |= (uint8_t)(1u << k);
            rc = rc ? rc : upload(h, h->sown, own.data(), N);
            if (!rc && !hm.outlet_faces.empty()) rc = upload(h, h->outlet_faces, hm.outlet_faces.data(), hm.outlet_faces.size());
            rc = rc ? rc : upload(h, h->area, hm.area.data(), F);
            rc = rc ? rc : upload(h, h->lam, hm.lam.data(), F);
            rc = rc ? rc : upload(h, h->rl, hm.rl.data(), F);
            rc = rc ? rc : upload(h, h->vol, hm.vol.data(), N);
            rc = rc ? rc : upload(h, h->rho, hm.rho.data(), N);
            if (!rc) cudaStreamSynchronize(h->stream);
            rc = rc ? rc : upload3(h, h->Sx, h->Sy, h->Sz, hm.S, F);
            rc = rc ? rc : upload3(h, h->xf, h->yf, h->zf, hm.xf, F);
            rc = rc ? rc : upload3(h, h->xc, h->yc, h->zc, hm.xc, N);
            if (!rc && h->reordered) {
                rc = upload(h, h->d_cell_n2o, h->cell_n2o.data(), N);
                rc = rc ? rc : upload(h, h->d_cell_o2n, h->cell_o2n.data(), N);
                rc = rc ? rc : upload(h, h->d_face_o2n, h->face_o2n.data(), F);
                if (!rc) cudaStreamSynchronize(h->stream);
            }
            if (!rc) {
                // inlet values of the scalars, as the reference computes them
                // (FlowSolver.inl:2625-2659; FlowSolver.hpp:421, 431-432)
                const double u = params->inlet_u;
                const double velmag2 = std::pow(u, 2) + std::pow(0.0, 2) + std::pow(0.0, 2);
                Physics &ph0 = h->ph;
                ph0.sc_inlet[SC_TERBTE] = 3.0 / 2.0 * ((0.1 * 0.1) * velmag2);
                ph0.sc_inlet[SC_TERBED] = std::pow(0.09, 0.75) * std::pow((3.0 / 2.0 * ((0.1 * 0.1) * velmag2)), 1.5);
                ph0.sc_inlet[SC_TEMP] = params->temperature0;
                ph0.sc_inlet[SC_FUEL] = 0.1;
                ph0.sc_inlet[SC_PROG] = 0.0;
                ph0.sc_inlet[SC_VARFU] = 0.1;
                ph0.sc_inlet[SC_VARPR] = 0.0;
                ph0.cmu75 = std::pow(0.09, 0.75);
                h->has_scalars = params->transport_scalars != 0;
                if (h->has_scalars) rc = setup_scalars(h);
            }
            rc = rc ? rc : initial_fields(h, hm.btype);
            if (!rc) {
                std::vector<uint32_t> code;
                int doff[6];
                if (build_dir_codes(hm, code, doff) && !dir_codes_disabled()) {
                    rc = upload(h, h->dcode, code.data(), N);
                    if (!rc) cudaStreamSynchronize(h->stream);
                    h->dc.code = h->dcode;
                    for (int d = 0; d < 6; d++) h->dc.doff[d] = doff[d];
                    // the most frequent code word and its per-slot offsets
                    std::unordered_map<uint32_t, int> freq;
                    for (uint32_t cw : code) freq[cw]++;
                    uint32_t canon = code[0];
                    for (const auto &f : freq)
                        if (f.second > freq[canon]) canon = f.first;
                    h->dc.canon = canon;
                    for (int k = 0; k < 6; k++) {
                        const unsigned d = (canon >> (3 * k)) & 7u;
                        h->dc.coff[k] = d < 6 ? doff[d] : 0;
                    }
                    h->line_ex = x_line_length(code, doff, (int)N);
                    uint32_t pos = 0;
                    if (!row_store_disabled() && row_direction_order(code, pos)) {
                        h->rows.code = h->dcode;
                        h->rows.pos = pos;
                        h->dc_rows = by_direction(h->dc);
                        for (int d = 0; d < 6; d++) h->dc_rows.doff[(pos >> (3 * d)) & 7u] = doff[d];
                        h->hcode.swap(code);
                    }
                }
            }
            const int form = pressure_copy_form();
            if (!rc && h->dc.code && form > 0 && (form == 2 || sym_applies(h->dc))) {
                // the solvers' by-direction copy of the pressure-correction matrix
                const bool sym = form != 2;
                const cudaError_t e =
                    cudaMalloc((void **)&h->p_dir64, (size_t)(sym ? 3 : 6) * N * sizeof(double));
                if (e != cudaSuccess) rc = fail(h, MC_ERR_NOMEM, "cudaMalloc (pressure copy)");
                else h->dc_pdir = sym ? by_direction_sym(h->dc) : by_direction(h->dc);
            }
            if (!rc && params->pressure_solver == MC_PSOLVER_PCG_AMG) rc = build_amg(h, hm);
            if (!rc) rc = setup_guess(h, hm);
            if (!rc && params->precision == MC_PRECISION_FP32_REFINED) rc = setup_bicg_refined(h);
        }
        if (!rc) {
            h->hcol.assign((size_t)6 * hm.N, -1);
            for (int k = 0; k < 6; k++)
                for (int c = 0; c < hm.N; c++) {
                    const int f = hm.sface[(size_t)k * hm.N + c];
                    if (hm.fc1[f] < hm.N) h->hcol[(size_t)k * hm.N + c] = hm.col[(size_t)k * hm.N + c];
                }
            Physics &ph = h->ph;
            ph.N = hm.N;
            ph.mode = params->mode;
            ph.cell0 = h->reordered ? h->cell_o2n[0] : 0;
            for (int s = 0; s < 6; s++) {
                ph.btype[s] = hm.btype[s];
                ph.last_bface[s] = hm.last_bface[s];
            }
            ph.mu = params->viscosity;
            ph.inlet_mu = inlet_effective_viscosity(params->viscosity, params->inlet_u);
            ph.u_in = params->inlet_u;
            ph.rho_in = params->density;
            ph.T_ref = params->temperature0;
            ph.rdelta = 1.0 / params->delta;
            ph.urf_u = params->urf_momentum;
            ph.urf_T = params->urf_temperature;
            ph.urf_p = params->urf_pressure;
            ph.flux_corr = params->flux_corr;
            MeshArgs &m = h->margs;
            m.F = hm.F;
            m.fc0 = h->fc0; m.fc1 = h->fc1; m.sface = h->sface; m.col = h->col; m.own = h->sown;
            m.area = h->area; m.lam = h->lam; m.rl = h->rl;
            m.Sx = h->Sx; m.Sy = h->Sy; m.Sz = h->Sz;
            m.xf = h->xf; m.yf = h->yf; m.zf = h->zf;
            m.xc = h->xc; m.yc = h->yc; m.zc = h->zc;
            m.vol = h->vol; m.rho = h->rho;
            m.outlet_faces = h->outlet_faces;
        }
    }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = fail(h, MC_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc) {
        mc_flow_destroy(h);
        return rc;
    }
    *out = h;
    return MC_OK;
}

int mc_flow_destroy(mc_flow *h)
{
    if (!h) return MC_ERR_ARG;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (cudaGraphExec_t g : {h->g_pcg, h->g_b3, h->g_b1, h->g_pcg_amg, h->g_pcg_amg32, h->g_b3_32, h->g_b1_32,
                              h->l_pcg, h->l_b3, h->l_b1, h->l_pcg_amg, h->l_pcg_amg32, h->l_b3_32, h->l_b1_32})
        if (g) cudaGraphExecDestroy(g);
    if (h->amg_mem) cudaFree(h->amg_mem);
    if (h->p_dir64) cudaFree(h->p_dir64);
    for (cudaEvent_t e : h->timing.ev) cudaEventDestroy(e);
    if (h->arena.base) cudaFree(h->arena.base);
    if (h->h_pcg) cudaFreeHost(h->h_pcg);
    if (h->h_b3) cudaFreeHost(h->h_b3);
    if (h->h_b1) cudaFreeHost(h->h_b1);
    if (h->h_scalars) cudaFreeHost(h->h_scalars);
    if (h->h_pcg_inner) cudaFreeHost(h->h_pcg_inner);
    if (h->snap) mc_flow_snapshot_close(h);
    if (h->h_gs) cudaFreeHost(h->h_gs);
    if (h->gnn_mem) cudaFree(h->gnn_mem);
    if (h->bir_mem) cudaFree(h->bir_mem);
    if (h->scal_mem) cudaFree(h->scal_mem);
    if (h->node_mem) cudaFree(h->node_mem);
    if (h->xin_mem) cudaFree(h->xin_mem);
    for (cudaGraphExec_t g : {h->g_bs, h->l_bs})
        if (g) cudaGraphExecDestroy(g);
    for (void *p : {(void *)h->h_bi3, (void *)h->h_bi1, (void *)h->h_bo3, (void *)h->h_bo1})
        if (p) cudaFreeHost(p);
    if (h->side) cudaStreamSynchronize(h->side);  // no inverse still being formed into freed memory
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ev_levels) cudaEventDestroy(h->ev_levels);
    if (h->ev_inverse) cudaEventDestroy(h->ev_inverse);
    delete h;
    return MC_OK;
}

int mc_flow_set_field(mc_flow *h, int field, const double *vals)
{
    if (!h || !vals) return MC_ERR_ARG;
    double *dst = field_ptr(h, field);
    if (!dst) return MC_ERR_UNSUPPORTED;
    const size_t NB = (size_t)h->N + 6;
    if (h->reordered) {
        CUDA_TRY(h, cudaMemcpyAsync(h->stage, vals, NB * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        permute(h, dst, h->stage, h->d_cell_n2o, h->N, 6);
    } else {
        CUDA_TRY(h, cudaMemcpyAsync(dst, vals, NB * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return MC_OK;
}

int mc_flow_get_field(mc_flow *h, int field, double *vals)
{
    if (!h || !vals) return MC_ERR_ARG;
    const double *src = field_ptr(h, field);
    if (!src) return MC_ERR_UNSUPPORTED;
    const size_t NB = (size_t)h->N + 6;
    if (h->reordered) {
        permute(h, h->stage, src, h->d_cell_o2n, h->N, 6);
        src = h->stage;
    }
    CUDA_TRY(h, cudaMemcpyAsync(vals, src, NB * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return MC_OK;
}

int mc_flow_set_guess_params(mc_flow *h, const float *params, int count)
{
    if (!h || !params || count != GNN_NPARAM) return MC_ERR_ARG;
    if (h->prm.initial_guess != MC_GUESS_LEARNED) return fail(h, MC_ERR_ARG, "initial_guess is not MC_GUESS_LEARNED");
    CUDA_TRY(h, cudaMemcpyAsync(h->gnn_p, params, (size_t)GNN_NPARAM * 4, cudaMemcpyHostToDevice, h->stream));
    gnn_pack(h->stream, h->gnn_p, h->gnn_pk);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->gnn_loaded = true;
    return MC_OK;
}

int mc_flow_snapshot_open(mc_flow *h, const char *path, int max_records)
{
    if (!h || !path || max_records <= 0) return MC_ERR_ARG;
    if (h->snap) mc_flow_snapshot_close(h);
    const size_t bytes = (size_t)4 * h->N * sizeof(float);
    if (!h->snap_mem) {
        CUDA_TRY(h, cudaMalloc((void **)&h->snap_mem, bytes));
        CUDA_TRY(h, cudaMallocHost((void **)&h->snap_host, bytes));
        h->snap_dev = reinterpret_cast<float *>(h->snap_mem);
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(h, MC_ERR_ARG, std::string("cannot open ") + path);
    unsigned char head[64] = {0};
    memcpy(head, "MCSNAP01", 8);
    const uint32_t meta[4] = {1u, (uint32_t)h->N, 4u, 0u};
    memcpy(head + 8, meta, sizeof(meta));
    if (std::fwrite(head, 1, 64, f) != 64) {
        std::fclose(f);
        return fail(h, MC_ERR_ARG, "snapshot header write failed");
    }
    h->snap = f;
    h->snap_max = max_records;
    h->snap_count = 0;
    return MC_OK;
}

int mc_flow_snapshot_close(mc_flow *h)
{
    if (!h) return MC_ERR_ARG;
    int rc = MC_OK;
    if (h->snap) {
        const uint64_t count = (uint64_t)h->snap_count;
        if (std::fseek(h->snap, 24, SEEK_SET) != 0 || std::fwrite(&count, 8, 1, h->snap) != 1) rc = MC_ERR_ARG;
        if (std::fclose(h->snap) != 0) rc = MC_ERR_ARG;
        h->snap = nullptr;
    }
    if (h->snap_mem) {
        cudaFree(h->snap_mem);
        cudaFreeHost(h->snap_host);
        h->snap_mem = nullptr;
        h->snap_host = nullptr;
        h->snap_dev = nullptr;
    }
    return rc;
}

// ------------------------------------------------------------- VTK output

namespace {

// A field in the caller's numbering (cells + 6 values).
int fetch_field(mc_flow *h, int field, std::vector<double> &out)
{
    out.resize((size_t)h->N + 6);
    return mc_flow_get_field(h, field, out.data());
}

// "x y z" as the reference's print_vec writes it (a fresh stream: default
// precision), utils.hpp:357-362.
std::string vec_text(double x, double y, double z)
{
    std::stringstream b;
    b << x << " " << y << " " << z;
    return b.str();
}

} // namespace

int mc_flow_write_vtk(mc_flow *h, const char *prefix, int id)
{
    if (!h || !prefix) return MC_ERR_ARG;
    const int N = h->N;
    static const int needed[] = {MC_FIELD_U, MC_FIELD_V, MC_FIELD_W, MC_FIELD_P, MC_FIELD_TE, MC_FIELD_ED,
                                 MC_FIELD_TEM, MC_FIELD_FUL, MC_FIELD_PRO, MC_FIELD_VARF, MC_FIELD_VARP};
    std::vector<double> f[MC_FIELD_VARP + 1];
    for (int k : needed) {
        if (!field_ptr(h, k)) {
            f[k].assign((size_t)N + 6, 0.0);  // not transported by this handle: written as zeros
            continue;
        }
        const int rc = fetch_field(h, k, f[k]);
        if (rc) return rc;
    }
    // cell centres in the caller's numbering
    std::vector<double> c[3];
    const double *dc[3] = {h->xc, h->yc, h->zc};
    std::vector<double> tmp((size_t)N);
    for (int d = 0; d < 3; d++) {
        CUDA_TRY(h, cudaMemcpy(tmp.data(), dc[d], (size_t)N * 8, cudaMemcpyDeviceToHost));
        c[d].resize((size_t)N);
        for (int i = 0; i < N; i++) c[d][i] = tmp[h->reordered ? h->cell_o2n[i] : i];
    }
    const std::string name = std::string(prefix) + "_flow0_timestep" + std::to_string(id) + ".vtk";
    std::ofstream v(name);
    if (!v) return fail(h, MC_ERR_ARG, "cannot open " + name);
    v << "# vtk DataFile Version 3.0 " << std::endl;
    v << "MiniCOMBUST " << std::endl;
    v << "ASCII " << std::endl;
    v << "DATASET POLYDATA " << std::endl;
    v << std::endl << "POINTS " << (uint64_t)N << " float" << std::endl;
    for (int i = 0; i < N; i++) {
        if (i % 10 == 0)
            v << std::endl;
        else
            v << "  ";
        v << vec_text(c[0][i], c[1][i], c[2][i]) << "\t";
    }
    v << std::endl << std::endl;
    v << std::endl << "VERTICES " << (uint64_t)N << " " << (uint64_t)N * 2 << std::endl;
    for (uint64_t i = 0; i < (uint64_t)N; i++) v << "1 " << i << "\t";
    v << std::endl;
    v << std::endl << "POINT_DATA " << (uint64_t)N << std::endl;
    v << "VECTORS flow_velocity float" << std::endl;
    for (int i = 0; i < N; i++) v << f[MC_FIELD_U][i] << " " << f[MC_FIELD_V][i] << " " << f[MC_FIELD_W][i] << " " << "\t";
    v << std::endl;
    // the scalar blocks in the reference's order and labels (the ones labelled
    // flow_ful and flow_pro carry PRO and FUL respectively, as there); from
    // flow_tem on, values are written with 11 significant digits
    struct Block { const char *label; int field; bool p11; };
    static const Block blocks[] = {{"flow_pressure", MC_FIELD_P, false}, {"flow_te", MC_FIELD_TE, false},
                                   {"flow_ed", MC_FIELD_ED, false},      {"flow_tem", MC_FIELD_TEM, true},
                                   {"flow_ful", MC_FIELD_PRO, true},     {"flow_pro", MC_FIELD_FUL, true},
                                   {"flow_varf", MC_FIELD_VARF, true},   {"flow_varp", MC_FIELD_VARP, true}};
    for (const Block &b : blocks) {
        v << "SCALARS " << b.label << " float" << std::endl;
        v << "LOOKUP_TABLE default" << std::endl;
        for (int i = 0; i < N; i++) {
            if (b.p11) v << std::setprecision(11);
            v << f[b.field][i] << "\t";
        }
        v << std::endl;
    }
    v.close();
    if (!v) return fail(h, MC_ERR_ARG, "write failed: " + name);
    return MC_OK;
}

// ------------------------------------------------------- checkpoint / resume

namespace {

constexpr char kCkptMagic[8] = {'M', 'C', 'C', 'K', 'P', 'T', '0', '1'};

struct CkptHeader {
    char magic[8];
    uint32_t version, cells, faces, mode, reorder, scalars, precision, pressure_solver;
    uint64_t timestep_count;
    int32_t pass_in_step, first_pressure, sources_set, pad;
    double mass_source_total;
    char reserved[128 - 8 - 8 * 4 - 8 - 4 * 4 - 8];
};
static_assert(sizeof(CkptHeader) == 128, "checkpoint header is 128 bytes");

// The device arrays that carry state from one pass to the next, in the
// handle's own cell and face order: the fields, the face mass fluxes, the
// pressure-correction system (stale across passes in compat mode), the
// particle sources, the previous correction and the momentum diagonal.
std::vector<std::pair<double *, size_t>> checkpoint_arrays(mc_flow *h)
{
    const size_t N = (size_t)h->N, NB = N + 6, F = (size_t)h->F;
    std::vector<std::pair<double *, size_t>> a;
    for (int g = 0; g < G_NFIELDS; g++) a.push_back({h->phi[g], NB});
    if (h->has_scalars)
        for (int f : kScalarFields) a.push_back({h->sfield[f], NB});
    a.push_back({h->mdot, F});
    a.push_back({h->off_p, 6 * N});
    a.push_back({h->diag_p, N});
    a.push_back({h->b_p, N});
    a.push_back({h->src, 5 * N});
    a.push_back({h->pp_prev, N});
    a.push_back({h->AU, N});
    return a;
}

} // namespace

int mc_flow_checkpoint_write(mc_flow *h, const char *path)
{
    if (!h || !path) return MC_ERR_ARG;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return fail(h, MC_ERR_ARG, std::string("cannot open ") + path);
    CkptHeader hd{};
    std::memcpy(hd.magic, kCkptMagic, 8);
    hd.version = 1;
    hd.cells = (uint32_t)h->N;
    hd.faces = (uint32_t)h->F;
    hd.mode = (uint32_t)h->prm.mode;
    hd.reorder = (uint32_t)h->prm.reorder;
    hd.scalars = h->has_scalars ? 1u : 0u;
    hd.precision = (uint32_t)h->prm.precision;
    hd.pressure_solver = (uint32_t)h->prm.pressure_solver;
    hd.timestep_count = h->timestep_count;
    hd.pass_in_step = h->pass_in_step;
    hd.first_pressure = h->first_pressure;
    hd.sources_set = h->sources_set;
    hd.mass_source_total = h->mass_source_total;
    if (h->mass_source_on_device)  // sources set from device memory: their total lives on the device
        CUDA_TRY(h, cudaMemcpy(&hd.mass_source_total, h->scalars + 2, sizeof(double), cudaMemcpyDeviceToHost));
    bool ok = std::fwrite(&hd, sizeof(hd), 1, fp) == 1;
    std::vector<double> buf;
    for (const auto &arr : checkpoint_arrays(h)) {
        if (!ok) break;
        buf.resize(arr.second);
        if (cudaMemcpy(buf.data(), arr.first, arr.second * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fclose(fp);
            return fail(h, MC_ERR_CUDA, "checkpoint copy");
        }
        ok = std::fwrite(buf.data(), 8, arr.second, fp) == arr.second;
    }
    if (std::fclose(fp) != 0) ok = false;
    return ok ? MC_OK : fail(h, MC_ERR_ARG, std::string("checkpoint write failed: ") + path);
}

int mc_flow_checkpoint_read(mc_flow *h, const char *path)
{
    if (!h || !path) return MC_ERR_ARG;
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return fail(h, MC_ERR_ARG, std::string("cannot open ") + path);
    CkptHeader hd{};
    if (std::fread(&hd, sizeof(hd), 1, fp) != 1 || std::memcmp(hd.magic, kCkptMagic, 8) != 0 || hd.version != 1) {
        std::fclose(fp);
        return fail(h, MC_ERR_ARG, std::string("not a checkpoint: ") + path);
    }
    if (hd.cells != (uint32_t)h->N || hd.faces != (uint32_t)h->F || hd.mode != (uint32_t)h->prm.mode ||
        hd.reorder != (uint32_t)h->prm.reorder || hd.scalars != (h->has_scalars ? 1u : 0u) ||
        hd.precision != (uint32_t)h->prm.precision || hd.pressure_solver != (uint32_t)h->prm.pressure_solver) {
        std::fclose(fp);
        return fail(h, MC_ERR_ARG, "checkpoint was written by a handle with another mesh size or options");
    }
    std::vector<double> buf;
    for (const auto &arr : checkpoint_arrays(h)) {
        buf.resize(arr.second);
        if (std::fread(buf.data(), 8, arr.second, fp) != arr.second) {
            std::fclose(fp);
            return fail(h, MC_ERR_ARG, "checkpoint is truncated");
        }
        CUDA_TRY(h, cudaMemcpy(arr.first, buf.data(), arr.second * 8, cudaMemcpyHostToDevice));
    }
    std::fclose(fp);
    h->timestep_count = hd.timestep_count;
    h->pass_in_step = hd.pass_in_step;
    h->first_pressure = hd.first_pressure;
    h->sources_set = hd.sources_set;
    h->mass_source_total = hd.mass_source_total;
    h->mass_source_on_device = false;
    // the solvers' by-direction copy of a carried-over pressure system
    if (h->p_dir64)
        k_dir_rows64<<<blocks_for(h->N), MCB_THREADS, 0, h->stream>>>(h->N, h->off_p, h->dc.code, h->p_dir64,
                                                                     h->dc_pdir.sym);
    // a pressure system carried over from before (compat mode) needs its AMG
    // values; the coarsest inverse is formed in line
    if (h->use_amg && !h->first_pressure) {
        h->inverse_ready = false;
        h->inverse_pending = false;
        const int rs = setup_amg_values(h);
        if (rs) return rs;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return check_launch(h);
}

// ------------------------------------------------------ flow/particle exchange

namespace {

// Device memory of at least `bytes` for the rows or requests of one call.
int input_buffer(mc_flow *h, size_t bytes, char **out)
{
    if (bytes > h->xin_bytes) {
        if (h->xin_mem) cudaFree(h->xin_mem);
        h->xin_mem = nullptr;
        h->xin_bytes = 0;
        CUDA_TRY(h, cudaMalloc((void **)&h->xin_mem, bytes));
        h->xin_bytes = bytes;
    }
    *out = h->xin_mem;
    return MC_OK;
}

// The node tables of the interpolation: cell -> nodes (caller order), node
// coordinates, node -> its cells (handle ids, ascending caller id).
int setup_nodes(mc_flow *h)
{
    if (h->node_mem) return MC_OK;
    const size_t N = (size_t)h->N, P = (size_t)h->P;
    std::vector<int> off(P + 1, 0), cells(8 * N);
    for (size_t i = 0; i < 8 * N; i++) off[(size_t)h->h_cell_nodes[i] + 1]++;
    for (size_t p = 0; p < P; p++) off[p + 1] += off[p];
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (size_t c = 0; c < N; c++)  // caller ids ascending: each node's list is sorted by caller id
        for (int v = 0; v < 8; v++) {
            const int node = h->h_cell_nodes[8 * c + v];
            cells[fill[node]++] = h->reordered ? h->cell_o2n[c] : (int)c;
        }
    std::vector<double> xyz[3];
    for (int d = 0; d < 3; d++) {
        xyz[d].resize(P);
        for (size_t p = 0; p < P; p++) xyz[d][p] = h->h_points[3 * p + d];
    }
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t nb = (P + 1023) / 1024 + 1;
    const size_t bytes = al(8 * N * 4) + 3 * al(P * 8) + al((P + 1) * 4) + al(8 * N * 4) + al(P) + al(nb * 4) + 256 +
                         al(P * 4) + al(5 * P * 8);
    CUDA_TRY(h, cudaMalloc((void **)&h->node_mem, bytes));
    char *q = h->node_mem;
    auto take = [&](size_t b) { char *r = q; q += al(b); return r; };
    h->d_cell_nodes = (int *)take(8 * N * 4);
    h->px = (double *)take(P * 8);
    h->py = (double *)take(P * 8);
    h->pz = (double *)take(P * 8);
    h->pc_off = (int *)take((P + 1) * 4);
    h->pc_cells = (int *)take(8 * N * 4);
    h->node_flag = (unsigned char *)take(P);
    h->node_counts = (int *)take(nb * 4);
    h->node_count = (int *)take(256);
    h->node_list = (int *)take(P * 4);
    h->node_out = (double *)take(5 * P * 8);
    CUDA_TRY(h, cudaMemcpy(h->d_cell_nodes, h->h_cell_nodes.data(), 8 * N * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->px, xyz[0].data(), P * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->py, xyz[1].data(), P * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->pz, xyz[2].data(), P * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->pc_off, off.data(), (P + 1) * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->pc_cells, cells.data(), 8 * N * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemset(h->node_flag, 0, P));
    return MC_OK;
}

} // namespace

int mc_flow_ingest_particles(mc_flow *h, int64_t rows, const uint64_t *cells, const double *terms)
{
    if (!h || rows < 0 || (rows > 0 && (!cells || !terms))) return MC_ERR_ARG;
    if (rows > (int64_t)1 << 29) return fail(h, MC_ERR_UNSUPPORTED, "more than 2^29 particle rows in one call");
    const int n = (int)rows;
    std::vector<int> cell32((size_t)n);
    for (int i = 0; i < n; i++) {
        if (cells[i] >= (uint64_t)h->N) return fail(h, MC_ERR_ARG, "particle row " + std::to_string(i) + ": no such cell");
        cell32[i] = (int)cells[i];
    }
    const size_t N = (size_t)h->N;
    CUDA_TRY(h, cudaMemsetAsync(h->src, 0, 5 * N * 8, h->stream));
    if (n > 0) {
        int n2 = 2048;
        while (n2 < n) n2 <<= 1;
        char *buf = nullptr;
        const size_t keys_b = (size_t)n2 * 8, rows_b = ((size_t)5 * n * 8 + 255) & ~(size_t)255;
        int rc = input_buffer(h, keys_b + rows_b + (size_t)n * 4, &buf);
        if (rc) return rc;
        uint64_t *keys = (uint64_t *)buf;
        double *d_rows = (double *)(buf + keys_b);
        int *d_cells = (int *)(buf + keys_b + rows_b);
        CUDA_TRY(h, cudaMemcpyAsync(d_cells, cell32.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(d_rows, terms, (size_t)5 * n * 8, cudaMemcpyHostToDevice, h->stream));
        launch(h, K_EXCHANGE, [&] { particle_keys(h->stream, n, n2, d_cells, keys); });
        launch(h, K_EXCHANGE, [&] { sort_keys(h->stream, keys, n2); });
        launch(h, K_EXCHANGE, [&] {
            particle_sums(h->stream, n, keys, d_rows, h->reordered ? h->d_cell_o2n : nullptr, h->N, h->src);
        });
        rc = check_launch(h);
        if (rc) return rc;
    }
    // the total mass source, summed in the caller's cell order as mc_flow_set_sources does
    std::vector<double> fuel(N);
    CUDA_TRY(h, cudaMemcpyAsync(fuel.data(), h->src + 4 * N, N * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    double total = 0.0;
    for (size_t i = 0; i < N; i++) total += fuel[h->reordered ? (size_t)h->cell_o2n[i] : i];
    h->mass_source_total = total;
    h->mass_source_on_device = false;
    h->sources_set = 1;
    return MC_OK;
}

int mc_flow_get_sources(mc_flow *h, double *terms)
{
    if (!h || !terms) return MC_ERR_ARG;
    const size_t N = (size_t)h->N;
    std::vector<double> soa(5 * N);
    CUDA_TRY(h, cudaMemcpyAsync(soa.data(), h->src, 5 * N * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < N; i++) {
        const size_t j = h->reordered ? (size_t)h->cell_o2n[i] : i;
        for (int k = 0; k < 5; k++) terms[5 * i + k] = soa[k * N + j];
    }
    return MC_OK;
}

int mc_flow_interpolate_nodes(mc_flow *h, int64_t n_cells, const uint64_t *cells, int64_t max_nodes,
                              int64_t *n_nodes, uint64_t *node_ids, double *node_fields)
{
    if (!h || n_cells < 0 || (n_cells > 0 && !cells) || !n_nodes) return MC_ERR_ARG;
    if (n_cells > INT32_MAX) return fail(h, MC_ERR_UNSUPPORTED, "too many requested cells");
    const int n = (int)n_cells;
    std::vector<int> req((size_t)n);
    for (int i = 0; i < n; i++) {
        if (cells[i] >= (uint64_t)h->N) return fail(h, MC_ERR_ARG, "requested cell " + std::to_string(i) + ": no such cell");
        req[i] = (int)cells[i];
    }
    int rc = setup_nodes(h);
    if (rc) return rc;
    int count = 0;
    if (n > 0) {
        char *buf = nullptr;
        rc = input_buffer(h, (size_t)n * 4, &buf);
        if (rc) return rc;
        int *d_req = (int *)buf;
        CUDA_TRY(h, cudaMemcpyAsync(d_req, req.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->stream));
        launch(h, K_EXCHANGE, [&] { mark_nodes(h->stream, n, d_req, h->d_cell_nodes, h->node_flag); });
        launch(h, K_EXCHANGE,
               [&] { compact_nodes(h->stream, h->P, h->node_flag, h->node_counts, h->node_list, h->node_count); });
        CUDA_TRY(h, cudaMemcpyAsync(&count, h->node_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        rc = check_launch(h);
        if (rc) return rc;
    }
    *n_nodes = count;
    if (!node_ids && !node_fields) return MC_OK;  // size query
    if (count > max_nodes) return fail(h, MC_ERR_ARG, "max_nodes is smaller than the number of nodes");
    if (count == 0) return MC_OK;
    ensure_pressure_gradient(h);
    NodeArgs a{};
    a.U = h->phi[G_U];
    a.V = h->phi[G_V];
    a.W = h->phi[G_W];
    a.P = h->phi[G_P];
    a.T = h->phi[G_T];
    for (int d = 0; d < 3; d++) {
        a.gU[d] = h->grad[G_U][d];
        a.gV[d] = h->grad[G_V][d];
        a.gW[d] = h->grad[G_W][d];
        a.gP[d] = h->grad[G_P][d];
        a.gT[d] = h->grad[G_T][d];
    }
    a.xc = h->xc;
    a.yc = h->yc;
    a.zc = h->zc;
    a.px = h->px;
    a.py = h->py;
    a.pz = h->pz;
    a.pc_off = h->pc_off;
    a.pc_cells = h->pc_cells;
    a.u_ref = h->prm.inlet_u;
    a.p_ref = h->prm.pressure0;
    a.t_ref = h->prm.temperature0;
    launch(h, K_EXCHANGE, [&] { node_values(h->stream, count, h->node_list, a, h->node_out); });
    rc = check_launch(h);
    if (rc) return rc;
    std::vector<int> ids((size_t)count);
    CUDA_TRY(h, cudaMemcpyAsync(ids.data(), h->node_list, (size_t)count * 4, cudaMemcpyDeviceToHost, h->stream));
    if (node_fields)
        CUDA_TRY(h, cudaMemcpyAsync(node_fields, h->node_out, (size_t)count * 5 * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (node_ids)
        for (int i = 0; i < count; i++) node_ids[i] = (uint64_t)ids[i];
    return MC_OK;
}

int mc_flow_get_cell_order(mc_flow *h, int *cell_new_to_old)
{
    if (!h || !cell_new_to_old) return MC_ERR_ARG;
    for (int i = 0; i < h->N; i++) cell_new_to_old[i] = h->reordered ? h->cell_n2o[i] : i;
    return MC_OK;
}

int mc_flow_get_gradient(mc_flow *h, int field, double *vals)
{
    if (!h || !vals) return MC_ERR_ARG;
    if (!grad_ptr(h, field, 0)) return MC_ERR_UNSUPPORTED;
    if (field == MC_FIELD_P) ensure_pressure_gradient(h);
    std::vector<double> tmp((size_t)h->N);
    for (int d = 0; d < 3; d++) {
        const double *src = grad_ptr(h, field, d);
        if (h->reordered) {
            permute(h, h->stage, src, h->d_cell_o2n, h->N, 0);
            src = h->stage;
        }
        CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), src, (size_t)h->N * 8, cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        for (int i = 0; i < h->N; i++) vals[3 * (size_t)i + d] = tmp[i];
    }
    return MC_OK;
}

int mc_flow_set_sources(mc_flow *h, const double *terms)
{
    if (!h || !terms) return MC_ERR_ARG;
    const size_t N = (size_t)h->N;
    std::vector<double> soa(5 * N);
    double total = 0.0;
    for (size_t i = 0; i < N; i++) {
        const size_t j = h->reordered ? (size_t)h->cell_o2n[i] : i;
        for (int k = 0; k < 5; k++) soa[k * N + j] = terms[5 * i + k];
        total += terms[5 * i + 4];
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->src, soa.data(), 5 * N * 8, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->mass_source_total = total;
    h->mass_source_on_device = false;
    h->sources_set = 1;
    return MC_OK;
}

int mc_flow_set_sources_device(mc_flow *h, const double *terms_soa)
{
    if (!h || !terms_soa) return MC_ERR_ARG;
    const size_t N = (size_t)h->N;
    for (int k = 0; k < 5; k++) {
        if (h->reordered)
            permute(h, h->src + k * N, terms_soa + k * N, h->d_cell_n2o, h->N, 0);
        else
            CUDA_TRY(h, cudaMemcpyAsync(h->src + k * N, terms_soa + k * N, N * 8, cudaMemcpyDeviceToDevice,
                                        h->stream));
    }
    launch(h, K_PERMUTE, [&] {
        k_sum<<<krylov_grid(h->N), MCB_THREADS, 0, h->stream>>>(h->N, h->src + 4 * N, h->partials, h->counter,
                                                                h->scalars + 2);
    });
    const int rc = check_launch(h);
    if (rc) return rc;
    h->mass_source_on_device = true;
    h->sources_set = 1;
    return MC_OK;
}

int mc_flow_get_face_array(mc_flow *h, int which, double *vals)
{
    if (!h || !vals) return MC_ERR_ARG;
    const size_t F = (size_t)h->F;
    auto get1 = [&](const double *d, int stride, int comp) -> int {
        std::vector<double> tmp(F);
        if (h->reordered) {
            permute(h, h->stage, d, h->d_face_o2n, h->F, 0);
            d = h->stage;
        }
        CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), d, F * 8, cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < F; i++) vals[stride * i + comp] = tmp[i];
        return MC_OK;
    };
    switch (which) {
    case 0: return get1(h->mdot, 1, 0);
    case 1: return get1(h->area, 1, 0);
    case 2: return get1(h->lam, 1, 0);
    case 3: return get1(h->rl, 1, 0);
    case 4: { int rc = get1(h->ff0, 2, 0); return rc ? rc : get1(h->ff1, 2, 1); }
    case 5: { int rc = get1(h->Sx, 3, 0); rc = rc ? rc : get1(h->Sy, 3, 1); return rc ? rc : get1(h->Sz, 3, 2); }
    case 6: { int rc = get1(h->xf, 3, 0); rc = rc ? rc : get1(h->yf, 3, 1); return rc ? rc : get1(h->zf, 3, 2); }
    default: return MC_ERR_ARG;
    }
}

int mc_flow_get_cell_array(mc_flow *h, int which, double *vals)
{
    if (!h || !vals) return MC_ERR_ARG;
    const double *src = which == 0 ? h->AU : which == 1 ? h->diag_p : which == 2 ? h->vol : which == 3 ? h->rho : nullptr;
    if (!src) return MC_ERR_ARG;
    if (h->reordered) {
        permute(h, h->stage, src, h->d_cell_o2n, h->N, 0);
        src = h->stage;
    }
    CUDA_TRY(h, cudaMemcpyAsync(vals, src, (size_t)h->N * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return MC_OK;
}

int mc_flow_get_csr(mc_flow *h, int system, int *n, int *nnz, int *row_ptr, int *col, double *val, double *rhs)
{
    if (!h || !n || !nnz) return MC_ERR_ARG;
    const size_t N = (size_t)h->N;
    const double *d_diag, *d_off, *d_rhs;
    switch (system) {
    case MC_SYSTEM_MOMENTUM: d_diag = h->AU; d_off = h->off_m; d_rhs = h->b_m; break;
    case MC_SYSTEM_PRESSURE: d_diag = h->diag_p; d_off = h->off_p; d_rhs = h->b_p; break;
    case MC_SYSTEM_TEMPERATURE: d_diag = h->diag_t; d_off = h->off_t; d_rhs = h->b_t; break;
    case 3: d_diag = h->AU; d_off = h->off_m; d_rhs = h->b_m + N; break;      // momentum, V right-hand side
    case 4: d_diag = h->AU; d_off = h->off_m; d_rhs = h->b_m + 2 * N; break;  // momentum, W right-hand side
    default: return MC_ERR_ARG;
    }
    size_t count = N;
    for (int c : h->hcol) count += c >= 0;
    *n = (int)N;
    *nnz = (int)count;
    if (!row_ptr && !col && !val && !rhs) return MC_OK;
    std::vector<double> diag(N), off(6 * N), b(N);
    CUDA_TRY(h, cudaMemcpyAsync(diag.data(), d_diag, N * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(off.data(), d_off, 6 * N * 8, cudaMemcpyDeviceToHost, h->stream));
    if (rhs) CUDA_TRY(h, cudaMemcpyAsync(b.data(), d_rhs, N * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (h->rows.code && system != MC_SYSTEM_PRESSURE) {  // rows stored by direction: back to slot order
        std::vector<double> dir(off);
        for (size_t i = 0; i < N; i++)
            for (int k = 0; k < 6; k++) {
                const unsigned d = (h->hcode[i] >> (3 * k)) & 7u;
                off[k * N + i] = d < 6 ? dir[(size_t)((h->rows.pos >> (3 * d)) & 7u) * N + i] : 0.0;
            }
    }
    size_t pos = 0;
    std::vector<std::pair<int, double>> row;
    // rows and columns in the caller's numbering
    for (size_t o = 0; o < N; o++) {
        const size_t i = h->reordered ? (size_t)h->cell_o2n[o] : o;
        row.clear();
        row.push_back({(int)o, diag[i]});
        if (rhs) rhs[o] = b[i];
        for (int k = 0; k < 6; k++) {
            const int c = h->hcol[k * N + i];
            if (c >= 0) row.push_back({h->reordered ? h->cell_n2o[c] : c, off[k * N + i]});
        }
        std::sort(row.begin(), row.end(), [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
            return a.first < b.first;
        });
        if (row_ptr) row_ptr[o] = (int)pos;
        for (auto &e : row) {
            if (col) col[pos] = e.first;
            if (val) val[pos] = e.second;
            pos++;
        }
    }
    if (row_ptr) row_ptr[N] = (int)pos;
    return MC_OK;
}

int mc_flow_stage_gradients(mc_flow *h)
{
    if (!h) return MC_ERR_ARG;
    int rc = stage_gradients(h);
    if (!rc) CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    flush_timing(h);
    return rc;
}

int mc_flow_stage_set_up_field(mc_flow *h)
{
    if (!h) return MC_ERR_ARG;
    int rc = stage_set_up_field(h);
    if (!rc) CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    flush_timing(h);
    return rc;
}

int mc_flow_stage_momentum(mc_flow *h, mc_iter_stats *st)
{
    if (!h) return MC_ERR_ARG;
    const int rc = stage_momentum(h, st);
    flush_timing(h);
    return rc;
}

int mc_flow_stage_pressure(mc_flow *h, mc_iter_stats *st)
{
    if (!h) return MC_ERR_ARG;
    const int rc = stage_pressure(h, st);
    if (rc != MC_ERR_CUDA) CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    flush_timing(h);
    return rc;
}

int mc_flow_stage_temperature(mc_flow *h, mc_iter_stats *st)
{
    if (!h) return MC_ERR_ARG;
    const int rc = stage_temperature(h, st);
    flush_timing(h);
    return rc;
}

int mc_flow_stage_scalar(mc_flow *h, int field, mc_iter_stats *st)
{
    if (!h) return MC_ERR_ARG;
    const int rc = stage_scalar(h, field, st);
    const int rs = check_launch(h);
    if (rs) return rs;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    flush_timing(h);
    return rc;
}

// One pass of FlowSolver::timestep's loop (FlowSolver.inl:3188-3268).
int mc_flow_simple_iteration(mc_flow *h, mc_iter_stats *st)
{
    if (!h) return MC_ERR_ARG;
    mc_iter_stats local{};
    mc_iter_stats *s = st ? st : &local;
    memset(s, 0, sizeof(*s));
    int worst = MC_OK;
    auto track = [&](int rc) -> int {
        if (rc == MC_ERR_CUDA || rc == MC_ERR_NONFINITE) return rc;
        if (rc != MC_OK && worst == MC_OK) worst = rc;
        return MC_OK;
    };
    int rc = stage_gradients(h);
    if (rc) return rc;
    if (h->timestep_count == 0 && h->pass_in_step == 0) {
        rc = stage_set_up_field(h);
        if (rc) return rc;
    }
    if ((rc = track(stage_momentum(h, s)))) return rc;
    if ((rc = track(stage_pressure(h, s)))) return rc;
    if (h->has_scalars) {
        // the reference's order, FlowSolver.inl:3229-3261
        const int order[7] = {MC_FIELD_TE, MC_FIELD_ED, MC_FIELD_TEM, MC_FIELD_FUL, MC_FIELD_PRO, MC_FIELD_VARF,
                              MC_FIELD_VARP};
        for (int f : order)
            if ((rc = track(stage_scalar(h, f, s)))) return rc;
    } else {
        if ((rc = track(stage_temperature(h, s)))) return rc;
    }
    // the mass imbalance was formed by the temperature stage's kernel
    CUDA_TRY(h, cudaMemcpyAsync(h->h_scalars + 1, h->scalars + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    flush_timing(h);
    rc = check_launch(h);
    if (rc) return rc;
    s->mass_imbalance = h->h_scalars[1];
    h->pass_in_step++;
    if (h->pass_in_step == 3) {
        h->pass_in_step = 0;
        h->timestep_count++;
    }
    return worst;
}

int mc_flow_timestep(mc_flow *h, mc_iter_stats *st)
{
    if (!h) return MC_ERR_ARG;
    int worst = MC_OK;
    do {
        const int rc = mc_flow_simple_iteration(h, st);
        if (rc == MC_ERR_CUDA || rc == MC_ERR_NONFINITE || rc == MC_ERR_ARG) return rc;
        if (rc != MC_OK && worst == MC_OK) worst = rc;
    } while (h->pass_in_step != 0);
    return worst;
}

int mc_flow_set_timing(mc_flow *h, int enable)
{
    if (!h) return MC_ERR_ARG;
    flush_timing(h);
    h->timing.on = enable != 0;
    return MC_OK;
}

int mc_flow_kernel_count(void) { return K_COUNT; }

const char *mc_flow_kernel_name(int id) { return (id >= 0 && id < K_COUNT) ? kKernelNames[id] : ""; }

int mc_flow_get_kernel_times(mc_flow *h, double *total_ms, long *launches)
{
    if (!h) return MC_ERR_ARG;
    flush_timing(h);
    for (int i = 0; i < K_COUNT; i++) {
        if (total_ms) total_ms[i] = h->timing.total_ms[i];
        if (launches) launches[i] = h->timing.count[i];
    }
    return MC_OK;
}

int mc_flow_reset_kernel_times(mc_flow *h)
{
    if (!h) return MC_ERR_ARG;
    flush_timing(h);
    for (int i = 0; i < K_COUNT; i++) {
        h->timing.total_ms[i] = 0.0;
        h->timing.count[i] = 0;
    }
    return MC_OK;
}

void *mc_flow_stream(mc_flow *h) { return h ? (void *)h->stream : nullptr; }
long mc_flow_launch_count(mc_flow *h) { return h ? h->launches : 0; }
const char *mc_flow_last_error(mc_flow *h) { return h ? h->err.c_str() : ""; }

const char *mc_status_string(int s)
{
    switch (s) {
    case MC_OK: return "ok";
    case MC_ERR_ARG: return "invalid argument";
    case MC_ERR_CUDA: return "CUDA error";
    case MC_ERR_NOT_CONVERGED: return "linear solve did not converge";
    case MC_ERR_NONFINITE: return "non-finite value";
    case MC_ERR_MESH: return "inconsistent mesh";
    case MC_ERR_NOMEM: return "out of memory";
    case MC_ERR_UNSUPPORTED: return "unsupported option";
    case MC_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
    }
}

} // extern "C"
