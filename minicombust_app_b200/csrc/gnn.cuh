// Message-passing network over the cell-face graph that predicts an initial
// guess for the pressure-correction solve.
//
// Inputs per cell (normalised on the device, per sample):
//   b^ = (b - shift) / s_b      s_b = RMS of the mean-projected right-hand side
//   d^ = diag / s_d             s_d = mean diagonal
//   p^ = prev / s_x             s_x = s_b / s_d (the unit of the solution)
//   v^ = vol / mean(vol)
// Inputs per face (per cell slot): e = [area / mean area, rlencos / mean
// rlencos] over internal faces.
//
// Network (hidden width H = 32, L = 4 layers, BF16 weights and activations,
// FP32 accumulation):
//   h0   = relu(We x + ce)
//   m_i  = sum over internal slots k of g_k (.) h_j,   g_k = Wg e_k + cg
//   h'_i = h_i + W2 relu(W1 [h_i; m_i] + c1) + c2      (each layer)
//   y_i  = wo . relu(Wd h_i + cd) + co
// Prediction x0 = s_x * y.  Training minimises the mean squared difference
// to the converged correction in units of s_x, after removing the mean
// difference (the pressure-correction system is singular in the constant).
//
// The dense products run on the tensor cores as mma.sync m16n8k16 BF16 tiles
// of 128 cells per block.  The forward gather stages a tile's own and
// neighbour rows in shared memory with asynchronous 16-byte copies, all in
// flight at once; the backward gathers put one channel per lane.
#pragma once

#include <stdint.h>

#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace mcb {

constexpr int GNN_H = 32;
constexpr int GNN_L = 4;
constexpr int GNN_IN = 4;
constexpr int GNN_TILE = 128;   // cells per block

// Parameter layout (FP32 master copy, flat).
constexpr int GP_WE = 0;                         // [H][IN]
constexpr int GP_CE = GP_WE + GNN_H * GNN_IN;    // [H]
constexpr int GP_LAYER0 = GP_CE + GNN_H;
constexpr int GPL_WG = 0;                        // [H][2]
constexpr int GPL_CG = GPL_WG + GNN_H * 2;       // [H]
constexpr int GPL_W1 = GPL_CG + GNN_H;           // [H][2H]
constexpr int GPL_C1 = GPL_W1 + GNN_H * 2 * GNN_H;
constexpr int GPL_W2 = GPL_C1 + GNN_H;           // [H][H]
constexpr int GPL_C2 = GPL_W2 + GNN_H * GNN_H;
constexpr int GPL_SIZE = GPL_C2 + GNN_H;
constexpr int GP_DEC = GP_LAYER0 + GNN_L * GPL_SIZE;
constexpr int GPD_WD = 0;                        // [H][H]
constexpr int GPD_CD = GPD_WD + GNN_H * GNN_H;
constexpr int GPD_WO = GPD_CD + GNN_H;
constexpr int GPD_CO = GPD_WO + GNN_H;
constexpr int GPD_SIZE = GPD_CO + 1;
constexpr int GNN_NPARAM = GP_DEC + GPD_SIZE;

// BF16 copies of the matrices the tensor cores read, row-major [out][in].
constexpr int GK_LAYER0 = 0;
constexpr int GKL_W1 = 0;
constexpr int GKL_W2 = GNN_H * 2 * GNN_H;
constexpr int GKL_SIZE = GKL_W2 + GNN_H * GNN_H;
constexpr int GK_WD = GNN_L * GKL_SIZE;
constexpr int GNN_NPACK = GK_WD + GNN_H * GNN_H;

struct GnnScales {
    double sb, sd, sx, shift;
    double rb, rd, rx;   // reciprocals (0 where the scale is 0)
};

// Graph in the solver's cell order.  Slot k is direction k of the
// reference's cell_faces (FRONT, BACK, LEFT, RIGHT, DOWN, UP): col[k][i] is
// the neighbour through it (the row itself on the boundary), edge[k][i] its
// face features, vhat the normalised volumes.
// Offset form (`affine`): every internal slot k of every cell i has the
// neighbour i + doff[k] and the face features ebits[k] -- a uniform box in
// x-fastest order; mask[i] bit k marks the internal slots.  The forward
// kernels then need neither col nor edge.
struct GnnGraph {
    int n;
    const int *col;                  // [6][n]
    const __nv_bfloat162 *edge;      // [6][n]
    const float *vhat;               // [n]
    int affine;
    int doff[6];
    uint32_t ebits[6];
    const uint8_t *mask;             // [n], nullptr unless affine
};

// One sample's raw inputs (device arrays of length n, type T).
template <typename T>
struct GnnInput {
    const T *b;
    const double *shift;   // device scalar subtracted from b (nullptr: 0)
    const T *diag;
    const T *prev;         // nullptr: zero
};

// Device scratch for one graph size.
struct GnnWork {
    int n = 0, nblocks = 0;
    bool train = false;
    __nv_bfloat16 *h[GNN_L + 1] = {};   // activations [n][H]; inference uses h[0], h[1] as ping-pong
    __nv_bfloat16 *a[GNN_L] = {};       // training: relu(W1 u + c1) per layer
    __nv_bfloat16 *q = nullptr;          // training: decoder hidden
    float *y = nullptr;                  // [n] network output (units of s_x)
    float *dh[2] = {};                   // training: [n][H] gradient ping-pong
    float *dm = nullptr;                 // training: [n][H]
    float *dy = nullptr;                 // training: [n]
    float *gpart = nullptr;              // training: [nblocks][NPARAM] per-block gradient partials
    double *partials = nullptr;          // reductions
    unsigned int *counter = nullptr;
    GnnScales *scales = nullptr;
    double *loss = nullptr;              // [2]: mean offset, loss
    __nv_bfloat16 *fold = nullptr;       // [L][7][H][H] offset-form weights (inference)
    int *status = nullptr;               // nonzero: a tensor-core layer gave up waiting (prediction zeroed)
};

size_t gnn_work_bytes(int n, bool train);
// Carve a work area out of `base` (gnn_work_bytes(n, train) bytes, 256-byte aligned).
void gnn_work_carve(GnnWork &w, char *base, int n, bool train);

// Host: Kaiming-uniform initialisation (splitmix64 stream from `seed`).
void gnn_init_params(float *p, uint64_t seed);
// Device: refresh the BF16 copies from the FP32 parameters.
void gnn_pack(cudaStream_t s, const float *p, __nv_bfloat16 *pk);

// Forward pass (inference).  Writes y (units of s_x) and, when x0 is given,
// x0 = s_x y in FP64 (the initial guess in the solver's units).  On a graph in
// offset form the per-direction gates are folded into the first weight
// matrix, [W1h | W1m diag(g_1) | ... | W1m diag(g_6)], so that each layer is
// one tensor-core product over the seven staged row tiles.
// `parts` selects the launches (for timing them apart): the scales and the
// encoder (GNN_FWD_BEGIN), the GNN_L layers (GNN_FWD_LAYERS), the decoder
// (GNN_FWD_END); called in that order on one stream.
enum { GNN_FWD_BEGIN = 1, GNN_FWD_LAYERS = 2, GNN_FWD_END = 4, GNN_FWD_ALL = 7 };
template <typename T>
void gnn_forward(cudaStream_t s, const GnnGraph &g, const GnnInput<T> &in, const float *p, const __nv_bfloat16 *pk,
                 GnnWork &w, double *x0, int parts = GNN_FWD_ALL);
int gnn_forward_launches();

// Layer kernel of the offset form: the tcgen05 kernel (default), the same
// kernel with no fall-back (MC_GNN_LAYER=umma), or the mma.sync kernel
// (MC_GNN_LAYER=mma).
enum class GnnLayerPath { Umma, UmmaRequired, Mma };
GnnLayerPath gnn_layer_path();

// TMA descriptor of the activations h ([n][32] BF16) in tiles of 128 rows
// with the 64-byte swizzle (an opaque CUtensorMap).
struct alignas(64) GnnTmaMap {
    unsigned char raw[128];
};
bool gnn_umma_map(GnnTmaMap *m, const __nv_bfloat16 *h, int n);
// Launch attributes of the layer kernel (false: the kernel cannot run).
bool gnn_umma_ready();
// The decoder fused into the last layer: y = wo . relu(Wd h' + cd) + co and
// x0 = s_x y (x0 may be null) instead of storing h'.
struct GnnUmmaDecode {
    const __nv_bfloat16 *pkd;  // Wd, BF16 [32][32]
    const float *pd;           // the decoder's FP32 parameters
    const GnnScales *scales;
    float *y;
    double *x0;
};
// One offset-form layer on the tcgen05 tensor cores, `grid` persistent
// blocks, hin (described by `map`) -> hout, or with dec the network's output.
void gnn_layer_umma(cudaStream_t s, const GnnGraph &g, const GnnTmaMap &map, const float *pl,
                    const __nv_bfloat16 *wf, const __nv_bfloat16 *pkl, const __nv_bfloat16 *hin,
                    __nv_bfloat16 *hout, int *status, int grid, const GnnUmmaDecode *dec = nullptr);

// Training: forward, loss against `target` (units of the solution), backward;
// adds this sample's gradient, scaled by `weight`, into grad[NPARAM] and
// the sample's loss into w.loss[1] (overwritten).
void gnn_loss_backward(cudaStream_t s, const GnnGraph &g, const GnnInput<float> &in, const float *target,
                       const float *p, const __nv_bfloat16 *pk, GnnWork &w, float *grad, float weight);

// Host: graph arrays of a solver mesh (its own numbering): direction-slot
// columns, the per-slot face features as BF16 pairs, normalised volumes.
// `aff` receives the offset form when it applies (aff.affine = 1, mask
// filled), else aff.affine = 0 and mask is empty.
struct HostMesh;
void gnn_graph_host(const HostMesh &hm, std::vector<int> &col, std::vector<uint32_t> &edge, std::vector<float> &vhat,
                    GnnGraph &aff, std::vector<uint8_t> &mask);

// Adam with bias correction; step t >= 1.
void gnn_adam(cudaStream_t s, float *p, const float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
              int t);

} // namespace mcb
