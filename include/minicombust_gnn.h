/* C ABI of the learned pressure-correction guess (message-passing network
 * over the cell-face graph).  No reference counterpart: the reference starts
 * every pressure solve from zero (PETSc KSP / AmgX defaults,
 * FlowSolver.inl:2203-2273).
 *
 * The network and its kernels are described in the library sources
 * (gnn.cuh).  Training and inference run on the device; sample arrays are
 * DEVICE pointers of n floats in the mesh's own cell numbering.  All calls
 * return 0 or a negative mc_status code (minicombust_flow.h). */
#ifndef MINICOMBUST_GNN_H
#define MINICOMBUST_GNN_H

#include <stdint.h>

#include "minicombust_flow.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mc_gnn mc_gnn;
typedef struct mc_gnn_graph mc_gnn_graph;

/* One training or inference sample (device arrays, n floats each).
 * rhs: pressure-correction right-hand side projected to mean zero;
 * diag: matrix diagonal; prev: previous converged correction (may be NULL);
 * target: converged correction (training only). */
typedef struct mc_gnn_sample {
    const float *rhs;
    const float *diag;
    const float *prev;
    const float *target;
} mc_gnn_sample;

/* Number of FP32 parameters (the layout is fixed by the library). */
int mc_gnn_param_count(void);
/* A network with seeded initial parameters on `device`. */
int mc_gnn_create(int device, uint64_t seed, mc_gnn **out);
int mc_gnn_destroy(mc_gnn *net);
int mc_gnn_set_params(mc_gnn *net, const float *host_params, int count);
int mc_gnn_get_params(mc_gnn *net, float *host_params, int count);
/* The cell-face graph of a mesh (caller numbering): neighbours through
 * internal faces, face features [area, rlencos] normalised by their means
 * over internal faces, cell volumes normalised by their mean. */
int mc_gnn_graph_create(mc_gnn *net, const mc_mesh_view *mesh, mc_gnn_graph **out);
int mc_gnn_graph_destroy(mc_gnn_graph *graph);
/* Host copies of a graph's arrays: col [6][n] (unused slots hold the row),
 * edge [6][n] packed BF16 pairs (area, rlencos; low half first), vhat [n]. */
int mc_gnn_graph_export(const mc_gnn_graph *graph, int *n, int *col, uint32_t *edge, float *vhat);
/* Prediction for one sample: y (units of rhs_rms / diag_mean) and the
 * guess x0 = s_x y in the units of the solution; either output may be NULL.
 * Device pointers of n values. */
int mc_gnn_predict(mc_gnn *net, const mc_gnn_graph *graph, const mc_gnn_sample *sample, float *y, double *x0);
/* Mean loss over `batch` samples and its gradient (kept on the device for
 * mc_gnn_adam_step; copied to host_grad when not NULL). */
int mc_gnn_loss_grad(mc_gnn *net, const mc_gnn_graph *graph, int batch, const mc_gnn_sample *samples,
                     double *loss, float *host_grad);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) with the last gradient. */
int mc_gnn_adam_step(mc_gnn *net, float lr);
/* mc_gnn_loss_grad followed by mc_gnn_adam_step. */
int mc_gnn_train_step(mc_gnn *net, const mc_gnn_graph *graph, int batch, const mc_gnn_sample *samples, float lr,
                      double *loss);

#ifdef __cplusplus
}
#endif

#endif
