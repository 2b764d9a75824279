// C ABI of the learned guess network (include/minicombust_gnn.h).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gnn.cuh"
#include "mesh_setup.h"
#include "minicombust_gnn.h"

namespace mcb {

void gnn_graph_host(const HostMesh &hm, std::vector<int> &col, std::vector<uint32_t> &edge, std::vector<float> &vhat,
                    GnnGraph &aff, std::vector<uint8_t> &mask)
{
    const int N = hm.N;
    double asum = 0.0, rsum = 0.0;
    long cnt = 0;
    for (int f = 0; f < hm.F; f++)
        if (hm.fc1[f] < N) {
            asum += hm.area[f];
            rsum += hm.rl[f];
            cnt++;
        }
    const double ra = cnt && asum > 0 ? cnt / asum : 0.0, rr = cnt && rsum > 0 ? cnt / rsum : 0.0;
    // slot k = direction k (the sum over neighbours does not depend on the
    // slot order; a direction order makes the offsets of a box constant)
    col.assign((size_t)6 * N, 0);
    edge.assign((size_t)6 * N, 0u);
    for (int k = 0; k < 6; k++)
        for (int i = 0; i < N; i++) {
            const int j = hm.nbr[(size_t)k * N + i];
            col[(size_t)k * N + i] = j >= 0 ? j : i;
            if (j < 0) continue;
            int f = -1;
            for (int s = 0; s < 6; s++)
                if (hm.col[(size_t)s * N + i] == j) f = hm.sface[(size_t)s * N + i];
            if (f < 0) continue;
            const __nv_bfloat162 e = __floats2bfloat162_rn((float)(hm.area[f] * ra), (float)(hm.rl[f] * rr));
            uint32_t bits;
            std::memcpy(&bits, &e, 4);
            edge[(size_t)k * N + i] = bits;
        }
    double vsum = 0.0;
    for (int i = 0; i < N; i++) vsum += hm.vol[i];
    const double rv = vsum > 0 ? N / vsum : 0.0;
    vhat.resize(N);
    for (int i = 0; i < N; i++) vhat[i] = (float)(hm.vol[i] * rv);
    // offset form
    aff.affine = 0;
    mask.clear();
    bool ok = true, seen[6] = {false, false, false, false, false, false};
    std::vector<uint8_t> mk(N, 0);
    for (int k = 0; k < 6 && ok; k++)
        for (int i = 0; i < N; i++) {
            const int j = col[(size_t)k * N + i];
            if (j == i) continue;
            const uint32_t e = edge[(size_t)k * N + i];
            if (!seen[k]) {
                seen[k] = true;
                aff.doff[k] = j - i;
                aff.ebits[k] = e;
            } else if (j - i != aff.doff[k] || e != aff.ebits[k]) {
                ok = false;
                break;
            }
            mk[i] |= (uint8_t)(1u << k);
        }
    if (ok) {
        for (int k = 0; k < 6; k++)
            if (!seen[k]) {
                aff.doff[k] = 0;
                aff.ebits[k] = 0u;
            }
        aff.affine = 1;
        mask.swap(mk);
    }
}

} // namespace mcb

using namespace mcb;

struct mc_gnn {
    int dev = 0;
    cudaStream_t stream = nullptr;
    float *p = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *pk = nullptr;
    int t = 0;
    char *work_mem = nullptr;
    size_t work_bytes = 0;
    GnnWork work;
    double *h_loss = nullptr;  // pinned [2]
};

struct mc_gnn_graph {
    int dev = 0;
    GnnGraph g{};
    char *mem = nullptr;
};

namespace {

// MC_GNN_GENERAL_GATHER=1 keeps the general (column-list) gather even where
// the offset form applies; the tests use it to check both paths.
bool gnn_force_general()
{
    const char *v = std::getenv("MC_GNN_GENERAL_GATHER");
    return v && v[0] == '1';
}

int cuda_status(cudaError_t e) { return e == cudaSuccess ? MC_OK : (e == cudaErrorMemoryAllocation ? MC_ERR_NOMEM : MC_ERR_CUDA); }

#define GNN_TRY(call)                          \
    do {                                       \
        const int rc_ = cuda_status(call);     \
        if (rc_) return rc_;                   \
    } while (0)

int ensure_work(mc_gnn *net, int n)
{
    const size_t need = gnn_work_bytes(n, true);
    if (net->work_mem && net->work.n == n) return MC_OK;
    if (net->work_mem) {
        cudaStreamSynchronize(net->stream);
        cudaFree(net->work_mem);
        net->work_mem = nullptr;
    }
    GNN_TRY(cudaMalloc((void **)&net->work_mem, need));
    GNN_TRY(cudaMemsetAsync(net->work_mem, 0, need, net->stream));
    net->work_bytes = need;
    gnn_work_carve(net->work, net->work_mem, n, true);
    return MC_OK;
}

GnnInput<float> input_of(const mc_gnn_sample &s) { return GnnInput<float>{s.rhs, nullptr, s.diag, s.prev}; }

} // namespace

extern "C" {

int mc_gnn_param_count(void) { return GNN_NPARAM; }

int mc_gnn_create(int device, uint64_t seed, mc_gnn **out)
{
    if (!out) return MC_ERR_ARG;
    *out = nullptr;
    mc_gnn *net = new (std::nothrow) mc_gnn();
    if (!net) return MC_ERR_NOMEM;
    net->dev = device;
    std::vector<float> host(GNN_NPARAM);
    gnn_init_params(host.data(), seed);
    int rc = cuda_status(cudaSetDevice(device));
    if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking));
    const size_t pb = (size_t)GNN_NPARAM * sizeof(float);
    if (!rc) rc = cuda_status(cudaMalloc((void **)&net->p, 4 * pb + (size_t)GNN_NPACK * sizeof(__nv_bfloat16)));
    if (!rc) {
        net->grad = net->p + GNN_NPARAM;
        net->m = net->grad + GNN_NPARAM;
        net->v = net->m + GNN_NPARAM;
        net->pk = reinterpret_cast<__nv_bfloat16 *>(net->v + GNN_NPARAM);
        rc = cuda_status(cudaMemcpyAsync(net->p, host.data(), pb, cudaMemcpyHostToDevice, net->stream));
    }
    if (!rc) rc = cuda_status(cudaMemsetAsync(net->grad, 0, 3 * pb, net->stream));
    if (!rc) {
        gnn_pack(net->stream, net->p, net->pk);
        rc = cuda_status(cudaGetLastError());
    }
    if (!rc) rc = cuda_status(cudaMallocHost((void **)&net->h_loss, 2 * sizeof(double)));
    if (!rc) rc = cuda_status(cudaStreamSynchronize(net->stream));
    if (rc) {
        mc_gnn_destroy(net);
        return rc;
    }
    *out = net;
    return MC_OK;
}

int mc_gnn_destroy(mc_gnn *net)
{
    if (!net) return MC_ERR_ARG;
    cudaSetDevice(net->dev);
    if (net->stream) cudaStreamSynchronize(net->stream);
    if (net->work_mem) cudaFree(net->work_mem);
    if (net->p) cudaFree(net->p);
    if (net->h_loss) cudaFreeHost(net->h_loss);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
    return MC_OK;
}

int mc_gnn_set_params(mc_gnn *net, const float *host, int count)
{
    if (!net || !host || count != GNN_NPARAM) return MC_ERR_ARG;
    GNN_TRY(cudaSetDevice(net->dev));
    GNN_TRY(cudaMemcpyAsync(net->p, host, (size_t)GNN_NPARAM * 4, cudaMemcpyHostToDevice, net->stream));
    GNN_TRY(cudaMemsetAsync(net->m, 0, (size_t)2 * GNN_NPARAM * 4, net->stream));
    net->t = 0;
    gnn_pack(net->stream, net->p, net->pk);
    GNN_TRY(cudaGetLastError());
    GNN_TRY(cudaStreamSynchronize(net->stream));
    return MC_OK;
}

int mc_gnn_get_params(mc_gnn *net, float *host, int count)
{
    if (!net || !host || count != GNN_NPARAM) return MC_ERR_ARG;
    GNN_TRY(cudaSetDevice(net->dev));
    GNN_TRY(cudaMemcpyAsync(host, net->p, (size_t)GNN_NPARAM * 4, cudaMemcpyDeviceToHost, net->stream));
    GNN_TRY(cudaStreamSynchronize(net->stream));
    return MC_OK;
}

int mc_gnn_graph_create(mc_gnn *net, const mc_mesh_view *mesh, mc_gnn_graph **out)
{
    if (!net || !mesh || !out) return MC_ERR_ARG;
    *out = nullptr;
    HostMesh hm;
    std::string err;
    std::vector<int> col;
    std::vector<uint32_t> edge;
    std::vector<float> vhat;
    std::vector<uint8_t> mask;
    GnnGraph aff{};
    try {
        const int rc = build_host_mesh(mesh, HostPhysics{1.0}, hm, err);
        if (rc) return rc;
        gnn_graph_host(hm, col, edge, vhat, aff, mask);
    } catch (const std::bad_alloc &) {
        return MC_ERR_NOMEM;
    }
    mc_gnn_graph *gr = new (std::nothrow) mc_gnn_graph();
    if (!gr) return MC_ERR_NOMEM;
    const int N = hm.N;
    const size_t cb = (size_t)6 * N * 4, eb = (size_t)6 * N * 4, vb = (size_t)N * 4, mb = mask.size();
    gr->dev = net->dev;
    int rc = cuda_status(cudaSetDevice(net->dev));
    if (!rc) rc = cuda_status(cudaMalloc((void **)&gr->mem, cb + eb + vb + mb));
    if (!rc) rc = cuda_status(cudaMemcpy(gr->mem, col.data(), cb, cudaMemcpyHostToDevice));
    if (!rc) rc = cuda_status(cudaMemcpy(gr->mem + cb, edge.data(), eb, cudaMemcpyHostToDevice));
    if (!rc) rc = cuda_status(cudaMemcpy(gr->mem + cb + eb, vhat.data(), vb, cudaMemcpyHostToDevice));
    if (!rc && mb) rc = cuda_status(cudaMemcpy(gr->mem + cb + eb + vb, mask.data(), mb, cudaMemcpyHostToDevice));
    if (rc) {
        mc_gnn_graph_destroy(gr);
        return rc;
    }
    gr->g.n = N;
    gr->g.col = reinterpret_cast<const int *>(gr->mem);
    gr->g.edge = reinterpret_cast<const __nv_bfloat162 *>(gr->mem + cb);
    gr->g.vhat = reinterpret_cast<const float *>(gr->mem + cb + eb);
    gr->g.affine = aff.affine && !gnn_force_general();
    for (int k = 0; k < 6; k++) {
        gr->g.doff[k] = aff.doff[k];
        gr->g.ebits[k] = aff.ebits[k];
    }
    gr->g.mask = mb ? reinterpret_cast<const uint8_t *>(gr->mem + cb + eb + vb) : nullptr;
    *out = gr;
    return MC_OK;
}

int mc_gnn_graph_destroy(mc_gnn_graph *gr)
{
    if (!gr) return MC_ERR_ARG;
    cudaSetDevice(gr->dev);
    if (gr->mem) cudaFree(gr->mem);
    delete gr;
    return MC_OK;
}

int mc_gnn_graph_export(const mc_gnn_graph *gr, int *n, int *col, uint32_t *edge, float *vhat)
{
    if (!gr || !n) return MC_ERR_ARG;
    *n = gr->g.n;
    const size_t N = (size_t)gr->g.n;
    GNN_TRY(cudaSetDevice(gr->dev));
    if (col) GNN_TRY(cudaMemcpy(col, gr->g.col, 6 * N * 4, cudaMemcpyDeviceToHost));
    if (edge) GNN_TRY(cudaMemcpy(edge, gr->g.edge, 6 * N * 4, cudaMemcpyDeviceToHost));
    if (vhat) GNN_TRY(cudaMemcpy(vhat, gr->g.vhat, N * 4, cudaMemcpyDeviceToHost));
    return MC_OK;
}

int mc_gnn_predict(mc_gnn *net, const mc_gnn_graph *gr, const mc_gnn_sample *s, float *y, double *x0)
{
    if (!net || !gr || !s || !s->rhs || !s->diag) return MC_ERR_ARG;
    GNN_TRY(cudaSetDevice(net->dev));
    int rc = ensure_work(net, gr->g.n);
    if (rc) return rc;
    gnn_forward<float>(net->stream, gr->g, input_of(*s), net->p, net->pk, net->work, x0);
    if (y) GNN_TRY(cudaMemcpyAsync(y, net->work.y, (size_t)gr->g.n * 4, cudaMemcpyDeviceToDevice, net->stream));
    GNN_TRY(cudaGetLastError());
    int status = 0;
    GNN_TRY(cudaMemcpyAsync(&status, net->work.status, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
    GNN_TRY(cudaStreamSynchronize(net->stream));
    return status ? MC_ERR_TIMEOUT : MC_OK;
}

int mc_gnn_loss_grad(mc_gnn *net, const mc_gnn_graph *gr, int batch, const mc_gnn_sample *samples, double *loss,
                     float *host_grad)
{
    if (!net || !gr || batch <= 0 || !samples) return MC_ERR_ARG;
    for (int b = 0; b < batch; b++)
        if (!samples[b].rhs || !samples[b].diag || !samples[b].target) return MC_ERR_ARG;
    GNN_TRY(cudaSetDevice(net->dev));
    int rc = ensure_work(net, gr->g.n);
    if (rc) return rc;
    GNN_TRY(cudaMemsetAsync(net->grad, 0, (size_t)GNN_NPARAM * 4, net->stream));
    double total = 0.0;
    for (int b = 0; b < batch; b++) {
        gnn_loss_backward(net->stream, gr->g, input_of(samples[b]), samples[b].target, net->p, net->pk, net->work,
                          net->grad, 1.0f / batch);
        GNN_TRY(cudaGetLastError());
        GNN_TRY(cudaMemcpyAsync(net->h_loss, net->work.loss, 2 * sizeof(double), cudaMemcpyDeviceToHost, net->stream));
        GNN_TRY(cudaStreamSynchronize(net->stream));
        total += net->h_loss[1];
    }
    if (loss) *loss = total / batch;
    if (host_grad) {
        GNN_TRY(cudaMemcpyAsync(host_grad, net->grad, (size_t)GNN_NPARAM * 4, cudaMemcpyDeviceToHost, net->stream));
        GNN_TRY(cudaStreamSynchronize(net->stream));
    }
    return MC_OK;
}

int mc_gnn_adam_step(mc_gnn *net, float lr)
{
    if (!net || !(lr > 0)) return MC_ERR_ARG;
    GNN_TRY(cudaSetDevice(net->dev));
    net->t++;
    gnn_adam(net->stream, net->p, net->grad, net->m, net->v, lr, 0.9f, 0.999f, 1e-8f, net->t);
    gnn_pack(net->stream, net->p, net->pk);
    GNN_TRY(cudaGetLastError());
    GNN_TRY(cudaStreamSynchronize(net->stream));
    return MC_OK;
}

int mc_gnn_train_step(mc_gnn *net, const mc_gnn_graph *gr, int batch, const mc_gnn_sample *samples, float lr,
                      double *loss)
{
    const int rc = mc_gnn_loss_grad(net, gr, batch, samples, loss, nullptr);
    return rc ? rc : mc_gnn_adam_step(net, lr);
}

} // extern "C"
