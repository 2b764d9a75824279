"""The learned-guess kernels (forward, backward, Adam) through the C ABI,
against the CPU FP64 network (oracle/gnn_oracle.py).

Tolerances: the device keeps activations and GEMM operands in BF16 with FP32
accumulation.  Against the oracle run with the same BF16 roundings the
outputs and gradients agree to 1e-2 (relative 2-norm per parameter group;
isolated roundings that fall the other way at a BF16 midpoint are the only
source of difference); against the plain FP64 oracle to 5e-2 overall and 1e-1 per group.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import gnn_oracle as G  # noqa: E402

from minicombust_app_b200 import flow, gnn  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b, floor=1e-300):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), floor)


def groups():
    out = {"We": slice(G.GP_WE, G.GP_CE), "ce": slice(G.GP_CE, G.GP_LAYER0)}
    for l in range(G.L):
        b = G.GP_LAYER0 + l * G.GPL_SIZE
        for name, lo, hi in (("Wg", G.GPL_WG, G.GPL_CG), ("cg", G.GPL_CG, G.GPL_W1), ("W1", G.GPL_W1, G.GPL_C1),
                             ("c1", G.GPL_C1, G.GPL_W2), ("W2", G.GPL_W2, G.GPL_C2), ("c2", G.GPL_C2, G.GPL_SIZE)):
            out[f"{name}{l}"] = slice(b + lo, b + hi)
    d = G.GP_DEC
    out.update({"Wd": slice(d + G.GPD_WD, d + G.GPD_CD), "cd": slice(d + G.GPD_CD, d + G.GPD_WO),
                "wo": slice(d + G.GPD_WO, d + G.GPD_CO), "co": slice(d + G.GPD_CO, d + G.GPD_CO + 1)})
    return out


def setup(dims, seed=0, nsamples=2, local_target=False):
    import torch
    net = gnn.GuessNet(seed=seed)
    mesh = flow.Mesh.box(*dims, 0.2, 0.1, 0.1)
    gr = net.graph(mesh)
    col, edge, vhat = gr.export()
    graph = G.graph_from_arrays(col, edge, vhat)
    n = mesh.n_cells
    rng = np.random.default_rng(seed + 100)
    host, dev = [], []
    for s in range(nsamples):
        b = rng.standard_normal(n).astype(np.float32)
        b -= b.mean()
        diag = rng.uniform(1.0, 3.0, n).astype(np.float32)
        prev = (0.3 * rng.standard_normal(n)).astype(np.float32)
        target = np.cumsum(rng.standard_normal(n)).astype(np.float32) * 1e-2
        if local_target:  # a function of the cell's own inputs: learnable
            target = (b / diag + prev).astype(np.float32)
        host.append((b, diag, prev, target))
        dev.append(tuple(torch.tensor(a, device="cuda") for a in (b, diag, prev, target)))
    return net, gr, graph, host, dev


def test_graph_export_matches_the_mesh(gpu):
    net = gnn.GuessNet()
    mesh = flow.Mesh.box(7, 4, 3, 0.2, 0.1, 0.1)
    col, edge, vhat = net.graph(mesh).export()
    n = mesh.n_cells
    nb = mesh.cell_neighbours  # uint64, UINT64_MAX on the boundary
    for i in range(n):
        want = sorted(int(j) for j in nb[i] if j < n)
        got = sorted(int(j) for j in col[:, i] if j != i)
        assert got == want
    assert np.all(edge[col == np.arange(n)[None, :]] == 0)
    g = G.graph_from_arrays(col, edge, vhat)
    internal = col != np.arange(n)[None, :]
    assert np.allclose(g["edge"][internal].mean(axis=0), 1.0, rtol=1e-2)
    assert abs(vhat.mean() - 1.0) < 1e-6


@pytest.mark.parametrize("gather", ["offset", "general"])
@pytest.mark.parametrize("dims", [(16, 8, 8), (9, 5, 3)])
def test_forward_matches_oracle(gpu, dims, gather, monkeypatch):
    """Both gathers: the constant-offset form of a box mesh and the general column list."""
    import torch
    if gather == "general":
        monkeypatch.setenv("MC_GNN_GENERAL_GATHER", "1")
    net, gr, graph, host, dev = setup(dims, seed=1)
    p = net.params().astype(np.float64)
    b, diag, prev, _ = host[0]
    n = len(b)
    y = torch.empty(n, device="cuda")
    x0 = torch.empty(n, device="cuda", dtype=torch.float64)
    net.predict(gr, dev[0][0], dev[0][1], dev[0][2], y=y, x0=x0)
    y_bf, cache = G.forward(p, graph, b, diag, prev, bf16=True)
    y_64, _ = G.forward(p, graph, b, diag, prev, bf16=False)
    assert rel(y.cpu().numpy(), y_bf) <= 1e-2
    assert rel(y.cpu().numpy(), y_64) <= 5e-2
    assert np.allclose(x0.cpu().numpy(), cache["sx"] * y.cpu().numpy().astype(np.float64), rtol=1e-6)


@pytest.mark.parametrize("dims", [(16, 8, 8), (9, 5, 3)])
def test_gradient_matches_oracle(gpu, dims):
    net, gr, graph, host, dev = setup(dims, seed=2)
    # move away from the initialisation so every ReLU branch is exercised
    rng = np.random.default_rng(5)
    p = (net.params() + 0.05 * rng.standard_normal(G.NPARAM)).astype(np.float32)
    net.set_params(p)
    loss, grad = net.loss_grad(gr, dev)
    l_bf, g_bf = G.loss_grad(p.astype(np.float64), graph, host, bf16=True)
    l_64, g_64 = G.loss_grad(p.astype(np.float64), graph, host, bf16=False)
    assert abs(loss - l_bf) <= 1e-2 * l_bf
    assert abs(loss - l_64) <= 5e-2 * l_64
    # a group whose exact gradient vanishes (co: the loss ignores a constant
    # offset) is compared against the scale of the whole gradient
    floor = 1e-4 * np.linalg.norm(g_64)
    for name, sl in groups().items():
        assert rel(grad[sl], g_bf[sl], floor) <= 1e-2, (name, rel(grad[sl], g_bf[sl], floor))
        assert rel(grad[sl], g_64[sl], floor) <= 1e-1, (name, rel(grad[sl], g_64[sl], floor))
    assert rel(grad, g_64) <= 5e-2


def test_adam_training_reduces_the_loss(gpu):
    net, gr, graph, host, dev = setup((16, 8, 8), seed=3, nsamples=4, local_target=True)
    first = net.loss_grad(gr, dev, want_grad=False)[0]
    for _ in range(60):
        last = net.train_step(gr, dev, 2e-3)
    assert last < 0.5 * first
    # deterministic: same seed, same steps, same parameters
    net2, gr2, _, _, dev2 = setup((16, 8, 8), seed=3, nsamples=4, local_target=True)
    for _ in range(60):
        net2.train_step(gr2, dev2, 2e-3)
    assert np.array_equal(net.params(), net2.params())


@pytest.mark.parametrize("layer", ["umma", "mma"])
@pytest.mark.parametrize("dims", [(16, 8, 8), (9, 5, 3)])
def test_offset_layer_kernels_match_oracle(gpu, dims, layer, monkeypatch):
    """Both offset-form layer kernels -- tcgen05 (TMA tiles, TMEM accumulators)
    and mma.sync -- explicitly selected, against the BF16-emulating oracle."""
    import torch
    monkeypatch.setenv("MC_GNN_LAYER", layer)
    net, gr, graph, host, dev = setup(dims, seed=4)
    p = net.params().astype(np.float64)
    b, diag, prev, _ = host[0]
    y = torch.empty(len(b), device="cuda")
    net.predict(gr, dev[0][0], dev[0][1], dev[0][2], y=y)
    y_bf, _ = G.forward(p, graph, b, diag, prev, bf16=True)
    assert rel(y.cpu().numpy(), y_bf) <= 1e-2


def test_tensor_core_layer_matches_mma_layer_on_many_tiles(gpu, monkeypatch):
    """65,536 cells = 512 tiles: every persistent block runs several tiles, so
    the three copy stages and both epilogue groups wrap their barrier phases."""
    import torch
    net, gr, graph, host, dev = setup((64, 32, 32), seed=5, nsamples=1)
    rng = np.random.default_rng(9)
    net.set_params((net.params() + 0.05 * rng.standard_normal(G.NPARAM)).astype(np.float32))
    n = len(host[0][0])
    ys = {}
    for layer in ("umma", "mma"):
        monkeypatch.setenv("MC_GNN_LAYER", layer)
        y = torch.empty(n, device="cuda")
        net.predict(gr, dev[0][0], dev[0][1], dev[0][2], y=y)
        ys[layer] = y.cpu().numpy().astype(np.float64)
    # same BF16 operands, FP32 accumulation in a different order: the layer
    # outputs differ only where a BF16 rounding falls the other way
    assert rel(ys["umma"], ys["mma"]) <= 1e-2
    assert np.mean(np.abs(ys["umma"] - ys["mma"]) <= 1e-2 * np.abs(ys["mma"]).max()) > 0.99
