"""Pins of the CPU FP64 network (oracle/gnn_oracle.py), the checker of the
library's learned-guess kernels: its analytic gradient against central
finite differences, and its BF16 rounding against torch's."""
import os
import sys

import numpy as np
import pytest
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import gnn_oracle as G  # noqa: E402

from minicombust_app_b200 import flow, gnn  # noqa: E402


def box_graph(ex, ey, ez, seed=0):
    """Graph of a box mesh built from the mesh arrays (slot order = cell_faces order)."""
    mesh = flow.Mesh.box(ex, ey, ez, 0.1 * ex, 0.1 * ey, 0.1 * ez)
    n = mesh.n_cells
    nb = mesh.cell_neighbours  # uint64, UINT64_MAX on the boundary
    col = np.where(nb < n, nb, np.arange(n, dtype=np.uint64)[:, None]).astype(np.int64).T.copy()
    rng = np.random.default_rng(seed)
    face_feat = G.bf16_round(rng.uniform(0.5, 1.5, size=(mesh.n_faces, 2)))
    edge = face_feat[mesh.cell_faces.astype(np.int64)].transpose(1, 0, 2)   # [6][n][2], same value on both sides
    edge = np.where((col != np.arange(n))[:, :, None], edge, 0.0)
    vhat = np.ones(n)
    return {"col": col, "edge": edge, "vhat": vhat}, mesh


def sample(n, seed):
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(n)
    b -= b.mean()
    diag = rng.uniform(1.0, 2.0, n)
    prev = 0.1 * rng.standard_normal(n)
    target = rng.standard_normal(n)
    return b, diag, prev, target


def test_param_count_matches_library():
    assert gnn.param_count() == G.NPARAM


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).standard_normal(10000) * np.logspace(-20, 20, 10000)
    x = np.concatenate([x, [0.0, -0.0, 1.0, 1.00390625, 1.0078125 + 2 ** -9, 3.4e38]])
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(G.bf16_round(x), ref)


@pytest.mark.parametrize("bf16", [False])
def test_oracle_gradient_matches_finite_differences(bf16):
    graph, _ = box_graph(4, 3, 2)
    n = graph["col"].shape[1]
    rng = np.random.default_rng(3)
    p = rng.standard_normal(G.NPARAM) * 0.3
    samples = [sample(n, 10), sample(n, 11)]
    loss, grad = G.loss_grad(p, graph, samples, bf16=bf16)
    assert np.isfinite(loss) and loss > 0
    idx = np.concatenate([rng.choice(G.NPARAM, 60, replace=False),
                          [G.GP_WE, G.GP_CE, G.GP_LAYER0 + G.GPL_WG, G.GP_LAYER0 + G.GPL_CG, G.GP_DEC + G.GPD_CO]])
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (G.loss_grad(pp, graph, samples)[0] - G.loss_grad(pm, graph, samples)[0]) / (2 * eps)
        noise = 1e-14 * abs(loss) / eps  # rounding of the two loss evaluations
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)) + noise, (i, fd, grad[i])


def test_oracle_loss_ignores_a_constant_offset():
    graph, _ = box_graph(3, 3, 2)
    n = graph["col"].shape[1]
    p = np.random.default_rng(4).standard_normal(G.NPARAM) * 0.3
    b, d, pr, t = sample(n, 5)
    l1, _ = G.loss_grad(p, graph, [(b, d, pr, t)])
    l2, _ = G.loss_grad(p, graph, [(b, d, pr, t + 7.0)])
    assert abs(l1 - l2) <= 1e-12 * max(1.0, l1)
