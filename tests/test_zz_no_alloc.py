"""The allocation-free solve (mc_solve_bicgstab_noalloc).

Some callers cannot allocate device memory: hosts that hand all device memory
to their own pool or fixed budget at start-up (a cudaMalloc from a library
fails there, or takes memory the host promised elsewhere), and time-critical
loops where cudaMalloc and cudaFree would synchronise the device.  For them
the library offers one entry point that takes every scratch byte from a
file-scope device array instead of cudaMalloc.

This test solves the temperature system that the handle-based temperature
stage (mc_flow_stage_temperature, the existing entry point) assembled and
solved, this time through the allocation-free entry point on caller-owned
device arrays, twice in a row (the second call reuses the array the first
left behind), and compares both solutions with the stage's result within the
parity tolerance of the other GPU tests.  A second test solves a system of
exactly the stated maximum size (the limit read from the header) and checks
its residual on the CPU, so the partitioning of the array is exercised at the
edge.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from checkers import noisy_initial_fields
from minicombust_app_b200 import flow

pytestmark = pytest.mark.gpu

PARITY = 1e-9


def ell_from_csr(rp, col, val):
    """The library's ELL layout: diag[n], off[6][n], col[6][n], unused slots
    pointing at their own row with value 0."""
    n = len(rp) - 1
    diag = np.zeros(n)
    off = np.zeros((6, n))
    ecol = np.tile(np.arange(n, dtype=np.int32), (6, 1))
    for i in range(n):
        k = 0
        for j in range(rp[i], rp[i + 1]):
            if col[j] == i:
                diag[i] = val[j]
            else:
                off[k, i] = val[j]
                ecol[k, i] = col[j]
                k += 1
    return diag, off, ecol


def test_noalloc_solve_matches_temperature_stage(gpu):
    import torch

    mesh = flow.Mesh.box(32, 16, 16, 0.2, 0.1, 0.1)
    params = flow.default_params(flow.MODE_SIMPLE, u_rtol=1e-12, p_rtol=1e-10)
    solver = flow.FlowSolver(mesh, params=params)
    base = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 1500.0}
    for name, vals in noisy_initial_fields(solver.N, base, 7).items():
        a = solver.field(name)
        a[:solver.N] = vals
        solver.set_field(name, a)
    for stage in ("gradients", "set_up_field", "momentum", "pressure", "temperature"):
        solver.stage(stage)
    n = solver.N
    expected = solver.field("TEM")[:n]
    rp, col, val, rhs = solver.csr(flow.SYSTEM_TEMPERATURE)
    diag, off, ecol = ell_from_csr(rp, col, val)

    dev = torch.device("cuda", 0)
    d_diag = torch.from_numpy(diag).to(dev)
    d_off = torch.from_numpy(np.ascontiguousarray(off)).to(dev)
    d_col = torch.from_numpy(np.ascontiguousarray(ecol)).to(dev)
    d_b = torch.from_numpy(rhs).to(dev)
    L = flow.library()
    for call in range(2):
        x = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        its = ctypes.c_int(-1)
        rc = L.mc_solve_bicgstab_noalloc(n, d_diag.data_ptr(), d_off.data_ptr(), d_col.data_ptr(), d_b.data_ptr(),
                                         x.data_ptr(), params.u_rtol, params.max_iters, None, ctypes.byref(its))
        assert rc == flow.MC_OK, (call, rc)
        assert its.value > 0
        got = x.cpu().numpy()
        err = np.abs(got - expected).max() / np.abs(expected).max()
        assert err <= PARITY, (call, err)

    # sizes beyond the stated maximum are refused before anything runs
    too_big = flow.header_define("MC_SOLVE_NOALLOC_MAX_ROWS")
    rc = L.mc_solve_bicgstab_noalloc(too_big + 1, d_diag.data_ptr(), d_off.data_ptr(), d_col.data_ptr(),
                                     d_b.data_ptr(), d_b.data_ptr(), 1e-8, 10, None, None)
    assert rc == flow.MC_ERR_ARG
    solver.close()


def test_noalloc_solve_at_the_size_limit(gpu):
    """A 7-point system of exactly MC_SOLVE_NOALLOC_MAX_ROWS rows (a 64^3 grid,
    diagonally dominant, non-symmetric) solved twice; the true residual is
    checked in FP64 on the CPU."""
    import torch

    n = flow.header_define("MC_SOLVE_NOALLOC_MAX_ROWS")
    m = round(n ** (1.0 / 3.0))
    assert m ** 3 == n
    rng = np.random.default_rng(11)
    idx = np.arange(n, dtype=np.int64)
    i, j, k = idx % m, (idx // m) % m, idx // (m * m)
    steps = [(i > 0, -1), (i < m - 1, 1), (j > 0, -m), (j < m - 1, m), (k > 0, -m * m), (k < m - 1, m * m)]
    off = np.zeros((6, n))
    ecol = np.tile(idx.astype(np.int32), (6, 1))
    for s, (ok, d) in enumerate(steps):
        off[s, ok] = -(0.8 + 0.4 * rng.random(int(ok.sum())))
        ecol[s, ok] = (idx[ok] + d).astype(np.int32)
    diag = 1.05 * np.abs(off).sum(axis=0) + 0.1
    b = rng.standard_normal(n)

    dev = torch.device("cuda", 0)
    d_diag = torch.from_numpy(diag).to(dev)
    d_off = torch.from_numpy(np.ascontiguousarray(off)).to(dev)
    d_col = torch.from_numpy(np.ascontiguousarray(ecol)).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    L = flow.library()
    rtol = 1e-10
    for call in range(2):
        x = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        its = ctypes.c_int(-1)
        rc = L.mc_solve_bicgstab_noalloc(n, d_diag.data_ptr(), d_off.data_ptr(), d_col.data_ptr(), d_b.data_ptr(),
                                         x.data_ptr(), rtol, 2000, None, ctypes.byref(its))
        assert rc == flow.MC_OK, (call, rc)
        got = x.cpu().numpy()
        ax = diag * got + (off * got[ecol]).sum(axis=0)
        rel = np.linalg.norm(b - ax) / np.linalg.norm(b)
        assert rel <= 10 * rtol, (call, rel, its.value)
