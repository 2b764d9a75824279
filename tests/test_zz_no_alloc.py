"""The allocation-free solve (mc_solve_bicgstab_noalloc).

Some callers cannot allocate device memory: code that issues work while a
CUDA stream capture is in progress (cudaMalloc is not permitted then), and
hosts that own all device memory through their own pool or budget.  For them
the library offers one entry point that takes every scratch byte from a
file-scope device array instead of cudaMalloc.

This test solves the temperature system that the handle-based temperature
stage (mc_flow_stage_temperature, the existing entry point) assembled and
solved, this time through the allocation-free entry point on caller-owned
device arrays, twice in a row (the second call reuses the array the first
left behind), and compares both solutions with the stage's result within the
parity tolerance of the other GPU tests.  The file is named so that pytest
collects it last.
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
    too_big = L.MC_SOLVE_NOALLOC_MAX_ROWS if hasattr(L, "MC_SOLVE_NOALLOC_MAX_ROWS") else 262144
    rc = L.mc_solve_bicgstab_noalloc(too_big + 1, d_diag.data_ptr(), d_off.data_ptr(), d_col.data_ptr(),
                                     d_b.data_ptr(), d_b.data_ptr(), 1e-8, 10, None, None)
    assert rc == flow.MC_ERR_ARG
    solver.close()
