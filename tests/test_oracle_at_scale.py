"""The GPU path against the CPU oracle at a benchmark size, not only at
16,000 cells: the 2*64^3 = 524,288-cell box of the second benchmark
configuration (200 seeded source blobs, simple-mode physics, pressure PCG
with the aggregation-AMG V-cycle, RCM cell order), 5 SIMPLE passes with every
solve at 1e-12 on both sides, max relative difference <= 1e-9 per field.
The oracle's passes take about half a minute of host CPU.
"""
import numpy as np
import pytest

from checkers import SIMPLE, Oracle, oracle_mesh, oracle_params
from minicombust_app_b200 import flow
from minicombust_app_b200.workload import gaussian_blobs, noisy_fields

pytestmark = pytest.mark.gpu

FIELDS = ("U", "V", "W", "P", "TEM")


@pytest.mark.parametrize("precision", [flow.PRECISION_FP64, flow.PRECISION_FP32_REFINED], ids=["fp64", "fp32_refined"])
def test_config2_box_five_passes_match_oracle(gpu, precision):
    m = 64
    dims, lengths = (2 * m, m, m), (0.2, 0.1, 0.1)
    orc = Oracle(oracle_mesh(*dims, *lengths), oracle_params(SIMPLE, u_rtol=1e-12, p_rtol=1e-12))
    solver = flow.FlowSolver(flow.Mesh.box(*dims, *lengths),
                             params=flow.default_params(flow.MODE_SIMPLE, u_rtol=1e-12, p_rtol=1e-12,
                                                        pressure_solver=flow.PSOLVER_PCG_AMG,
                                                        precision=precision, reorder=flow.REORDER_RCM))
    assert not np.array_equal(solver.cell_order(), np.arange(solver.N))
    for name, vals in noisy_fields(solver.N, seed=0).items():
        for obj in (solver, orc):
            a = obj.field(name)
            a[:solver.N] = vals
            obj.set_field(name, a)
    src = gaussian_blobs(dims, lengths, 200, seed=0)
    solver.set_sources(src)
    orc.set_sources(src)
    for _ in range(5):
        solver.simple_iteration()
        assert orc.step() == 0
    errs = {}
    for name in FIELDS:
        a, b = solver.field(name), orc.field(name)
        errs[name] = float(np.abs(a - b).max() / np.abs(b).max())
    print(f"\n2*64^3, 5 passes, precision {precision}: max relative difference per field {errs}")
    assert max(errs.values()) <= 1e-9, errs
