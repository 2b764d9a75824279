"""The snapshot dataset writer (mc_flow_snapshot_open/close): header, record
count and layout, read back and checked against the solver's own state, in
natural and RCM cell order (records are in the caller's numbering)."""
import os

import numpy as np
import pytest

from checkers import noisy_initial_fields
from minicombust_app_b200 import flow

pytestmark = pytest.mark.gpu

BASE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 1500.0}


@pytest.mark.parametrize("reorder", [flow.REORDER_NONE, flow.REORDER_RCM], ids=["natural", "rcm"])
def test_snapshot_records(gpu, tmp_path, reorder):
    dims = (16, 8, 8)
    mesh = flow.Mesh.box(*dims, 0.2, 0.1, 0.1)
    s = flow.FlowSolver(mesh, params=flow.default_params(flow.MODE_SIMPLE, pressure_solver=flow.PSOLVER_PCG_AMG,
                                                         initial_guess=flow.GUESS_PREVIOUS, reorder=reorder))
    for name, vals in noisy_initial_fields(s.N, BASE, 4).items():
        a = s.field(name)
        a[:s.N] = vals
        s.set_field(name, a)
    path = str(tmp_path / "snap.bin")
    max_records = 3
    s.snapshot_open(path, max_records)
    pp_after = []
    solves = 0
    for _ in range(4):
        s.simple_iteration()
        solves += s.last_stats.pressure_solves
        pp_after.append(s.field("PP")[:s.N].copy())
    diag = s.cell_array(1)
    s.snapshot_close()
    s.close()

    with open(path, "rb") as f:
        head = f.read(64)
    assert head[:8] == flow.SNAPSHOT_MAGIC
    version, cells, fields, dtype = np.frombuffer(head[8:24], dtype=np.uint32)
    records = int(np.frombuffer(head[24:32], dtype=np.uint64)[0])
    assert (version, cells, fields, dtype) == (1, s.N, 4, 0)
    assert records == min(max_records, solves)
    assert head[32:] == bytes(32)
    assert os.path.getsize(path) == 64 + records * 4 * s.N * 4
    data = flow.read_snapshots(path)
    assert data.shape == (records, 4, s.N)
    assert np.isfinite(data).all()
    # right-hand sides are projected to mean zero; diagonals are the
    # pressure-correction diagonal (unchanged within a pass) in the caller's order
    for r in range(records):
        assert abs(float(data[r, 0].astype(np.float64).mean())) <= 1e-6 * float(np.abs(data[r, 0]).max())
    assert np.allclose(data[-1, 1], diag.astype(np.float32), rtol=1e-6)
    # record k's "previous correction" is record k-1's correction
    for r in range(1, records):
        assert np.array_equal(data[r, 2], data[r - 1, 3])
    assert not np.any(data[0, 2])  # nothing before the first solve
