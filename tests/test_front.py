"""The reference-side C++ front (include/flow_b200/FlowSolver.inl): the
reference's FlowSolver<double> class over the C ABI, compiled against the
reference's own headers with the mesh from its own load_mesh
(src/examples/mesh_examples.cpp:120), driven by the flow branch of its
driver loop (tests/front/front_driver.cpp, built into oracle/_ref by
oracle/Makefile, target front).

On the GPU: two FlowSolver::timestep() calls (six SIMPLE passes) through the
front against the reference's own FlowSolver (oracle/_ref/libmcref.so) from
the constructor's initial state, all 13 fields within the parity gate.
Without a GPU: the front and the reference's mesh code link and run up to
the first device call, which fails with the library's status, not a crash.
"""
import os
import subprocess

import numpy as np
import pytest

from checkers import Reference, ref_available
from conftest import gpu_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "front_driver")
ALL_FIELDS = ("U", "V", "W", "P", "PP", "TE", "ED", "TP", "TEM", "FUL", "PRO", "VARF", "VARP")
needs_driver = pytest.mark.skipif(not os.path.exists(DRIVER), reason="front driver not built (needs the reference tree)")


@needs_driver
def test_front_links_and_reports_status_without_gpu(tmp_path):
    if gpu_available():
        pytest.skip("a GPU is present: the GPU test covers the front")
    r = subprocess.run([DRIVER, "4", "2", "2", "0.1", "0.05", "0.05", "1", str(tmp_path / "f.bin")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "mc_flow_create: CUDA error" in r.stderr


@pytest.mark.gpu
@needs_driver
@pytest.mark.skipif(not ref_available(), reason="reference not compiled here (oracle/_ref)")
def test_front_timesteps_match_reference(gpu, tmp_path):
    dims, L = (20, 10, 10), (0.2, 0.1, 0.1)
    out = tmp_path / "fields.bin"
    os.makedirs(tmp_path / "out" / "flow", exist_ok=True)
    r = subprocess.run([DRIVER, *map(str, dims), *map(str, L), "2", str(out), "vtk"], capture_output=True, text=True,
                       timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    ref = Reference(*dims, *L)
    n = ref.phi_len
    got = np.fromfile(out, dtype=np.float64).reshape(13, n)
    for _ in range(2):
        ref.timestep()
    for k, name in enumerate(ALL_FIELDS):
        want = ref.field(name)
        err = np.abs(got[k] - want).max() / max(np.abs(want).max(), 1e-300)
        assert err <= 1e-9, (name, err)
    # output_data wrote the reference's VTK file for each timestep
    for t in (1, 2):
        assert (tmp_path / "out" / "flow" / f"minicombust_flow0_timestep{t}.vtk").exists()
