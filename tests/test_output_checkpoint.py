"""VTK field output and checkpoint / resume (the reference's output path,
FlowSolver::output_data -> VisitWriter<T>::write_flow, VisitWriter.hpp:127-234;
checkpoints have no reference counterpart).

The VTK file written by the library for given fields is compared byte for
byte with the file the reference's own writer produces for the same fields
(oracle/_ref; skipped where the reference was not compiled).  A run
interrupted by a checkpoint and resumed in a new handle must give the
uninterrupted run's fields: bit for bit with the Jacobi-PCG path, within the
parity gate where the AMG coarsest inverse of the resumed handle is formed
afresh instead of carried from the previous pass.
"""
import os

import numpy as np
import pytest

from checkers import Reference, noisy_initial_fields, ref_available
from minicombust_app_b200 import flow

ALL_FIELDS = ("U", "V", "W", "P", "PP", "TE", "ED", "TP", "TEM", "FUL", "PRO", "VARF", "VARP")
BASE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 2000.0}


def seed(obj, n, base=BASE, s=0):
    for name, vals in noisy_initial_fields(n, base, s).items():
        a = obj.field(name)
        a[:n] = vals
        obj.set_field(name, a)


@pytest.mark.gpu
@pytest.mark.skipif(not ref_available(), reason="reference not compiled here (oracle/_ref)")
@pytest.mark.parametrize("reorder", [flow.REORDER_NONE, flow.REORDER_RCM], ids=["natural", "rcm"])
def test_vtk_matches_reference_writer_byte_for_byte(gpu, tmp_path, reorder):
    dims, L = (10, 4, 3), (0.1, 0.05, 0.04)
    ref = Reference(*dims, *L)
    seed(ref, ref.N)
    for _ in range(2):
        ref.step()
    solver = flow.FlowSolver(flow.Mesh.box(*dims, *L), params=flow.default_params(flow.MODE_COMPAT, reorder=reorder))
    for name in ALL_FIELDS:
        solver.set_field(name, ref.field(name))
    want = ref.write_flow(str(tmp_path / "ref"), 7)
    got = solver.output_data(7, prefix=str(tmp_path / "b200"))
    assert os.path.basename(got) == "b200_flow0_timestep7.vtk"
    with open(want, "rb") as a, open(got, "rb") as b:
        assert a.read() == b.read()


def run_passes(solver, k):
    for _ in range(k):
        solver.simple_iteration()


@pytest.mark.gpu
@pytest.mark.parametrize("mode,kw,exact", [
    (flow.MODE_COMPAT, {}, True),
    (flow.MODE_COMPAT, {"reorder": flow.REORDER_RCM}, True),
    (flow.MODE_SIMPLE, {"pressure_solver": flow.PSOLVER_PCG_AMG, "precision": flow.PRECISION_FP32_REFINED,
                        "initial_guess": flow.GUESS_PREVIOUS, "u_rtol": 1e-12, "p_rtol": 1e-12}, False),
], ids=["compat", "compat_rcm", "simple_refined_amg"])
def test_resume_continues_the_run(gpu, tmp_path, mode, kw, exact):
    dims, L = (12, 6, 5), (0.2, 0.1, 0.1)
    mesh = flow.Mesh.box(*dims, *L)
    p = flow.default_params(mode, **kw)
    base = BASE if mode == flow.MODE_COMPAT else dict(BASE, TEM=1500.0)
    a = flow.FlowSolver(mesh, params=p)
    seed(a, a.N, base)
    run_passes(a, 4)  # crosses a timestep boundary (3 passes per timestep)
    ck = str(tmp_path / "state.ckpt")
    a.checkpoint(ck)
    run_passes(a, 4)
    b = flow.FlowSolver(mesh, params=p)
    b.resume(ck)
    run_passes(b, 4)
    names = [n for n in ALL_FIELDS if p.transport_scalars or n in ("U", "V", "W", "P", "PP", "TEM")]
    for n in names:
        x, y = a.field(n), b.field(n)
        if exact:
            assert np.array_equal(x, y), n
        else:
            assert np.abs(x - y).max() <= 1e-9 * max(np.abs(x).max(), 1e-300), n
    assert np.array_equal(a.face_array(0), b.face_array(0)) or not exact


@pytest.mark.gpu
def test_resume_refuses_another_configuration(gpu, tmp_path):
    mesh = flow.Mesh.box(6, 3, 3, 0.1, 0.05, 0.05)
    a = flow.FlowSolver(mesh, params=flow.default_params(flow.MODE_COMPAT))
    ck = str(tmp_path / "a.ckpt")
    a.checkpoint(ck)
    b = flow.FlowSolver(mesh, params=flow.default_params(flow.MODE_SIMPLE))
    with pytest.raises(flow.FlowError) as e:
        b.resume(ck)
    assert e.value.status == flow.MC_ERR_ARG
    c = flow.FlowSolver(flow.Mesh.box(7, 3, 3, 0.1, 0.05, 0.05), params=flow.default_params(flow.MODE_COMPAT))
    with pytest.raises(flow.FlowError):
        c.resume(ck)
    with open(ck, "r+b") as f:  # a damaged header
        f.write(b"XXXX")
    with pytest.raises(flow.FlowError):
        a.resume(ck)
