"""The boundary's status codes on failure paths.

The reference reports nothing here: a Krylov solve that stops short is only
printed (FlowSolver.inl:1355-1360, :2255-2260) and a CUDA error exits the
process (gpu_kernels.cu:24-32).  Each call of this library returns a status
instead, and these tests provoke each one in a form that faults no GPU: a
mesh that fails validation on the host, a solve capped at one iteration, a
NaN written into a field, and the learned guess selected without its
parameters.
"""
import ctypes

import numpy as np
import pytest

from checkers import noisy_initial_fields
from minicombust_app_b200 import flow

BASE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 1500.0}


def create_status(mesh, **kw):
    L = flow.library()
    p = flow.default_params(flow.MODE_SIMPLE)
    for k, v in kw.items():
        setattr(p, k, v)
    mv = mesh.view()
    h = ctypes.c_void_p()
    rc = L.mc_flow_create(ctypes.byref(mv), ctypes.byref(p), ctypes.byref(h))
    if rc == flow.MC_OK:
        L.mc_flow_destroy(h)
    return rc


def corrupted(mesh, what):
    m = flow.Mesh(mesh.points, mesh.cell_nodes, mesh.face_cells.copy(), mesh.cell_faces.copy(),
                  mesh.cell_neighbours, mesh.cell_centers, mesh.boundary_types.copy())
    if what == "face_out_of_range":
        m.face_cells[3, 0] = mesh.n_cells + 10
    elif what == "face_order":
        internal = np.where(m.face_cells[:, 1] < mesh.n_cells)[0][0]
        m.face_cells[internal] = m.face_cells[internal][::-1]
    elif what == "boundary_side":
        b = np.where(m.face_cells[:, 1] >= mesh.n_cells)[0][0]
        m.face_cells[b, 1] = mesh.n_cells + 6
    elif what == "cell_faces":
        m.cell_faces[0, 1] = m.cell_faces[0, 0]
    elif what == "boundary_type":
        m.boundary_types[2] = 7
    return m


@pytest.mark.parametrize("what", ["face_out_of_range", "face_order", "boundary_side", "cell_faces",
                                  "boundary_type"])
def test_invalid_mesh_is_rejected_on_the_host(what):
    """Validation runs before any device call, so this runs without a GPU."""
    mesh = flow.Mesh.box(4, 3, 2, 0.1, 0.05, 0.05)
    assert create_status(corrupted(mesh, what)) == flow.MC_ERR_MESH


def test_invalid_params_are_rejected():
    mesh = flow.Mesh.box(4, 3, 2, 0.1, 0.05, 0.05)
    assert create_status(mesh, max_iters=0) == flow.MC_ERR_ARG
    assert create_status(mesh, mode=5) == flow.MC_ERR_ARG
    assert create_status(mesh, precision=flow.PRECISION_FP32_REFINED,
                         pressure_solver=flow.PSOLVER_PCG_JACOBI) == flow.MC_ERR_UNSUPPORTED


def seeded_solver(dims=(16, 8, 8), **kw):
    s = flow.FlowSolver(flow.Mesh.box(*dims, 0.2, 0.1, 0.1), params=flow.default_params(flow.MODE_SIMPLE, **kw))
    for name, vals in noisy_initial_fields(s.N, BASE, 0).items():
        a = s.field(name)
        a[:s.N] = vals
        s.set_field(name, a)
    return s


@pytest.mark.gpu
def test_iteration_cap_reports_not_converged(gpu):
    s = seeded_solver(max_iters=1, u_rtol=1e-13, p_rtol=1e-13)
    rc = s.simple_iteration(check=False)
    assert rc == flow.MC_ERR_NOT_CONVERGED
    st = s.last_stats
    assert st.momentum_iters[0] == 1 and st.pressure_iters_first == 1
    assert 1e-13 < st.pressure_rel_residual_first < 1.0  # the residual it reached, reported
    s.close()


@pytest.mark.gpu
def test_nan_field_reports_nonfinite(gpu):
    s = seeded_solver()
    u = s.field("U")
    u[5] = np.nan
    s.set_field("U", u)
    assert s.simple_iteration(check=False) == flow.MC_ERR_NONFINITE
    s.close()
    # the device is still usable afterwards
    t = seeded_solver()
    assert t.simple_iteration(check=False) == flow.MC_OK
    t.close()


@pytest.mark.gpu
def test_learned_guess_without_parameters_is_an_argument_error(gpu):
    s = seeded_solver(pressure_solver=flow.PSOLVER_PCG_AMG, initial_guess=flow.GUESS_LEARNED)
    assert s.simple_iteration(check=False) == flow.MC_ERR_ARG
    assert b"set_guess_params" in flow.library().mc_flow_last_error(s.h)
    s.close()
