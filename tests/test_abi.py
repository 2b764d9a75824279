"""The C-ABI library loads on a CPU-only machine, exports every entry point
declared in include/*.h (the flow solver and the guess network), and its
host-only parts (parameter defaults, box mesh builder) agree with the
reference/oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from checkers import oracle_mesh
from minicombust_app_b200 import flow

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "minicombust_flow.h")
GNN_HEADER = os.path.join(ROOT, "include", "minicombust_gnn.h")


def declared_symbols(header=HEADER):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = flow.library()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
        assert n in flow._SIGNATURES, f"{n} has no ctypes signature"


def test_library_exports_every_guess_network_symbol():
    from minicombust_app_b200 import gnn
    L = gnn.library()
    names = declared_symbols(GNN_HEADER)
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n
        assert n in gnn._SIGNATURES, f"{n} has no ctypes signature"
    assert L.mc_gnn_param_count() == 14177


def test_default_params_are_reference_constants():
    p = flow.default_params(flow.MODE_COMPAT)
    assert p.viscosity == 0.000014          # FlowSolver.hpp:296
    assert p.density == 1.2                 # FlowSolver.hpp:342
    assert p.inlet_u == 50.0                # Mesh.hpp:114
    assert p.pressure0 == 4000.0            # Mesh.hpp:115
    assert p.temperature0 == 2000.0         # Mesh.hpp:116
    assert p.urf_momentum == 0.5            # FlowSolver.inl:1731
    assert p.urf_pressure == 0.2            # FlowSolver.inl:2425
    assert p.flux_corr == 0.8               # FlowSolver.inl:1871
    assert p.urf_temperature == 0.95        # FlowSolver.inl:2939-2946
    assert p.delta == 1.0e-5                # minicombust.cpp:120
    s = flow.default_params(flow.MODE_SIMPLE)
    assert (s.viscosity, s.temperature0, s.urf_momentum, s.urf_pressure, s.p_rtol) == (1.8e-5, 1500.0, 0.7, 0.3, 1e-8)


@pytest.mark.parametrize("dims,lengths", [((6, 3, 3), (0.06, 0.03, 0.03)), ((40, 20, 20), (0.2, 0.1, 0.1)),
                                          ((1, 1, 1), (1.0, 1.0, 1.0)), ((3, 7, 2), (0.3, 0.7, 0.2))])
def test_box_mesh_matches_oracle(dims, lengths):
    a = flow.Mesh.box(*dims, *lengths)
    b = oracle_mesh(*dims, *lengths)
    assert np.array_equal(a.points, b.points)
    assert np.array_equal(a.cell_nodes, b.cells)
    assert np.array_equal(a.face_cells, b.faces)
    assert np.array_equal(a.cell_faces, b.cell_faces)
    assert np.array_equal(a.cell_neighbours, b.cell_neighbours)
    assert np.array_equal(a.cell_centers, b.cell_centers)
    assert np.array_equal(a.boundary_types, b.boundary_types)


def test_status_strings():
    L = flow.library()
    for s in range(-7, 1):
        assert L.mc_status_string(s)


def test_bad_arguments_are_rejected_without_gpu():
    L = flow.library()
    h = ctypes.c_void_p()
    assert L.mc_flow_create(None, None, ctypes.byref(h)) == flow.MC_ERR_ARG
    mesh = flow.Mesh.box(2, 1, 1, 0.2, 0.1, 0.1)
    mv = mesh.view()
    p = flow.default_params(flow.MODE_SIMPLE)
    p.mode = 7
    assert L.mc_flow_create(ctypes.byref(mv), ctypes.byref(p), ctypes.byref(h)) == flow.MC_ERR_ARG
    p = flow.default_params(flow.MODE_SIMPLE)
    p.max_iters = 0
    assert L.mc_flow_create(ctypes.byref(mv), ctypes.byref(p), ctypes.byref(h)) == flow.MC_ERR_ARG
    assert L.mc_flow_destroy(None) == flow.MC_ERR_ARG
    assert L.mc_flow_simple_iteration(None, None) == flow.MC_ERR_ARG


def test_refinement_floors():
    p = flow.default_params(flow.MODE_SIMPLE)
    assert (p.ir_inner_rtol, p.ir_inner_rtol_bicg) == (1e-5, 1e-4)
    L = flow.library()
    h = ctypes.c_void_p()
    mesh = flow.Mesh.box(2, 1, 1, 0.2, 0.1, 0.1)
    mv = mesh.view()
    for field, bad in (("ir_inner_rtol", 0.0), ("ir_inner_rtol", 1.0), ("ir_inner_rtol_bicg", 0.0),
                       ("ir_inner_rtol_bicg", 2.0)):
        q = flow.default_params(flow.MODE_SIMPLE, pressure_solver=flow.PSOLVER_PCG_AMG,
                                precision=flow.PRECISION_FP32_REFINED)
        setattr(q, field, bad)
        assert L.mc_flow_create(ctypes.byref(mv), ctypes.byref(q), ctypes.byref(h)) == flow.MC_ERR_UNSUPPORTED, field


def test_chebyshev_damping_parameter():
    p = flow.default_params(flow.MODE_SIMPLE)
    assert p.amg_cheb_ratio == 4.0
    L = flow.library()
    h = ctypes.c_void_p()
    mv = flow.Mesh.box(2, 1, 1, 0.2, 0.1, 0.1).view()
    for bad in (0.5, 1.0, -3.0):
        q = flow.default_params(flow.MODE_SIMPLE, pressure_solver=flow.PSOLVER_PCG_AMG, amg_cheb_ratio=bad)
        assert L.mc_flow_create(ctypes.byref(mv), ctypes.byref(q), ctypes.byref(h)) == flow.MC_ERR_ARG, bad
    q = flow.default_params(flow.MODE_SIMPLE, pressure_solver=flow.PSOLVER_PCG_AMG, amg_sweeps=9)
    assert L.mc_flow_create(ctypes.byref(mv), ctypes.byref(q), ctypes.byref(h)) == flow.MC_ERR_ARG


def test_inconsistent_mesh_is_rejected():
    L = flow.library()
    mesh = flow.Mesh.box(3, 2, 2, 0.3, 0.2, 0.2)
    mesh.cell_faces[1, 2] = mesh.cell_faces[1, 3]  # a cell listing a face twice
    mv = mesh.view()
    p = flow.default_params(flow.MODE_SIMPLE)
    h = ctypes.c_void_p()
    assert L.mc_flow_create(ctypes.byref(mv), ctypes.byref(p), ctypes.byref(h)) == flow.MC_ERR_MESH
    mesh = flow.Mesh.box(3, 2, 2, 0.3, 0.2, 0.2)
    mesh.face_cells[0, 0] = 10 ** 6  # a face pointing outside the mesh
    mv = mesh.view()
    assert L.mc_flow_create(ctypes.byref(mv), ctypes.byref(p), ctypes.byref(h)) == flow.MC_ERR_MESH
