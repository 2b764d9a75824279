"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's own outputs.

Tolerances: assembly stages (geometry, gradients, mass fluxes, matrix rows
and right-hand sides) are compared bit for bit -- the kernels evaluate the
reference's expressions in the same order with FMA contraction off.  After
Krylov solves, summation order differs, so whole passes are compared with the
gate of the task: max over cells |a - b| / max |b| <= 1e-9 per field after 10
SIMPLE passes (solver tolerances 1e-13 on both sides).
"""
import os

import numpy as np
import pytest

from checkers import COMPAT, SIMPLE, Oracle, noisy_initial_fields, oracle_mesh, oracle_params
from minicombust_app_b200 import flow

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BASE_COMPAT = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 2000.0}
BASE_SIMPLE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 1500.0}
FIELDS = ("U", "V", "W", "P", "TEM")
PARITY = 1e-9


def rel_err(a, b):
    scale = np.abs(b).max()
    return np.abs(a - b).max() / (scale if scale > 0 else 1.0)


def seed_both(solver, orc, base, seed=0):
    init = noisy_initial_fields(solver.N, base, seed)
    for name, vals in init.items():
        a = solver.field(name)
        a[:solver.N] = vals
        solver.set_field(name, a)
        b = orc.field(name)
        b[:orc.N] = vals
        orc.set_field(name, b)
    return init


def make_pair(dims, lengths, mode=COMPAT, **kw):
    mesh = flow.Mesh.box(*dims, *lengths)
    om = oracle_mesh(*dims, *lengths)
    okw = {k: v for k, v in kw.items() if k in ("u_rtol", "p_rtol", "max_iters")}
    p = flow.default_params(mode, **kw)
    orc = Oracle(om, oracle_params(mode, scalars=p.transport_scalars, **okw))
    solver = flow.FlowSolver(mesh, params=p)
    return solver, orc


def blobs(n_cells, centers, k, seed, amplitude):
    """Seeded Gaussian source blobs (momentum +x, energy, mass)."""
    rng = np.random.default_rng(seed)
    idx = rng.choice(n_cells, size=k, replace=False)
    h = np.linalg.norm(centers[1] - centers[0])
    src = np.zeros((n_cells, 5))
    for c in idx:
        r2 = np.sum((centers - centers[c]) ** 2, axis=1) / (2.0 * h) ** 2
        g = amplitude * np.exp(-0.5 * r2)
        src[:, 0] += g
        src[:, 3] += 1e3 * g
        src[:, 4] += 1e-2 * g
    return src


@pytest.mark.parametrize("reorder", [flow.REORDER_NONE, flow.REORDER_RCM], ids=["natural", "rcm"])
def test_geometry_bitwise(gpu, reorder):
    solver, orc = make_pair((8, 4, 4), (0.2, 0.1, 0.1), reorder=reorder)
    for w in (1, 2, 3, 5, 6):
        assert np.array_equal(solver.face_array(w), orc.face_array(w)), w
    assert np.array_equal(solver.cell_array(2), orc.cell_array(6))
    for name in FIELDS:
        assert np.array_equal(solver.field(name), orc.field(name)), name


@pytest.mark.parametrize("reorder", [flow.REORDER_NONE, flow.REORDER_RCM], ids=["natural", "rcm"])
def test_assembly_stages_bitwise(gpu, reorder):
    solver, orc = make_pair((9, 5, 4), (0.18, 0.1, 0.08), reorder=reorder)
    seed_both(solver, orc, BASE_COMPAT, seed=11)
    solver.stage("gradients")
    orc.L.mco_stage_gradients(orc.h)
    for name in FIELDS:
        assert np.array_equal(solver.gradient(name), orc.grad(name)), name
    solver.stage("set_up_field")
    orc.L.mco_stage_set_up_field(orc.h)
    assert np.array_equal(solver.cell_array(0), orc.cell_array(0))  # precomp_AU
    assert np.array_equal(solver.face_array(0), orc.face_array(0))  # mass fluxes
    solver.stage("momentum")
    orc.L.mco_stage_calculate_uvw(orc.h)
    rp, col, val, rhs_w = solver.csr(flow.SYSTEM_MOMENTUM_W)
    orp, ocol, oval = orc.csr(0)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(val, oval)
    assert np.array_equal(rhs_w, orc.rhs(0))
    assert np.array_equal(solver.cell_array(0), orc.cell_array(0))  # A_phi.U after under-relaxation
    for name in ("U", "V", "W"):
        assert rel_err(solver.field(name), orc.field(name)) < 1e-12, name
    # continue from identical velocities so the pressure assembly can be compared exactly
    for name in ("U", "V", "W"):
        solver.set_field(name, orc.field(name))
    solver.stage("pressure")
    orc.L.mco_stage_calculate_pressure(orc.h)
    rp, col, val, rhs = solver.csr(flow.SYSTEM_PRESSURE)
    orp, ocol, oval = orc.csr(1)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(val, oval)
    assert np.array_equal(rhs, orc.rhs(1))
    for name in ("U", "V", "W", "P"):
        assert rel_err(solver.field(name), orc.field(name)) < 1e-11, name
    assert rel_err(solver.face_array(0), orc.face_array(0)) < 1e-11
    # the corrected pressure's gradient: the pass forms it only in the cells
    # update_P needs, the whole field when it is read
    assert rel_err(solver.gradient("P"), orc.grad("P")) < 1e-8
    solver.stage("temperature")
    orc.L.mco_stage_scalar_temperature(orc.h)
    assert rel_err(solver.field("TEM"), orc.field("TEM")) < 1e-12


@pytest.mark.parametrize("reorder", [flow.REORDER_NONE, flow.REORDER_RCM], ids=["natural", "rcm"])
def test_compat_ten_passes_match_reference_golden(gpu, reorder):
    """The parity gate: 16,000 cells, 10 SIMPLE passes, against the reference's own output."""
    g = np.load(os.path.join(GOLDEN, "ref_cfg1_10passes.npz"))
    dims, L = tuple(int(x) for x in g["dims"]), tuple(float(x) for x in g["lengths"])
    solver = flow.FlowSolver(flow.Mesh.box(*dims, *L), params=flow.default_params(flow.MODE_COMPAT, reorder=reorder))
    if reorder == flow.REORDER_RCM:
        assert not np.array_equal(solver.cell_order(), np.arange(solver.N))
    init = noisy_initial_fields(solver.N, BASE_COMPAT, 0)
    for name, vals in init.items():
        a = solver.field(name)
        a[:solver.N] = vals
        solver.set_field(name, a)
    for _ in range(int(g["passes"])):
        solver.simple_iteration()
    for name in FIELDS:
        err = rel_err(solver.field(name), g[name])
        assert err <= PARITY, (name, err)
    rp, col, _, _ = solver.csr(flow.SYSTEM_PRESSURE)
    assert np.array_equal(rp, g["pressure_rowptr"]) and np.array_equal(col, g["pressure_col"])


@pytest.mark.parametrize("reorder", [flow.REORDER_NONE, flow.REORDER_RCM], ids=["natural", "rcm"])
def test_compat_passes_match_oracle(gpu, reorder):
    solver, orc = make_pair((8, 4, 4), (0.2, 0.1, 0.1), reorder=reorder)
    seed_both(solver, orc, BASE_COMPAT, seed=2)
    for p in range(10):
        solver.simple_iteration()
        assert orc.step() == 0
        for name in FIELDS:
            err = rel_err(solver.field(name), orc.field(name))
            assert err <= PARITY, (p, name, err)


def test_simple_mode_with_sources_matches_oracle(gpu):
    solver, orc = make_pair((40, 20, 20), (0.2, 0.1, 0.1), SIMPLE, u_rtol=1e-13, p_rtol=1e-13)
    seed_both(solver, orc, BASE_SIMPLE, seed=0)
    mesh = solver.mesh
    src = blobs(solver.N, mesh.cell_centers, 10, seed=0, amplitude=1e-3 * 1.2 * 50.0 * (0.1 / 20) ** 2)
    solver.set_sources(src)
    orc.set_sources(src)
    for p in range(10):
        solver.simple_iteration()
        assert orc.step() == 0
    for name in FIELDS:
        err = rel_err(solver.field(name), orc.field(name))
        assert err <= PARITY, (name, err)
    st = solver.last_stats
    assert st.mass_imbalance < 1e-8 * np.abs(solver.face_array(0)).max()


@pytest.mark.parametrize("dims,lengths", [((1, 1, 1), (0.1, 0.1, 0.1)), ((2, 1, 1), (0.2, 0.1, 0.1)),
                                          ((3, 7, 2), (0.3, 0.7, 0.2)), ((5, 2, 9), (0.05, 0.2, 0.09))])
def test_edge_meshes_match_oracle(gpu, dims, lengths):
    solver, orc = make_pair(dims, lengths)
    seed_both(solver, orc, BASE_COMPAT, seed=4)
    for p in range(4):
        solver.simple_iteration()
        assert orc.step() == 0
        for name in FIELDS:
            err = rel_err(solver.field(name), orc.field(name))
            assert err <= PARITY, (dims, p, name, err)


def test_deterministic(gpu):
    out = []
    for _ in range(2):
        s = flow.FlowSolver(flow.Mesh.box(16, 8, 8, 0.2, 0.1, 0.1), params=flow.default_params(flow.MODE_SIMPLE))
        init = noisy_initial_fields(s.N, BASE_SIMPLE, 9)
        for name, vals in init.items():
            a = s.field(name)
            a[:s.N] = vals
            s.set_field(name, a)
        for _ in range(3):
            s.simple_iteration()
        out.append([s.field(n) for n in FIELDS] + [s.face_array(0)])
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("dims,reorder", [((40, 20, 20), flow.REORDER_NONE), ((20, 10, 10), flow.REORDER_NONE),
                                          ((7, 3, 5), flow.REORDER_NONE), ((40, 20, 20), flow.REORDER_RCM)])
def test_amg_pressure_solver_matches_oracle(gpu, dims, reorder):
    """PCG with the aggregation-AMG V-cycle reaches the same solution as the
    oracle's conjugate gradients (both to 1e-13), in far fewer iterations than
    PCG with Jacobi."""
    lengths = (0.2, 0.1, 0.1)
    solver, orc = make_pair(dims, lengths, SIMPLE, u_rtol=1e-13, p_rtol=1e-13,
                            pressure_solver=flow.PSOLVER_PCG_AMG, reorder=reorder)
    jac = flow.FlowSolver(flow.Mesh.box(*dims, *lengths),
                          params=flow.default_params(flow.MODE_SIMPLE, u_rtol=1e-13, p_rtol=1e-13))
    seed_both(solver, orc, BASE_SIMPLE, seed=1)
    for name in FIELDS:
        jac.set_field(name, solver.field(name))
    for p in range(5):
        solver.simple_iteration()
        jac.simple_iteration()
        assert orc.step() == 0
    for name in FIELDS:
        err = rel_err(solver.field(name), orc.field(name))
        assert err <= PARITY, (name, err)
    if solver.N > 1000:
        assert solver.last_stats.pressure_iters_first * 3 < jac.last_stats.pressure_iters_first


@pytest.mark.parametrize("dims", [(40, 20, 20), (7, 3, 5)])
@pytest.mark.parametrize("line_steps", [2, 0], ids=["xline", "bicgstab"])
def test_fp32_refined_pressure_solver_matches_oracle(gpu, dims, line_steps):
    """FP64 iterative refinement around FP32 inner solves (AMG-PCG for the
    pressure correction; x-line block Jacobi or BiCGStab for momentum and
    temperature) reaches the FP64 answer: the outer residual is the true FP64
    residual, so with the tolerances at 1e-12/1e-13 the fields meet the same
    1e-9 gate as the all-FP64 solvers."""
    lengths = (0.2, 0.1, 0.1)
    solver, orc = make_pair(dims, lengths, SIMPLE, u_rtol=1e-13, p_rtol=1e-12,
                            pressure_solver=flow.PSOLVER_PCG_AMG, precision=flow.PRECISION_FP32_REFINED,
                            ir_line_steps=line_steps)
    seed_both(solver, orc, BASE_SIMPLE, seed=3)
    for p in range(5):
        solver.simple_iteration()
        assert orc.step() == 0
        # every solve that did work, relative to the first corrector's right-hand side
        assert 0.0 < solver.last_stats.pressure_rel_residual <= 1e-12
    for name in FIELDS:
        err = rel_err(solver.field(name), orc.field(name))
        assert err <= PARITY, (name, err)


@pytest.mark.parametrize("line_steps", [2, 0], ids=["xline", "bicgstab"])
def test_fp32_refined_reaches_rtol_at_default_tolerance(gpu, line_steps):
    """At the default 1e-8 tolerances the refined solves stop on the FP64 true
    residual and land within the solver tolerance of the FP64 solves."""
    dims, lengths = (48, 24, 24), (0.2, 0.1, 0.1)
    out = {}
    for prec in (flow.PRECISION_FP64, flow.PRECISION_FP32_REFINED):
        s = flow.FlowSolver(flow.Mesh.box(*dims, *lengths),
                            params=flow.default_params(flow.MODE_SIMPLE, pressure_solver=flow.PSOLVER_PCG_AMG,
                                                       precision=prec, ir_line_steps=line_steps))
        init = noisy_initial_fields(s.N, BASE_SIMPLE, 5)
        for name, vals in init.items():
            a = s.field(name)
            a[:s.N] = vals
            s.set_field(name, a)
        for _ in range(3):
            s.simple_iteration()
            assert s.last_stats.pressure_rel_residual <= 1e-8
        out[prec] = [s.field(n) for n in FIELDS]
        s.close()
    for name, a, b in zip(FIELDS, out[flow.PRECISION_FP32_REFINED], out[flow.PRECISION_FP64]):
        assert rel_err(a, b) <= 1e-6, name
