"""Pins the oracle (the C restatement in oracle/mc_oracle.c).

1. Against the reference itself (oracle/_ref, compiled from its sources with
   single-rank MPI/PETSc shims): mesh, geometry and 10 SIMPLE passes must agree
   bit for bit in compat mode.  Skipped where the reference was not built.
2. Against the committed golden vectors made from the reference by
   tests/golden/make_golden.py (runs everywhere).
3. Known-answer properties of the formulas on a uniform box (geometry, exact
   gradients of linear fields, Rhie-Chow uniform-flow identity, consistency of
   the singular pressure-correction system).
"""
import os

import numpy as np
import pytest

from checkers import (COMPAT, SIMPLE, Oracle, Reference, noisy_initial_fields, oracle_mesh, oracle_params,
                      ref_available)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BASE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 2000.0}
FIELDS = ("U", "V", "W", "P", "TEM")
needs_ref = pytest.mark.skipif(not ref_available(), reason="reference not compiled here (oracle/_ref)")


def seeded(obj, n, seed=0):
    init = noisy_initial_fields(n, BASE, seed)
    for name, vals in init.items():
        a = obj.field(name)
        a[:n] = vals
        obj.set_field(name, a)
    return init


@needs_ref
@pytest.mark.parametrize("dims,lengths", [((8, 4, 4), (0.2, 0.1, 0.1)), ((5, 3, 2), (0.05, 0.04, 0.03)),
                                          ((1, 1, 1), (0.1, 0.1, 0.1))])
def test_mesh_matches_reference(dims, lengths):
    ref = Reference(*dims, *lengths)
    rm = ref.mesh()
    om = oracle_mesh(*dims, *lengths)
    for k in ("points", "cells", "faces", "cell_faces", "cell_neighbours", "cell_centers", "boundary_types"):
        assert np.array_equal(getattr(rm, k), getattr(om, k)), k


@needs_ref
@pytest.mark.parametrize("dims,lengths,passes", [((8, 4, 4), (0.2, 0.1, 0.1), 10),
                                                 ((40, 20, 20), (0.2, 0.1, 0.1), 10),
                                                 ((7, 3, 5), (0.4, 0.1, 0.3), 6)])
def test_restatement_matches_reference_bitwise(dims, lengths, passes):
    ref = Reference(*dims, *lengths)
    orc = Oracle(ref.mesh(), oracle_params(COMPAT))
    assert ref.inlet_effective_viscosity() == orc.L.mco_inlet_effective_viscosity(orc.h)
    for w in (1, 2, 3, 5, 6):
        assert np.array_equal(ref.face_array(w), orc.face_array(w)), w
    assert np.array_equal(ref.cell_array(6), orc.cell_array(6))
    seeded(ref, ref.N)
    seeded(orc, orc.N)
    for p in range(passes):
        ref.step()
        orc.step()
        for name in FIELDS:
            assert np.array_equal(ref.field(name), orc.field(name)), (p, name)
        for name in FIELDS:
            assert np.array_equal(ref.grad(name), orc.grad(name)), (p, name)
        assert np.array_equal(ref.face_array(0), orc.face_array(0)), p
    for which in (0, 1):
        rp, col, _ = ref.csr(which)
        orp, ocol, _ = orc.csr(which)
        assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    rp, col, val = ref.csr(1)
    assert np.array_equal(val, orc.csr(1)[2])  # the stale pressure-correction matrix


@needs_ref
def test_harness_pass_equals_timestep():
    a = Reference(6, 3, 3, 0.06, 0.03, 0.03)
    b = Reference(6, 3, 3, 0.06, 0.03, 0.03)
    seeded(a, a.N)
    seeded(b, b.N)
    for _ in range(2):
        a.timestep()
        for _ in range(3):
            b.step()
    for name in FIELDS:
        assert np.array_equal(a.field(name), b.field(name)), name


def test_oracle_against_golden_small():
    g = np.load(os.path.join(GOLDEN, "ref_box6x3x3.npz"))
    dims, L = tuple(int(x) for x in g["dims"]), tuple(float(x) for x in g["lengths"])
    om = oracle_mesh(*dims, *L)
    for k, gk in (("points", "points"), ("cells", "cells"), ("faces", "faces"), ("cell_faces", "cell_faces"),
                  ("cell_neighbours", "cell_neighbours"), ("cell_centers", "cell_centers")):
        assert np.array_equal(getattr(om, k), g[gk]), k
    orc = Oracle(om, oracle_params(COMPAT))
    assert orc.L.mco_inlet_effective_viscosity(orc.h) == float(g["inlet_effective_viscosity"])
    for w, key in ((1, "face_area"), (2, "face_lambda"), (3, "face_rlencos"), (5, "face_normal"),
                   (6, "face_center")):
        assert np.array_equal(orc.face_array(w), g[key]), key
    assert np.array_equal(orc.cell_array(6), g["cell_volume"])
    for name in FIELDS:
        a = orc.field(name)
        a[:orc.N] = g[f"init_{name}"]
        orc.set_field(name, a)
    for p in range(4):
        orc.step()
        for name in FIELDS:
            assert np.array_equal(orc.field(name), g[f"pass{p + 1}_{name}"]), (p, name)
        assert np.array_equal(orc.face_array(0), g[f"pass{p + 1}_mdot"]), p
        if p == 0:
            rp, col, val = orc.csr(1)
            assert np.array_equal(rp, g["pressure_rowptr"]) and np.array_equal(col, g["pressure_col"])
            assert np.array_equal(val, g["pressure_val_pass1"])


@pytest.mark.slow
def test_oracle_against_golden_cfg1():
    g = np.load(os.path.join(GOLDEN, "ref_cfg1_10passes.npz"))
    dims, L = tuple(int(x) for x in g["dims"]), tuple(float(x) for x in g["lengths"])
    orc = Oracle(oracle_mesh(*dims, *L), oracle_params(COMPAT))
    seeded(orc, orc.N)
    for _ in range(int(g["passes"])):
        orc.step()
    for name in FIELDS:
        assert np.array_equal(orc.field(name), g[name]), name
    rp, col, _ = orc.csr(1)
    assert np.array_equal(rp, g["pressure_rowptr"]) and np.array_equal(col, g["pressure_col"])


# ---------------------------------------------------------------- known answers

def test_uniform_box_geometry():
    ex, ey, ez, lx, ly, lz = 6, 4, 3, 0.3, 0.2, 0.15
    m = oracle_mesh(ex, ey, ez, lx, ly, lz)
    orc = Oracle(m, oracle_params(COMPAT))
    dx, dy, dz = lx / ex, ly / ey, lz / ez
    internal = m.faces[:, 1] < m.n_cells
    lam = orc.face_array(2)
    area = orc.face_array(1)
    rl = orc.face_array(3)
    nrm = orc.face_array(5)
    np.testing.assert_allclose(lam[internal], 0.5, rtol=1e-12)
    np.testing.assert_allclose(lam[~internal], 1.0, rtol=0)
    np.testing.assert_allclose(orc.cell_array(6), dx * dy * dz, rtol=1e-12)
    # x-faces have area dy*dz and rlencos = A / dx (internal) or A / (dx/2) (boundary)
    xf = np.abs(nrm[:, 0]) > 0
    np.testing.assert_allclose(area[xf], dy * dz, rtol=1e-12)
    np.testing.assert_allclose(rl[xf & internal], dy * dz / dx, rtol=1e-12)
    np.testing.assert_allclose(rl[xf & ~internal], dy * dz / (dx / 2), rtol=1e-12)
    # normals point from cell0 to cell1 on internal faces, outwards on boundary faces
    cc = m.cell_centers
    c0 = m.faces[:, 0].astype(int)
    fc = orc.face_array(6)
    d = np.where(internal[:, None], cc[np.minimum(m.faces[:, 1], m.n_cells - 1).astype(int)] - cc[c0], fc - cc[c0])
    assert np.all(np.sum(d * nrm, axis=1) > 0)


def test_lsq_gradient_exact_for_linear_fields():
    m = oracle_mesh(6, 5, 4, 0.3, 0.25, 0.2)
    orc = Oracle(m, oracle_params(COMPAT))
    N = m.n_cells
    a, b, c = 3.0, -2.0, 5.0
    fc = orc.face_array(6)
    lin = m.cell_centers @ np.array([a, b, c]) + 7.0
    U = orc.field("U")
    U[:N] = lin
    # boundary slots hold one value per side; linear fields are exact only in cells without boundary faces
    orc.set_field("U", U)
    orc.L.mco_stage_gradients(orc.h)
    g = orc.grad("U")
    interior = np.all(m.cell_neighbours < N, axis=1)
    np.testing.assert_allclose(g[interior], np.tile([a, b, c], (interior.sum(), 1)), rtol=1e-10)
    assert np.isfinite(fc).all()


def test_rhie_chow_uniform_flow_identity():
    # uniform u, p: mass flux is rho u . S on every internal face and interior cells balance
    m = oracle_mesh(6, 4, 4, 0.3, 0.2, 0.2)
    orc = Oracle(m, oracle_params(COMPAT))
    orc.L.mco_stage_gradients(orc.h)
    orc.L.mco_stage_set_up_field(orc.h)
    md = orc.face_array(0)
    S = orc.face_array(5)
    internal = m.faces[:, 1] < m.n_cells
    np.testing.assert_allclose(md[internal], 1.2 * 50.0 * S[internal, 0], rtol=1e-12, atol=1e-15)
    N = m.n_cells
    div = np.zeros(N)
    np.add.at(div, m.faces[:, 0].astype(int), md)
    np.add.at(div, m.faces[internal, 1].astype(int), -md[internal])
    assert np.abs(div).max() < 1e-12 * np.abs(md).max()


def test_pressure_system_consistent_and_symmetric():
    m = oracle_mesh(8, 4, 4, 0.2, 0.1, 0.1)
    orc = Oracle(m, oracle_params(SIMPLE))
    seeded(orc, orc.N, seed=3)
    orc.step()
    rp, col, val = orc.csr(1)
    N = m.n_cells
    A = np.zeros((N, N))
    for i in range(N):
        A[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    np.testing.assert_allclose(A, A.T, rtol=0, atol=0)
    np.testing.assert_allclose(A.sum(axis=1), 0.0, atol=1e-12 * np.abs(A).max())


def test_simple_mode_conserves_mass_with_sources():
    m = oracle_mesh(10, 5, 5, 0.2, 0.1, 0.1)
    orc = Oracle(m, oracle_params(SIMPLE, p_rtol=1e-12, u_rtol=1e-12))
    seeded(orc, orc.N, seed=5)
    rng = np.random.default_rng(1)
    src = np.zeros((orc.N, 5))
    src[:, 0] = rng.uniform(0, 1e-6, orc.N)
    src[:, 3] = rng.uniform(0, 1e-3, orc.N)
    src[:, 4] = rng.uniform(0, 1e-7, orc.N)
    orc.set_sources(src)
    for _ in range(3):
        assert orc.step() == 0
        st = orc.stats()
        md = orc.face_array(0)
        assert st.mass_imbalance < 1e-9 * np.abs(md).max()
