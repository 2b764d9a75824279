"""Pins the oracle's restatement of the other scalar transports (k and
epsilon with wall functions, mixture fraction, progress variable and the two
variances; FlowSolver.inl:2516-3076) against the reference itself.

With params.scalars the oracle runs the reference's whole pass, so after
every pass all 13 fields and all 11 gradients must equal the reference's
bit for bit (compat mode, same shim solver), and each Scalar_solve stage on
its own must leave the same field, matrix and right-hand side.  The golden
vectors (all 13 fields after 10 passes on 16,000 cells) are checked without
the reference tree.
"""
import os

import numpy as np
import pytest

from checkers import COMPAT, SIMPLE, Oracle, Reference, noisy_initial_fields, oracle_mesh, oracle_params, \
    ref_available

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BASE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 2000.0}
ALL_FIELDS = ("U", "V", "W", "P", "PP", "TE", "ED", "TP", "TEM", "FUL", "PRO", "VARF", "VARP")
GRAD_FIELDS = ("U", "V", "W", "P", "TE", "ED", "TEM", "FUL", "PRO", "VARF", "VARP")
SCALARS = ("TE", "ED", "TEM", "FUL", "PRO", "VARF", "VARP")
needs_ref = pytest.mark.skipif(not ref_available(), reason="reference not compiled here (oracle/_ref)")


def seeded(obj, n, seed=0):
    for name, vals in noisy_initial_fields(n, BASE, seed).items():
        a = obj.field(name)
        a[:n] = vals
        obj.set_field(name, a)


@needs_ref
@pytest.mark.parametrize("dims,lengths,passes", [((8, 4, 4), (0.2, 0.1, 0.1), 10),
                                                 ((7, 3, 5), (0.4, 0.1, 0.3), 6),
                                                 ((1, 1, 1), (0.1, 0.1, 0.1), 4)])
def test_all_fields_match_reference_bitwise(dims, lengths, passes):
    ref = Reference(*dims, *lengths)
    orc = Oracle(ref.mesh(), oracle_params(COMPAT, scalars=1))
    for name in ALL_FIELDS:  # the constructor's initial state, boundary slots included
        assert np.array_equal(ref.field(name), orc.field(name)), name
    seeded(ref, ref.N)
    seeded(orc, orc.N)
    for p in range(passes):
        ref.step()
        assert orc.step() == 0
        for name in ALL_FIELDS:
            assert np.array_equal(ref.field(name), orc.field(name)), (p, name)
        for name in GRAD_FIELDS:
            assert np.array_equal(ref.grad(name), orc.grad(name)), (p, name)
    st = orc.stats()
    assert all(k > 0 for k in st.scalar_iters)


@needs_ref
@pytest.mark.parametrize("name", SCALARS)
def test_each_scalar_stage_matches_reference(name):
    """One Scalar_solve from the same state: field, matrix values and b."""
    dims, lengths = (9, 5, 4), (0.18, 0.1, 0.08)
    ref = Reference(*dims, *lengths)
    orc = Oracle(ref.mesh(), oracle_params(COMPAT, scalars=1))
    seeded(ref, ref.N, seed=3)
    seeded(orc, orc.N, seed=3)
    for _ in range(2):  # a developed state: k, epsilon and the fluxes away from their initial values
        ref.step()
        orc.step()
    orc.L.mco_stage_gradients(orc.h)
    ref.L.mcref_stage_gradients(ref.h)
    ref.stage_scalar(name)
    assert orc.stage_scalar(name) == 0
    assert np.array_equal(ref.field(name), orc.field(name))
    assert np.array_equal(ref.field("TP"), orc.field("TP"))
    rp, col, val = ref.csr(0)
    orp, ocol, oval = orc.csr(0)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol) and np.array_equal(val, oval)
    assert np.array_equal(ref.vec(0), orc.rhs(0))


def test_golden_all_fields_against_oracle():
    """The oracle reproduces the reference's golden output for all 13 fields."""
    g = np.load(os.path.join(GOLDEN, "ref_cfg1_10passes.npz"))
    dims, L = tuple(int(x) for x in g["dims"]), tuple(float(x) for x in g["lengths"])
    orc = Oracle(oracle_mesh(*dims, *L), oracle_params(COMPAT, scalars=1))
    seeded(orc, orc.N)
    for _ in range(int(g["passes"])):
        assert orc.step() == 0
    for name in ALL_FIELDS:
        assert np.array_equal(orc.field(name), g[name]), name


def negative_k_state(obj, mesh, seed=0):
    """k set below zero on a block of adjacent interior cells (no wall face, so
    the wall function's sqrt(k) stays defined) of the seeded initial state."""
    N = mesh.n_cells
    interior = np.where((mesh.cell_neighbours < N).all(axis=1))[0]
    te = obj.field("TE")
    te[interior[: len(interior) // 2]] = -1.0 - np.arange(len(interior) // 2) * 1e-3
    obj.set_field("TE", te)
    return interior[: len(interior) // 2]


def test_negative_k_replaced_in_cell_order():
    """k below zero after its solve takes the mean of its internal neighbours
    in ascending cell order, so a negative cell sees the replaced value of an
    earlier negative neighbour (FlowSolver.inl:2956-2985)."""
    mesh = oracle_mesh(8, 6, 6, 0.08, 0.06, 0.06)
    orc = Oracle(mesh, oracle_params(COMPAT, scalars=1))
    seeded(orc, orc.N)
    cells = negative_k_state(orc, mesh)
    orc.L.mco_stage_gradients(orc.h)
    assert orc.stage_scalar("TE") == 0
    got = orc.field("TE")[:orc.N]
    assert (got[cells] > 0).all()
    # the first negative cell of the block: mean of its neighbours, all of
    # which are later than it or non-negative
    assert got[cells[0]] > 0
    if ref_available():
        ref = Reference(8, 6, 6, 0.08, 0.06, 0.06)
        seeded(ref, ref.N)
        negative_k_state(ref, mesh)
        ref.L.mcref_stage_gradients(ref.h)
        ref.stage_scalar("TE")
        assert np.array_equal(ref.field("TE"), orc.field("TE"))


def test_simple_mode_scalars_run():
    """Simple-mode physics with the scalars on: every solve converges."""
    orc = Oracle(oracle_mesh(10, 5, 5, 0.2, 0.1, 0.1), oracle_params(SIMPLE, scalars=1))
    for name, vals in noisy_initial_fields(orc.N, dict(BASE, TEM=1500.0), 1).items():
        a = orc.field(name)
        a[:orc.N] = vals
        orc.set_field(name, a)
    for _ in range(3):
        assert orc.step() == 0
    assert all(k > 0 for k in orc.stats().scalar_iters)
