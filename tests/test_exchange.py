"""The flow side of the flow/particle exchange (FlowSolver::update_flow_field,
FlowSolver.inl:496-736): particle rows summed into the cells' source terms,
and the flow state interpolated to the nodes of the cells the particle ranks
asked about (get_neighbour_cells / interpolate_to_nodes, :293-494).

The reference runs its whole exchange here: the MPI shim stages the
particle ranks' messages (cell indexes, particle_aos rows) and records what
the flow rank sends back.  The device sums each cell's rows in arrival
order, so the source terms must match bit for bit; the node values sum a
node's cells in ascending cell id where the reference uses hash-set order,
so they must match to 1e-13 of the field's scale.
"""
import numpy as np
import pytest

from checkers import Reference, noisy_initial_fields, ref_available
from minicombust_app_b200 import flow

needs_ref = pytest.mark.skipif(not ref_available(), reason="reference not compiled here (oracle/_ref)")
BASE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 2000.0}


def messages(n_cells, seed):
    """Two particle ranks; the second sends cells with several particles each
    (repeated ids), the first a spread of single particles."""
    rng = np.random.default_rng(seed)
    m1 = rng.choice(n_cells, size=min(40, n_cells), replace=False).astype(np.uint64)
    m2 = rng.integers(0, max(1, n_cells // 4), size=60).astype(np.uint64)
    return {1: (m1, rng.standard_normal((len(m1), 5)) * [1e-3, 1e-4, 1e-4, 5.0, 1e-5]),
            2: (m2, rng.standard_normal((len(m2), 5)) * [1e-3, 1e-4, 1e-4, 5.0, 1e-5])}


@needs_ref
def test_reference_exchange_runs_through_the_shim():
    ref = Reference(6, 4, 3, 0.06, 0.04, 0.03)
    msgs = messages(ref.N, 0)
    terms, sent = ref.exchange(msgs)
    want = np.zeros_like(terms)
    for cells, rows in msgs.values():
        for c, r in zip(cells, rows):
            want[int(c)] += r
    assert np.allclose(terms, want, rtol=1e-14, atol=0)
    assert sorted(sent) == [1, 2]
    for rank, (ids, vals) in sent.items():
        assert len(ids) == vals.shape[0] and len(set(ids.tolist())) == len(ids)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("reorder", [flow.REORDER_NONE, flow.REORDER_RCM], ids=["natural", "rcm"])
def test_exchange_matches_reference(gpu, reorder):
    dims, L = (10, 6, 5), (0.1, 0.06, 0.05)
    ref = Reference(*dims, *L)
    solver = flow.FlowSolver(flow.Mesh.box(*dims, *L), params=flow.default_params(flow.MODE_COMPAT, reorder=reorder))
    for name, vals in noisy_initial_fields(ref.N, BASE, 3).items():
        a = ref.field(name)
        a[:ref.N] = vals
        ref.set_field(name, a)
        solver.set_field(name, a)
    ref.L.mcref_stage_gradients(ref.h)
    solver.stage("gradients")
    msgs = messages(ref.N, 1)
    terms, sent = ref.exchange(msgs)
    cells = np.concatenate([m[0] for m in msgs.values()])
    rows = np.concatenate([m[1] for m in msgs.values()])
    solver.ingest_particles(cells, rows)
    assert np.array_equal(solver.sources(), terms)
    for rank, (cells_r, _) in msgs.items():
        ids, vals = solver.interpolate_nodes(cells_r)
        rids, rvals = sent[rank]
        order = np.argsort(rids)
        assert np.array_equal(ids, rids[order])
        rvals = rvals[order]
        for k in range(5):
            scale = max(np.abs(rvals[:, k]).max(), 1.0)
            assert np.abs(vals[:, k] - rvals[:, k]).max() <= 1e-13 * scale, k


@pytest.mark.gpu
def test_ingest_many_rows_and_reuse(gpu):
    """200,000 rows on 16,000 cells (the device sort across many tiles), twice:
    each call replaces the sources; sums against a float64 numpy
    accumulation in arrival order."""
    s = flow.FlowSolver(flow.Mesh.box(40, 20, 20, 0.2, 0.1, 0.1), params=flow.default_params(flow.MODE_SIMPLE))
    rng = np.random.default_rng(4)
    for call in range(2):
        n = 200_000
        cells = rng.integers(0, s.N, size=n).astype(np.uint64)
        rows = rng.standard_normal((n, 5))
        s.ingest_particles(cells, rows)
        want = np.zeros((s.N, 5))
        np.add.at(want, cells.astype(np.int64), rows)  # arrival order per cell
        assert np.array_equal(s.sources(), want), call
    s.ingest_particles(np.zeros(0, dtype=np.uint64), np.zeros((0, 5)))
    assert not s.sources().any()
    with pytest.raises(flow.FlowError) as e:
        s.ingest_particles(np.array([s.N], dtype=np.uint64), np.zeros((1, 5)))
    assert e.value.status == flow.MC_ERR_ARG
