"""Reverse Cuthill-McKee reordering: the host-side order (no GPU needed).

The order must be a permutation; on a scrambled mesh it must recover a band
as narrow as scipy's reverse_cuthill_mckee finds (the textbook algorithm,
used here as the checker), and renumbering round-trips.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

from minicombust_app_b200 import flow


def adjacency(mesh):
    N = mesh.n_cells
    fc = mesh.face_cells.astype(np.int64)
    internal = fc[:, 1] < N
    r, c = fc[internal, 0], fc[internal, 1]
    A = sp.coo_matrix((np.ones(len(r)), (r, c)), shape=(N, N))
    return (A + A.T + sp.identity(N)).tocsr()


def bandwidth(A, n2o=None):
    A = A.tocoo()
    if n2o is None:
        return int(np.abs(A.row - A.col).max())
    o2n = np.empty_like(n2o)
    o2n[n2o] = np.arange(len(n2o))
    return int(np.abs(o2n[A.row] - o2n[A.col]).max())


@pytest.mark.parametrize("dims", [(12, 6, 5), (7, 3, 5), (1, 1, 1), (2, 1, 1), (20, 10, 10)])
def test_rcm_is_a_permutation_with_a_narrow_band(dims):
    mesh = flow.Mesh.box(*dims, 0.1 * dims[0], 0.1 * dims[1], 0.1 * dims[2])
    order = mesh.rcm_order()
    assert np.array_equal(np.sort(order), np.arange(mesh.n_cells))
    A = adjacency(mesh)
    ref = reverse_cuthill_mckee(A, symmetric_mode=True)
    assert bandwidth(A, order) <= max(bandwidth(A, ref), 1) * 1.25


def test_rcm_recovers_a_band_from_a_scrambled_mesh():
    mesh = flow.Mesh.box(16, 8, 6, 0.2, 0.1, 0.1)
    rng = np.random.default_rng(7)
    scrambled = mesh.renumbered(rng.permutation(mesh.n_cells))
    A = adjacency(scrambled)
    assert bandwidth(A) > 4 * bandwidth(adjacency(mesh))
    order = scrambled.rcm_order()
    assert np.array_equal(np.sort(order), np.arange(mesh.n_cells))
    ref = reverse_cuthill_mckee(A, symmetric_mode=True)
    assert bandwidth(A, order) <= bandwidth(A, ref) * 1.25


def test_renumbering_round_trip():
    mesh = flow.Mesh.box(6, 4, 3, 0.3, 0.2, 0.15)
    order = mesh.rcm_order()
    back = np.argsort(order)
    again = mesh.renumbered(order).renumbered(back)
    assert np.array_equal(again.cell_nodes, mesh.cell_nodes)
    assert np.array_equal(again.cell_neighbours, mesh.cell_neighbours)
    assert np.array_equal(again.face_cells, mesh.face_cells)
    assert np.array_equal(again.cell_centers, mesh.cell_centers)
