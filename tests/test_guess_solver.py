"""The learned initial guess inside the solver (MC_GUESS_LEARNED), on a seed
held out from training (seeds 16-19 of the 2*32^3 dataset were held out;
this test uses 23, never seen), against the plain zero guess of the
reference's pressure solve (FlowSolver.inl:2203-2273).

What it shows: the trained network's guess starts the first pressure solve
below the zero guess's residual; the solve still runs to the same tolerance,
so the fields equal the zero-guess run's within the parity gate; parameters
that predict nothing fall back to the zero guess; and the PCG iterations with
and without the network are reported (the gain).
"""
import numpy as np
import pytest

from minicombust_app_b200 import flow, train_guess

pytestmark = pytest.mark.gpu

SEED = 23
PASSES = 6
FIELDS = ("U", "V", "W", "P", "TEM")


def run(guess, params=None, p_rtol=1e-12):
    """PASSES passes of the 2*32^3 training box (the dataset's physics and
    source density) from seed SEED, solves at tight tolerances."""
    dims = train_guess.box(32)
    mesh = flow.Mesh.box(*dims, *train_guess.LENGTHS)
    p = flow.default_params(flow.MODE_SIMPLE, pressure_solver=flow.PSOLVER_PCG_AMG, initial_guess=guess,
                            p_rtol=p_rtol, u_rtol=1e-12)
    s = flow.FlowSolver(mesh, params=p)
    for name, vals in train_guess.noisy_fields(s.N, SEED).items():
        a = s.field(name)
        a[:s.N] = vals
        s.set_field(name, a)
    k = max(1, int(round(train_guess.BLOBS_PER_CELL * s.N)))
    s.set_sources(train_guess.gaussian_blobs(dims, train_guess.LENGTHS, k, SEED))
    if params is not None:
        s.set_guess_params(params)
    stats = []
    for _ in range(PASSES):
        s.simple_iteration()
        stats.append(s.last_stats.as_dict())
    fields = {n: s.field(n) for n in FIELDS}
    s.close()
    return stats, fields


def test_learned_guess_gain_and_parity(gpu):
    zero_stats, zero_fields = run(flow.GUESS_ZERO)
    learned_stats, learned_fields = run(flow.GUESS_LEARNED, train_guess.load_params())
    # the guess is used and starts below the zero guess's residual
    assert all(st["guess_choice_first"] == 2 for st in learned_stats[1:])
    rel = [st["guess_rel_residual_first"] for st in learned_stats[1:]]
    assert max(rel) < 1.0, rel
    # same tolerance, same answer
    for n in FIELDS:
        a, b = learned_fields[n], zero_fields[n]
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-9, n
    # the gain, reported: first-corrector PCG iterations with and without the network
    it_zero = [st["pressure_iters_first"] for st in zero_stats]
    it_learned = [st["pressure_iters_first"] for st in learned_stats]
    print(f"\nfirst-solve residual of the learned guess vs zero: {np.round(rel, 3).tolist()}; "
          f"PCG iterations zero guess {it_zero}, learned {it_learned}")
    assert sum(it_learned) <= sum(it_zero)


def test_useless_parameters_fall_back_to_zero(gpu):
    stats, fields = run(flow.GUESS_LEARNED, np.zeros(train_guess.gnn.param_count(), dtype=np.float32))
    zero_stats, zero_fields = run(flow.GUESS_ZERO)
    for st in stats:
        assert st["guess_rel_residual_first"] <= 1.0 + 1e-12
    for n in FIELDS:
        assert np.abs(fields[n] - zero_fields[n]).max() / np.abs(zero_fields[n]).max() <= 1e-9, n
