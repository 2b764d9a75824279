"""Properties of the SIMPLE pass at the benchmark's full size, where the CPU
oracle is too slow to run in a test: the 2*128^3 = 4,194,304-cell box with
1,000 seeded source blobs (simple-mode physics, pressure PCG with the
aggregation-AMG V-cycle, the defaults' 1e-8 tolerances).

* The learned-guess + FP32-refined configuration and the plain FP64 one, three
  passes each from the same state, agree within 2e-6 per field: each solves to
  the same 1e-8 residual and lands within 1e-6 of the exact answer (the
  benchmark measures each against the CPU oracle run to 1e-12), so the FP32
  solves inside FP64 refinement reach the FP64 answer.
* Every pressure solve that does work reaches the 1e-8 tolerance (relative to
  the first corrector's right-hand side), and no cell's mass imbalance after a
  pass exceeds 1e-8 of the largest face flux.
* A second handle run from the same state gives the same fields bit for bit
  (every reduction sums in a fixed order).
The 2*64^3 box is compared with the CPU oracle itself in
test_oracle_at_scale.py.
"""
import numpy as np
import pytest

from minicombust_app_b200 import flow, train_guess
from minicombust_app_b200.workload import gaussian_blobs, noisy_fields

pytestmark = pytest.mark.gpu

M = 128
DIMS, LENGTHS = (2 * M, M, M), (0.2, 0.1, 0.1)
PASSES = 3
FIELDS = ("U", "V", "W", "P", "TEM")


def run(headline):
    mesh = flow.Mesh.box(*DIMS, *LENGTHS)
    kw = dict(pressure_solver=flow.PSOLVER_PCG_AMG)
    if headline:
        kw.update(initial_guess=flow.GUESS_LEARNED, precision=flow.PRECISION_FP32_REFINED)
    s = flow.FlowSolver(mesh, params=flow.default_params(flow.MODE_SIMPLE, **kw))
    for name, vals in noisy_fields(s.N, seed=0).items():
        a = s.field(name)
        a[:s.N] = vals
        s.set_field(name, a)
    s.set_sources(gaussian_blobs(DIMS, LENGTHS, 1000, seed=0))
    if headline:
        s.set_guess_params(train_guess.load_params())
    stats = []
    for _ in range(PASSES):
        s.simple_iteration()
        stats.append(s.last_stats.as_dict())
    fields = {n: s.field(n) for n in FIELDS}
    mdot = s.face_array(0)
    s.close()
    return stats, fields, mdot


def test_full_size_box_headline_against_fp64_and_determinism(gpu):
    plain_stats, plain_fields, plain_mdot = run(False)
    head_stats, head_fields, _ = run(True)
    errs = {n: float(np.abs(head_fields[n] - plain_fields[n]).max() / np.abs(plain_fields[n]).max())
            for n in FIELDS}
    print(f"\n2*128^3, {PASSES} passes: headline against plain FP64, max relative difference per field {errs}")
    assert max(errs.values()) <= 2e-6, errs
    for st in plain_stats + head_stats:
        assert 0.0 < st["pressure_rel_residual"] <= 1e-8, st["pressure_rel_residual"]
        assert st["mass_imbalance"] <= 1e-8 * np.abs(plain_mdot).max(), st["mass_imbalance"]
    # the learned guess is used and starts below the zero guess's residual
    assert all(st["guess_rel_residual_first"] < 1.0 for st in head_stats[1:])
    again_stats, again_fields, _ = run(True)
    for n in FIELDS:
        assert np.array_equal(again_fields[n], head_fields[n]), n
    assert [st["pressure_iters_total"] for st in again_stats] == [st["pressure_iters_total"] for st in head_stats]
