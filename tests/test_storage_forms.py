"""The solvers' storage forms on a structured box are layouts, not different
methods, and say so in numbers:

* the FP64 momentum, temperature and scalar rows stored by direction
  (positions in the order the directions occur in every row's slots) take
  the same iterations as the rows in slot order (MC_ROW_STORE=0) and give the
  same fields to the last bits: measured at most 5e-15 (plain) and 3e-11
  (headline, whose FP32 inner solves carry a last-bit difference of the FP64
  residual further) relative to each field's maximum after three passes;
  checked here at 1e-9;
* the FP16 copy of the FP32 V-cycle's level-0 couplings changes only the
  preconditioner: the refined solves still reach their FP64 tolerances, so the
  fields agree with those of the FP32 level 0 (MC_AMG_HALF=0) to the solves'
  accuracy, and the pressure iterations stay the same.

Both switches are read when a handle is created.
"""
import os

import numpy as np
import pytest

from minicombust_app_b200 import flow, train_guess
from minicombust_app_b200.workload import gaussian_blobs, noisy_fields

pytestmark = pytest.mark.gpu

M = 32
DIMS, LENGTHS = (2 * M, M, M), (0.2, 0.1, 0.1)
PASSES = 3
FIELDS = ("U", "V", "W", "P", "TEM")


def run(env, headline):
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        mesh = flow.Mesh.box(*DIMS, *LENGTHS)
        kw = dict(pressure_solver=flow.PSOLVER_PCG_AMG)
        if headline:
            kw.update(initial_guess=flow.GUESS_LEARNED, precision=flow.PRECISION_FP32_REFINED)
        s = flow.FlowSolver(mesh, params=flow.default_params(flow.MODE_SIMPLE, **kw))
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    for name, vals in noisy_fields(s.N, seed=3).items():
        a = s.field(name)
        a[:s.N] = vals
        s.set_field(name, a)
    s.set_sources(gaussian_blobs(DIMS, LENGTHS, 40, seed=3))
    if headline:
        s.set_guess_params(train_guess.load_params())
    its = []
    for _ in range(PASSES):
        s.simple_iteration()
        st = s.last_stats.as_dict()
        its.append((st["pressure_iters_total"], tuple(st["momentum_iters"]), st["temperature_iters"]))
    fields = {n: s.field(n) for n in FIELDS}
    s.close()
    return fields, its


@pytest.mark.parametrize("headline", [False, True], ids=["plain", "headline"])
def test_rows_by_direction_same_solves(gpu, headline):
    by_dir, its_d = run({}, headline)
    by_slot, its_s = run({"MC_ROW_STORE": "0"}, headline)
    assert its_d == its_s
    for n in FIELDS:
        rel = np.abs(by_dir[n] - by_slot[n]).max() / np.abs(by_slot[n]).max()
        assert rel <= 1e-9, (n, rel)
    again, _ = run({}, headline)  # each form on its own is bitwise reproducible
    for n in FIELDS:
        assert np.array_equal(again[n], by_dir[n]), n


def test_fp16_level0_preconditioner_only(gpu):
    half, its_h = run({}, True)
    full, its_f = run({"MC_AMG_HALF": "0"}, True)
    assert [i[0] for i in its_h] == [i[0] for i in its_f]
    for n in FIELDS:
        rel = np.abs(half[n] - full[n]).max() / np.abs(full[n]).max()
        assert rel <= 1e-6, (n, rel)
