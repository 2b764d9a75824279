"""The tensor-core layer's bounded waits, made to run out on purpose.

Every pipeline wait of the tcgen05 layer kernel gives up after a bounded
number of polls; the block then drains its copies and products in flight,
frees its tensor memory and returns, the prediction is zeroed and the call
returns MC_ERR_TIMEOUT instead of hanging.  MC_GNN_WAIT_POLLS=0 makes the
first pipeline wait fail at once (the drain waits keep their full bound), so
no wait is left to chance.  The next pass on the same handle, with the bound
restored, must succeed: the tensor memory was given back.  Runs in a child
process so the setting stays local.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys
sys.path.insert(0, os.environ["MC_ROOT"])
from minicombust_app_b200 import flow, train_guess
s = train_guess.make_solver(16, 3, guess=flow.GUESS_LEARNED, params=train_guess.load_params())
assert s.simple_iteration() == flow.MC_OK
os.environ["MC_GNN_WAIT_POLLS"] = "0"
rc = s.simple_iteration(check=False)
assert rc == flow.MC_ERR_TIMEOUT, rc
assert b"gave up" in flow.library().mc_flow_last_error(s.h)
del os.environ["MC_GNN_WAIT_POLLS"]
for _ in range(2):
    assert s.simple_iteration(check=False) == flow.MC_OK
    assert s.last_stats.guess_choice_first == 2
s.close()
print("timeout path ok")
"""


def test_layer_wait_timeout_is_reported_and_recovers(gpu):
    env = dict(os.environ, MC_ROOT=ROOT, MC_GNN_LAYER="umma")
    env.pop("MC_GNN_WAIT_POLLS", None)
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "timeout path ok" in r.stdout
