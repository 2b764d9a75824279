import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def _build_checkers():
    # liboracle.so always; oracle/_ref/libmcref.so only where the reference tree exists.
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True,
                   stdout=subprocess.DEVNULL)


def _build_library():
    from minicombust_app_b200 import build
    build.build()


@pytest.fixture(scope="session", autouse=True)
def built():
    _build_checkers()
    _build_library()
    yield


_gpu = None


def gpu_available():
    global _gpu
    if _gpu is None:
        try:
            import torch
            _gpu = bool(torch.cuda.is_available())
        except Exception:
            _gpu = False
    return _gpu


@pytest.fixture
def gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")
    yield
