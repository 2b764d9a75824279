import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def _build_checkers(front):
    # liboracle.so always; oracle/_ref/* only where the reference tree exists.
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build_checkers
    build_checkers.build(front=front)


def _build_library():
    from minicombust_app_b200 import build
    build.build()


@pytest.fixture(scope="session", autouse=True)
def built():
    _build_checkers(front=False)
    _build_library()
    _build_checkers(front=True)  # the front's driver links the library
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
