import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(autouse=True)
def default_library_options(request):
    """GPU tests start from the library's default options: the options are global
    state of libemmahydro (a ResidentHydro sets them), and the drop-in entries run
    with whatever was set last."""
    if request.node.get_closest_marker("gpu") is not None and gpu_available():
        import ctypes
        from emma_b200 import lib
        from emma_b200._lib import EmmaHydroOptions
        L = lib()
        o = EmmaHydroOptions()
        L.emma_hydro_default_options(ctypes.byref(o))
        L.emma_hydro_set_options(ctypes.byref(o))
        L.emma_hydro_clear_status()
    yield
