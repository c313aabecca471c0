import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def pytest_collection_modifyitems(config, items):
    # GPU tests cannot run without a device: skip them loudly rather than pass
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(autouse=True)
def _library_defaults(request):
    """After every GPU test, the library's process-wide settings go back to
    their defaults (whatever the test did or failed to undo), so that one
    failing test cannot change the conditions of the next."""
    yield
    if "gpu" not in request.keywords:
        return
    try:
        import libshalom_b200 as ls
        L = ls.lib()
    except Exception:
        return
    L.LibShalom_defer_flush()
    L.LibShalom_set_sync(1)
    L.LibShalom_set_stream(None)
    L.LibShalom_set_precision(0)
    L.LibShalom_set_dgemm_method(0, 0)
    L.LibShalom_set_splitk(0)
    L.LibShalom_set_tile_config(-1)
    L.LibShalom_set_autotune(1)
    L.LibShalom_set_graph_cache(0)
    L.LibShalom_set_thread_nums(0)
    L.LibShalom_set_tma(1)
