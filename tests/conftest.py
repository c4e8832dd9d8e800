import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


# A checkout of the reference project (read only).  CPU tests that load its
# modules skip when it is absent (e.g. on a GPU host).
REFERENCE_ROOT = os.environ.get("EL_REFERENCE_ROOT", "/root/reference")


def reference_module(relpath, name):
    """Load one module file of the reference checkout under a private name (a
    fresh module object, so a test may modify it), or skip."""
    import importlib.util
    path = os.path.join(REFERENCE_ROOT, relpath)
    if not os.path.exists(path):
        pytest.skip("reference checkout not present")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from energy_level_b200.build import build
    build()
    from energy_level_b200.core import Context
    c = Context(0)
    yield c
    c.close()
