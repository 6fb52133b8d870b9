import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_package():
    """Import imau-ice_b200/ (a directory name with a hyphen) as ``imau_ice_b200``."""
    if "imau_ice_b200" in sys.modules:
        return sys.modules["imau_ice_b200"]
    d = os.path.join(ROOT, "imau-ice_b200")
    spec = importlib.util.spec_from_file_location("imau_ice_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["imau_ice_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the libdiva_b200.so kernels")
    config.addinivalue_line("markers", "gpu_pending: needs a CUDA GPU (B200); kernels whose first GPU run is "
                                       "pending, selected with -m gpu_pending")


@pytest.fixture(scope="session")
def oracle():
    import oracle_backend
    return oracle_backend.oracle_backend()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from imau_ice_b200 import build, diva
    build.build()
    return diva.cuda_backend()
