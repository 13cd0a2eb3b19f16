import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    """Import t2-relion_b200/ (a hyphenated directory) as module t2relion_b200."""
    name = "t2relion_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "t2-relion_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def t2b():
    return load_package()


@pytest.fixture(scope="session")
def synth():
    load_package()
    import t2relion_b200.synthetic as s
    return s


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o
