"""Shared test fixtures.

`gpu` marks tests that need a CUDA device (run on a B200 with -m gpu); all
other tests run on the CPU.  The CUDA library is loaded from the package
directory (distance-occlusion_b200/libdol_b200.so, built by build.py); the CPU
oracle from oracle/ (liboracle.so, and oracle/_ref/libdolref.so when the
reference sources were available at build time).
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_dol():
    if "dol_b200" in sys.modules:
        return sys.modules["dol_b200"]
    spec = importlib.util.spec_from_file_location(
        "dol_b200", os.path.join(ROOT, "distance-occlusion_b200", "__init__.py"),
        submodule_search_locations=[os.path.join(ROOT, "distance-occlusion_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dol_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def dol():
    return load_dol()


@pytest.fixture(scope="session")
def O():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
