"""Shared test set-up: markers, the package loader and the checkers.

The package directory is named ``cuda-raytracer_b200`` (not importable as a
plain module name); it is loaded here as ``cuda_raytracer_b200``.
"""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cuda-raytracer_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def load_package():
    if "cuda_raytracer_b200" in sys.modules:
        return sys.modules["cuda_raytracer_b200"]
    spec = importlib.util.spec_from_file_location("cuda_raytracer_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cuda_raytracer_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cr():
    return load_package()


@pytest.fixture(scope="session")
def scenes():
    load_package()
    from cuda_raytracer_b200 import scenes as s
    return s


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def require_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA GPU is required for tests marked gpu")
