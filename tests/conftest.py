"""Shared test setup.

* Registers the ``gpu`` marker (tests that need a B200; run with -m gpu).
* Loads the product package from ``pose-memory-wiping_b200/`` as ``pose_b200``.
* Puts ``oracle/`` on sys.path: the oracle is test infrastructure and is
  imported only by tests, the smoke check and the bench's CPU legs.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "pose-memory-wiping_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
os.environ.setdefault("POSE_GPU_QUIET", "1")


def load_pkg():
    if "pose_b200" in sys.modules:
        return sys.modules["pose_b200"]
    spec = importlib.util.spec_from_file_location(
        "pose_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pose_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_workloads():
    load_pkg()
    import pose_b200.workloads as wl  # noqa: E402
    return wl


def golden(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def wl():
    return load_workloads()


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.init()
    return torch
