"""Shared test setup: the `gpu` marker, builds, and import helpers.

Tests marked `gpu` need a CUDA device (a B200); everything else runs on the CPU. The CUDA
library and the CPU oracle are built in-tree with make when missing (nvcc cross-compiles
sm_100a without a GPU).
"""
import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nse2d-channel-gpu_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on the B200 box)")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle_module(name):
    """A Python module of oracle/ (test infrastructure)."""
    return _load(name, os.path.join(ORACLE, name + ".py"))


def build_all():
    if not os.path.isfile(os.path.join(ORACLE, "_build", "liboracle.so")) or \
            not os.path.isfile(os.path.join(ORACLE, "_build", "nse2d_oracle")):
        subprocess.check_call(["make", "-s", "-C", ORACLE])
    if not os.path.isfile(os.path.join(PKG, "libnse2d_b200.so")) or not os.path.isfile(os.path.join(PKG, "nse2d")):
        subprocess.check_call(["make", "-s", "-C", PKG, "-j4"])


@pytest.fixture(scope="session")
def oracle():
    build_all()
    return _load("nse2d_oracle_py", os.path.join(ORACLE, "oracle.py"))


@pytest.fixture(scope="session")
def nse():
    build_all()
    return _load("nse2d_b200", os.path.join(PKG, "nse2d_b200.py"))


@pytest.fixture(scope="session")
def golden():
    import json
    return json.load(open(os.path.join(GOLDEN, "reference_cases.json")))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for tests marked gpu")
    return torch
