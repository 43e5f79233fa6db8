"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU.

The oracle (oracle/) is the checker: tests import it to compare against, never
as the thing under test.
"""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# The reference project's tree (its data/ and scripts/ fixtures), from GSLAM_REFERENCE;
# tests that need it skip when it is absent (e.g. on machines that only carry this repo).
REF_ROOT = os.environ.get("GSLAM_REFERENCE", "/root/reference")
REF_DATA = os.path.join(REF_ROOT, "data")
REF_DUMPS = os.path.join(REF_ROOT, "scripts", "_pose_dumps_vp")
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs through libgslam's CUDA path)")


def load_pkg():
    return importlib.import_module("g-slam_on_gpu_and_fpga_b200")


@pytest.fixture(scope="session")
def pkg():
    p = load_pkg()
    p.build.build() if hasattr(p, "build") else None
    return p


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O


def ref_data(name):
    path = os.path.join(REF_DATA, name)
    if not os.path.exists(path):
        pytest.skip("reference data not present on this machine")
    return path


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def assert_bitwise(a, b, what=""):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    bad = np.flatnonzero(bits(a).ravel() != bits(b).ravel())
    assert bad.size == 0, (f"{what}: {bad.size} of {a.size} values differ; first at {bad[:5]}: "
                           f"{a.ravel()[bad[:5]]} vs {b.ravel()[bad[:5]]}")
