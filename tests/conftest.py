"""Test configuration: the `gpu` marker, import paths, and a per-test OP2 session.

Tests marked `gpu` need a CUDA device and the in-tree libop2b.so; everything
else runs on the CPU (oracle pins against the reference's own builds and
golden fixtures, mesh properties, the C ABI's exported symbols).
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "op2-common_b200")
for p in (PKG, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device and libop2b.so")


@pytest.fixture
def op2():
    """op_init before the test, op_exit after it (the library's state is global)."""
    from op2b import build, lib as L
    build.build()
    L.load()
    L.op_init()
    try:
        yield L
    finally:
        L.op_exit()
