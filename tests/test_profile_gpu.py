"""Region profiling (op_profile_start/enter/next/exit/end/output, the
reference's op2/src/externlib/op_profile.cpp:557-570) on libop2b: the region
tree with device times from CUDA events on the library's stream, one kernel
node per op_par_loop at OP_PROFILE_LEVEL >= 2, and the JSON file of
OP_PROFILE_JSON_OUTPUT with the reference's node fields."""
import json
import os

import numpy as np
import pytest

from op2b import lib as L
from op2b import mesh as M
from op2b.airfoil import Airfoil

pytestmark = pytest.mark.gpu


def _tree(path):
    with open(path) as f:
        return json.load(f)


def _child(node, name):
    return next(c for c in node["children"] if c["name"] == name)


@pytest.mark.parametrize("level", [1, 2])
def test_region_tree_and_kernel_nodes(op2, tmp_path, monkeypatch, level):
    out = tmp_path / "prof.json"
    monkeypatch.setenv("OP_PROFILE_LEVEL", str(level))
    monkeypatch.setenv("OP_PROFILE_JSON_OUTPUT", str(out))
    lib = L.load()
    m = M.channel_bump(120, 60, seed=4)
    lib.op_profile_start(b"Airfoil")
    lib.op_profile_enter(b"setup")
    app = Airfoil(m)
    lib.op_profile_next(b"iterate")
    app.iterate(10)
    lib.op_profile_exit()
    lib.op_profile_end()
    lib.op_profile_output()
    root = _tree(out)
    assert root["name"] == "Airfoil" and root["clock"]["n"] == 1
    assert [c["name"] for c in root["children"]] == ["setup", "iterate"]
    it = _child(root, "iterate")
    assert it["clock"]["n"] == 1 and it["clock"]["total"] > 0
    assert set(it) >= {"name", "type", "clock", "num_ranks", "children"}
    kern = {c["name"]: c for c in it["children"] if c["type"] == 1}
    if level == 1:
        assert not kern
    else:
        # every loop the 10 iterations launched, as the runtime ran them
        assert kern, it["children"]
        assert all(k.endswith("/cuda/b200") for k in kern)
        launched = sum(k["clock"]["n"] for k in kern.values())
        assert launched >= 10 * 4
        # the loops' device time fits inside the region's
        assert sum(k["clock"]["total"] for k in kern.values()) <= it["clock"]["total"] * 1.01
    assert root["clock"]["total"] >= it["clock"]["total"]


def test_profiling_off_records_nothing(op2, tmp_path, monkeypatch):
    out = tmp_path / "prof.json"
    monkeypatch.setenv("OP_PROFILE_LEVEL", "0")
    monkeypatch.setenv("OP_PROFILE_JSON_OUTPUT", str(out))
    lib = L.load()
    lib.op_profile_start(b"off")
    lib.op_profile_enter(b"a")
    lib.op_profile_exit()
    lib.op_profile_end()
    lib.op_profile_output()
    assert not out.exists()
