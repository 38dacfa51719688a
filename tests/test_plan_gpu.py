"""GPU-built execution plans against the reference's own op_plan_core.

The golden fixtures (tests/golden/plan_*.npz) are the plan arrays the
reference's op_plan_get_stage produced for the Airfoil loops
(oracle/ref_plan_dump.cpp, tests/golden/make_golden.py).  Integer outputs must
match bit for bit; col_reord is compared per (block, colour) as a set, because
the reference orders equal colours with the C library's qsort.  Every plan is
also validated on the device: op_plan_check's invariants plus the colour
conflict checks.  Where the reference's build travels with the repository
(oracle/_ref), the full 2400x1200 plan of res_calc is compared live.
"""
import glob
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN
from op2b import lib as L
from op2b import mesh as M
from op2b.airfoil import Airfoil
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INDS = {"adt_calc": [0, 0, 0, 0, -1, -1], "res_calc": [0, 0, 1, 1, 2, 2, 3, 3],
        "bres_calc": [0, 0, 1, 2, 3, -1]}


def _loop_args(app, loop):
    return {"adt_calc": (app.cells, app.a_adt), "res_calc": (app.edges, app.a_res),
            "bres_calc": (app.bedges, app.a_bres)}[loop]


def _compare(d, g, staging):
    sc = g["scalars"]
    assert d["nblocks"] == sc[0]
    assert d["ncolors"] == sc[1], (d["ncolors"], sc[1])
    assert d["ninds_staged"] == sc[2]
    if staging != 4:
        assert d["nshared"] == sc[4]
    for k in ("nthrcol", "offset", "nelems", "ind_offs", "ind_sizes", "inds_staged"):
        assert np.array_equal(d[k], g[k]), k
    nind = len(g["nindirect"])
    assert np.array_equal(d["nindirect"][:nind], g["nindirect"])
    for k in g.files:
        if k.startswith("ind_map") or k.startswith("loc_map"):
            assert np.array_equal(d[k], g[k]), k
    nb = int(sc[0])
    if staging == 4:
        assert d["ncolblk"][0] == g["ncolblk"][0] and d["blkmap"][0] == g["blkmap"][0]
    else:
        assert np.array_equal(d["ncolblk"], g["ncolblk"])
        assert np.array_equal(d["blkmap"], g["blkmap"])
        assert np.array_equal(d["nsharedCol"], g["nsharedCol"])
    if staging in (3, 4):
        assert np.array_equal(d["thrcol"], g["thrcol"])
        assert np.array_equal(d["col_offsets"], g["col_offsets"])
        base = 0
        for b in range(nb):
            nc = int(d["nthrcol"][b])
            off = d["col_offsets"][base:base + nc + 1]
            lo = int(d["offset"][b])
            for c in range(nc):
                a = set(d["col_reord"][lo + off[c]:lo + off[c + 1]])
                r = set(g["col_reord"][lo + off[c]:lo + off[c + 1]])
                assert a == r, (b, c)
            base += nc + 1
    else:
        assert np.array_equal(d["thrcol"], g["thrcol"])
    tr = g["transfer"]
    if staging != 4:
        assert abs(d["transfer"] - tr[0]) <= 1e-6 * max(abs(tr[0]), 1)
        assert abs(d["transfer2"] - tr[1]) <= 1e-6 * max(abs(tr[1]), 1)


PLAN_FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "plan_*.npz")))


@pytest.mark.parametrize("fixture", PLAN_FIXTURES, ids=[os.path.basename(f) for f in PLAN_FIXTURES])
def test_plan_matches_reference(op2, fixture):
    m_ = re.match(r"plan_(\w+?)_(\d+)x(\d+)_s(\d+)_st(\d)_p(\d+)\.npz", os.path.basename(fixture))
    loop, I, J, seed, staging, part = m_.group(1), *map(int, m_.groups()[1:])
    g = np.load(fixture)
    mesh = M.channel_bump(I, J, seed=seed)
    app = Airfoil(mesh)
    set_, args = _loop_args(app, loop)
    p = L.op_plan_get_stage(loop, set_, part, args, INDS[loop], staging)
    _compare(L.plan_arrays(p), g, staging)
    n, det = L.plan_validate(p)
    assert n == 0, det
    # a second request returns the cached plan
    p2 = L.op_plan_get_stage(loop, set_, part, args, INDS[loop], staging)
    assert p2.contents.count == 2


@pytest.mark.skipif(not O.ref_binary("ref_plan_dump"), reason="reference plan builder not built")
@pytest.mark.parametrize("I,J,part", [(2400, 1200, 0), (600, 300, 1024)])
def test_full_size_res_calc_plan_matches_reference_live(op2, I, J, part):
    mesh = M.channel_bump(I, J, seed=1)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "m.bin")
        M.write_grid_bin(mesh, path)
        subprocess.run([O.ref_binary("ref_plan_dump"), path, "2", str(part),
                        os.path.join(tmp, "p")], check=True, capture_output=True, timeout=600)
        g = O.read_plan_dump(os.path.join(tmp, "p.res_calc.plan"))
    app = Airfoil(mesh)
    p = L.op_plan_get_stage("res_calc", app.edges, part, app.a_res, INDS["res_calc"], 2)
    d = L.plan_arrays(p)

    class G(dict):
        files = property(lambda self: list(self.keys()))
    _compare(d, G(g), 2)
    n, det = L.plan_validate(p)
    assert n == 0, det
