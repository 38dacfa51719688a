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


@pytest.mark.parametrize("I,J,staging,part,renumber", [(240, 120, 2, 0, False),
                                                       (240, 120, 3, 128, True),
                                                       (240, 120, 4, 0, False),
                                                       (2400, 1200, 2, 0, False),
                                                       (2400, 1200, 2, 0, True),
                                                       (2400, 1200, 4, 0, True)])
def test_parallel_colouring_is_conflict_free(op2, I, J, staging, part, renumber):
    """plan_mode 1: block and thread colours (and OP_COLOR2's element
    colours) by Jones-Plassmann rounds on the device instead of the
    reference's serial greedy walk (op_rt_support.cpp:684-884).  The colours
    differ from the greedy ones, so the plan is checked by its invariants: no
    two elements of a thread colour in a block, no two blocks of a block
    colour, touch the same OP_INC target; every element in exactly one
    block.  Its staging arrays (ind_maps, loc_maps) stay the reference's."""
    mesh = M.channel_bump(I, J, seed=1)
    app = Airfoil(mesh)
    if renumber:
        app.renumber()
    op2.set_option("plan_mode", 1)
    p = L.op_plan_get_stage("res_calc", app.edges, part, app.a_res, INDS["res_calc"], staging)
    d = L.plan_arrays(p)
    n, det = L.plan_validate(p)
    assert n == 0, det
    ms = L.load().op2b_plan_build_ms(p)
    assert d["ncolors"] >= 2 and ms > 0
    if staging != 4:
        # block colours: a partition of the blocks
        nc = int(d["ncolors"])
        assert d["ncolblk"][:nc].sum() == d["nblocks"]
        assert sorted(d["blkmap"][:d["nblocks"]]) == list(range(d["nblocks"]))
    if staging == 4 and I * J > 240 * 120:
        print(f"{I}x{J} OP_COLOR2 renumbered {renumber}: parallel colouring "
              f"{d['ncolors']} colours in {ms:.1f} ms")
        return  # (the greedy OP_COLOR2 walk is one device thread: seconds at this size)
    # the greedy plan of the same loop keeps the reference's integers
    op2.set_option("plan_mode", 2)
    g = L.plan_arrays(L.op_plan_get_stage("res_calc", app.edges, part, app.a_res,
                                          INDS["res_calc"], staging))
    if staging != 4:
        for k in ("ind_offs", "ind_sizes", "nindirect", "nelems", "offset"):
            assert np.array_equal(d[k], g[k]), k
    print(f"{I}x{J} staging {staging} renumbered {renumber}: parallel colouring "
          f"{d['ncolors']} colours in {ms:.1f} ms; greedy {g['ncolors']} colours")


@pytest.mark.parametrize("mode", [L.OP2B_INC_COLOR, L.OP2B_INC_HYBRID])
def test_loops_on_parallel_colouring_match_reference(op2, mode):
    gd = np.load(f"{GOLDEN}/airfoil_240x120_s1.npz")
    m = M.channel_bump(240, 120, seed=1)
    op2.set_option("plan_mode", 1)
    op2.set_option("inc_mode", mode)
    app = Airfoil(m)
    hist = app.iterate(100)
    rms = np.array([h[0] for h in hist])
    assert np.max(np.abs(rms / gd["rms"] - 1)) < 1e-12
    q = app.fetch()["q"]
    idx = gd["q_sample_idx"]
    scale = np.abs(gd["q_sample"]).max(axis=0)
    assert np.all(np.abs(q[idx] - gd["q_sample"]).max(axis=0) <= 1e-12 * scale)


@pytest.mark.parametrize("segmented", [0, 1])
def test_atomic_increments_match_reference(op2, segmented):
    """inc_mode 0 with per-edge atomics and with segmented atomics (a warp's
    increments to one cell combined first): within 1e-12 of the reference
    after 100 iterations, on the randomly numbered and the renumbered mesh."""
    gd = np.load(f"{GOLDEN}/airfoil_240x120_s1.npz")
    for renumber in (False, True):
        op2.set_option("inc_mode", L.OP2B_INC_ATOMIC)
        op2.set_option("atomic_segmented", segmented)
        m = M.channel_bump(240, 120, seed=1)
        app = Airfoil(m)
        if renumber:
            app.renumber()
        hist = app.iterate(100)
        rms = np.array([h[0] for h in hist])
        assert np.max(np.abs(rms / gd["rms"] - 1)) < 1e-12
        q = app.fetch_original()
        idx = gd["q_sample_idx"]
        scale = np.abs(gd["q_sample"]).max(axis=0)
        assert np.all(np.abs(q[idx] - gd["q_sample"]).max(axis=0) <= 1e-12 * scale)
        L.op_exit()
        L.op_init()
