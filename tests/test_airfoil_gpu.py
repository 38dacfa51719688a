"""GPU parity of the Airfoil loops against the oracle, through the C ABI.

Tolerances (north star: q and rms within 1e-12 relative after 100
iterations, increment order differing):
* direct loops (save_soln, adt_calc, update's q) are compared bit for bit:
  the kernels keep the reference's expression trees and are compiled without
  FMA contraction, like the oracle;
* indirect increments (res_calc, bres_calc) differ only in summation order:
  |res_gpu - res_oracle| <= 1e-12 * max|res_oracle| per component;
* q after 100 iterations: |dq| <= 1e-12 * max|q| per component; rms within
  1e-12 relative; maxerr within 1e-10 relative.
"""
import numpy as np
import pytest

from conftest import GOLDEN
from op2b import lib as L
from op2b import mesh as M
from op2b.airfoil import Airfoil
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = [L.OP2B_INC_ATOMIC, L.OP2B_INC_COLOR, L.OP2B_INC_HYBRID, L.OP2B_INC_GATHER]


def _state_after(m, c, niter):
    st, *_ = O.airfoil_run(m, c, niter)
    return st


def _upload(app, st):
    lib = L.load()
    for dat, arr in ((app.p_q, st.q), (app.p_qold, st.qold), (app.p_adt, st.adt),
                     (app.p_res, st.res)):
        a = np.ascontiguousarray(arr, dtype=app.dtype)
        assert lib.op2b_dat_upload(dat, a.ctypes.data, a.nbytes) == 0


def _close(a, b, rel):
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return np.all(np.abs(a - b).max(axis=0) <= rel * scale)


@pytest.mark.parametrize("mode", MODES)
def test_each_loop_against_oracle(op2, mode):
    op2.set_option("inc_mode", mode)
    m = M.channel_bump(60, 30, seed=21)
    c = M.airfoil_constants()
    st = _state_after(m, c, 3)
    st.res[:] = np.random.default_rng(0).standard_normal(st.res.shape) * 1e-3
    app = Airfoil(m, c)
    _upload(app, st)

    ref = st.copy()
    O.loop("save_soln", m, c, ref)
    app._loop(0)
    g = app.fetch()
    assert np.array_equal(g["qold"], ref.qold)

    O.loop("adt_calc", m, c, ref)
    app._loop(1)
    g = app.fetch()
    assert np.array_equal(g["adt"], ref.adt), "adt_calc must be bit-exact"

    O.loop("res_calc", m, c, ref)
    app._loop(2)
    g = app.fetch()
    assert _close(g["res"], ref.res, 1e-12)

    O.loop("bres_calc", m, c, ref)
    app._loop(3)
    g = app.fetch()
    assert _close(g["res"], ref.res, 1e-12)

    # update on the oracle's own res, so q is comparable bit for bit
    _upload(app, ref)
    app.rms[0] = 0.0
    app.maxerr[0] = 0.0
    app.errloc[0] = 0
    rms, mx, el = O.loop("update", m, c, ref)
    app._loop(4)
    g = app.fetch()
    assert np.array_equal(g["q"], ref.q), "update must be bit-exact in q"
    assert not g["res"].any()
    assert abs(app.rms[0] / rms - 1) < 1e-14
    assert app.maxerr[0] == mx and app.errloc[0] == el


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("fixture", ["airfoil_24x12_s3.npz", "airfoil_240x120_s1.npz"])
def test_100_iterations_match_reference_golden(op2, mode, fixture):
    op2.set_option("inc_mode", mode)
    gd = np.load(f"{GOLDEN}/{fixture}")
    m = M.channel_bump(int(gd["I"]), int(gd["J"]), seed=int(gd["seed"]))
    app = Airfoil(m)
    hist = app.iterate(int(gd["niter"]))
    rms = np.array([h[0] for h in hist])
    mx = np.array([h[1] for h in hist])
    el = np.array([h[2] for h in hist])
    assert np.max(np.abs(rms / gd["rms"] - 1)) < 1e-12
    assert np.max(np.abs(mx / gd["maxerr"] - 1)) < 1e-10
    assert (el == gd["errloc"]).mean() > 0.95
    q = app.fetch()["q"]
    if "q" in gd:
        assert _close(q, gd["q"], 1e-12)
    else:
        idx = gd["q_sample_idx"]
        assert _close(q[idx], gd["q_sample"], 1e-12)
        assert np.allclose(q.sum(axis=0), gd["q_sum"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("part", [0, 1024])
def test_colouring_is_deterministic_and_matches_atomics(op2, part):
    m = M.channel_bump(300, 150, seed=8)
    op2.set_option("part_size", part)
    runs = {}
    for mode in (L.OP2B_INC_ATOMIC, L.OP2B_INC_COLOR, L.OP2B_INC_COLOR, L.OP2B_INC_HYBRID,
                 L.OP2B_INC_GATHER):
        op2.set_option("inc_mode", mode)
        app = Airfoil(m)
        hist = app.iterate(20)
        runs.setdefault(mode, []).append(np.array([h[0] for h in hist]))
    c1, c2 = runs[L.OP2B_INC_COLOR]
    assert np.array_equal(c1, c2), "colouring must be deterministic"
    for mode in (L.OP2B_INC_ATOMIC, L.OP2B_INC_HYBRID, L.OP2B_INC_GATHER):
        assert np.max(np.abs(runs[mode][0] / c1 - 1)) < 1e-12


# (gather_kernel, pipe_block, gather_minblocks, bres_kernel)
GATHER_KERNELS = [(1, 0, 0, 0), (2, 0, 0, 1), (3, 0, 0, 1), (4, 64, 0, 1), (4, 96, 0, 1),
                  (4, 128, 0, 1), (4, 256, 0, 1), (5, 64, 0, 1), (5, 96, 0, 1), (5, 128, 0, 0),
                  (5, 256, 0, 1), (6, 64, 5, 1), (6, 64, 6, 1), (6, 128, 0, 1), (6, 128, 3, 0),
                  (6, 256, 0, 1), (7, 0, 0, 1), (7, 0, 0, 0)]


@pytest.mark.parametrize("kernel", GATHER_KERNELS,
                         ids=lambda k: f"g{k[0]}b{k[1]}m{k[2]}r{k[3]}")
@pytest.mark.parametrize("fixture", ["airfoil_24x12_s3.npz", "airfoil_240x120_s1.npz"])
def test_gather_mode_is_bit_exact_with_reference(op2, fixture, kernel):
    """inc_mode 3 adds each cell's increments in element order starting from
    res, as the reference's sequential loop does: q after 100 iterations is
    bit-identical to the reference's own build (rms differs only by the order
    of its global sum) -- for every gather kernel (CSR walk, 4 lanes, unrolled
    slot records, shared-memory and register pipelines at each block size,
    the register pipeline over corner records) and both bres_calc gathers."""
    op2.set_option("inc_mode", L.OP2B_INC_GATHER)
    op2.set_option("gather_kernel", kernel[0])
    if kernel[1]:
        op2.set_option("pipe_block", kernel[1])
    op2.set_option("gather_minblocks", kernel[2])
    op2.set_option("bres_kernel", kernel[3])
    gd = np.load(f"{GOLDEN}/{fixture}")
    m = M.channel_bump(int(gd["I"]), int(gd["J"]), seed=int(gd["seed"]))
    app = Airfoil(m)
    hist = app.iterate(int(gd["niter"]))
    g = app.fetch()
    if "q" in gd:
        assert np.array_equal(g["q"], gd["q"])
        assert np.array_equal(g["adt"], gd["adt"])
    else:
        assert np.array_equal(g["q"][gd["q_sample_idx"]], gd["q_sample"])
        assert np.array_equal(g["q"].sum(axis=0), gd["q_sum"])
    assert np.array_equal(np.array([h[1] for h in hist]), gd["maxerr"])
    assert np.array_equal(np.array([h[2] for h in hist]), gd["errloc"])
    # the rms sum over ~1e5 terms in a different order: ~1e-14 relative
    assert np.max(np.abs(np.array([h[0] for h in hist]) / gd["rms"] - 1)) < 1e-13


@pytest.mark.parametrize("I,J,renumber", [(240, 120, True), (600, 300, True), (600, 300, False),
                                          (2400, 1200, True), (2400, 1200, False)])
def test_flux_ring_is_bit_identical_to_corner_kernel(op2, I, J, renumber):
    """gather_kernel 7 computes each interior flux once (by the cell that
    comes first in its CTA's range) and sums every cell's fluxes from a
    shared-memory ring in the same slot order: q, adt and res equal the
    corner kernel's bit for bit, fused with bres_calc and alone, in both
    precisions.  On the renumbered mesh the ring records are built and used;
    on a randomly numbered mesh nearly every neighbour lies outside the
    cell's range, so the cells compute nearly every flux themselves, and
    whichever kernel serves, the results are the same."""
    m = M.channel_bump(I, J, seed=7)
    for dtype in (np.float64, np.float32):
        for fuse in (1, 0):
            out, used = [], []
            for gk in (6, 7):
                op2.set_option("gather_kernel", gk)
                op2.set_option("fuse", fuse)
                app = Airfoil(m, dtype=dtype)
                if renumber:
                    app.renumber()
                app.iterate(3)
                out.append(app.fetch())
                used.append(op2.get_option("ring_used"))
                op2.op_exit()
                op2.op_init()
            for k in ("q", "adt", "res"):
                assert np.array_equal(out[0][k], out[1][k]), (dtype, fuse, k)
            assert used[0] == 0
            if renumber:
                assert used[1] == 1, (I, J)


@pytest.mark.parametrize("hints", [0, 1])
def test_pipelined_kernels_are_bit_identical(op2, hints):
    """res_calc's register pipeline, with and without cache hints, against the
    one-pass slot-record kernel."""
    m = M.channel_bump(240, 120, seed=6)
    out = []
    for gk in (3, 5, 6):
        op2.set_option("gather_kernel", gk)
        op2.set_option("pipe_hints", hints)
        app = Airfoil(m)
        app.iterate(5)
        out.append(app.fetch())
    for o in out[1:]:
        for k in ("q", "adt", "res"):
            assert np.array_equal(out[0][k], o[k]), k


@pytest.mark.parametrize("fuse", [0, 1])
def test_speculative_adt_is_bit_identical(op2, fuse):
    """update computing the next adt_calc's result ahead (speculate_adt) gives
    the same q, qold, adt, res and history as recomputing it, in both
    precisions, with and without loop fusion."""
    m = M.channel_bump(96, 48, seed=13)
    for dtype in (np.float64, np.float32):
        out, hists, stats = [], [], []
        for spec in (0, 1):
            op2.set_option("fuse", fuse)
            op2.set_option("speculate_adt", spec)
            app = Airfoil(m, dtype=dtype)
            hists.append(app.iterate(5))
            out.append(app.fetch())
            stats.append(op2.loop_stats("update+adt_calc"))
            op2.op_exit()
            op2.op_init()
        assert hists[0] == hists[1], dtype
        for k in ("q", "qold", "adt", "res"):
            assert np.array_equal(out[0][k], out[1][k]), (dtype, k)
        assert stats[0] is None and stats[1]["calls"] == 10  # every update follows an adt_calc


def test_speculative_adt_is_invisible_and_invalidated(op2):
    """Between update and adt_calc the adt dat keeps its old values; a q
    uploaded, or a constant changed, in between makes adt_calc recompute."""
    m = M.channel_bump(64, 32, seed=14)
    c = M.airfoil_constants()

    def run(spec, between):
        op2.set_option("speculate_adt", spec)
        app = Airfoil(m, c)
        app.iterate(1)
        for i in (1, 2, 3, 4):        # adt_calc, res_calc, bres_calc, update
            app._loop(i)
        seen = app.fetch()["adt"]     # before the next adt_calc
        between(app)
        app._loop(1)
        got = app.fetch()["adt"]
        op2.op_exit()
        op2.op_init()
        return seen, got

    def nothing(app):
        pass

    def upload(app):
        q = app.fetch()["q"] * 1.01
        a = np.ascontiguousarray(q)
        assert op2.load().op2b_dat_upload(app.p_q, a.ctypes.data, a.nbytes) == 0

    def new_cfl(app):
        op2.op_decl_const(1, "double", 0.8, "cfl")

    for between in (nothing, upload, new_cfl):
        s0, g0 = run(0, between)
        s1, g1 = run(1, between)
        assert np.array_equal(s0, s1), between.__name__
        assert np.array_equal(g0, g1), between.__name__
        if between is not nothing:
            assert not np.array_equal(g1, run(1, nothing)[1]), between.__name__


def test_speculative_adt_restored_for_other_readers(op2):
    """A loop that reads adt right after update (res_calc without the
    adt_calc in between) sees the program's adt, not the early one."""
    m = M.channel_bump(64, 32, seed=15)
    res = []
    for spec in (0, 1):
        op2.set_option("speculate_adt", spec)
        app = Airfoil(m)
        app.iterate(1)
        for i in (1, 2, 3, 4, 2, 3):   # ..., update, then res_calc and bres_calc again
            app._loop(i)
        res.append(app.fetch())
        op2.op_exit()
        op2.op_init()
    for k in ("res", "adt", "q"):
        assert np.array_equal(res[0][k], res[1][k]), k


def test_speculative_res_calc_is_bit_identical(op2):
    """update launching the res_calc + bres_calc pair that follows it
    (speculate_res), and leaving res unwritten as a known zero that the pair
    starts from (lazy_res), each on or off: the same fields and history, in
    both precisions; with speculate_res every pair after the first is
    launched ahead, and with lazy_res no zeros are ever written."""
    m = M.channel_bump(96, 48, seed=16)
    combos = [(0, 0), (1, 0), (0, 1), (1, 1)]
    for dtype in (np.float64, np.float32):
        out, hists, seen, zeroed = [], [], [], []
        for spec, lazy in combos:
            op2.set_option("speculate_res", spec)
            op2.set_option("lazy_res", lazy)
            op2.load().op2b_reset_stats()
            app = Airfoil(m, dtype=dtype)
            hists.append(app.iterate(5))
            seen.append(op2.loop_stats("bres_calc(speculated)"))
            zeroed.append(op2.loop_stats("res zeroed"))
            out.append(app.fetch())
            op2.op_exit()
            op2.op_init()
        for i in range(1, len(combos)):
            assert hists[0] == hists[i], (dtype, combos[i])
            for k in ("q", "qold", "adt", "res"):
                assert np.array_equal(out[0][k], out[i][k]), (dtype, combos[i], k)
        assert seen[0] is None and seen[1]["calls"] == 9
        # lazy_res: zeros are written once, when the statistics call observes
        # the last update's res; the iterations never wrote any
        assert zeroed[0] is None and zeroed[1] is None
        assert zeroed[2]["calls"] == 1 and zeroed[3]["calls"] == 1


def test_speculative_res_calc_is_invisible(op2):
    """Whatever the program does between update and the res_calc /
    bres_calc it is expected to call, it sees the state of the calls it
    made: res zero after update, res_calc's increments alone after res_calc,
    and a changed constant or a skipped loop gives the results of the
    program's own order."""
    m = M.channel_bump(64, 32, seed=17)

    def run(spec, between, after):
        op2.set_option("speculate_res", spec)
        op2.set_option("lazy_res", spec)
        app = Airfoil(m)
        app.iterate(1)
        for i in (1, 2, 3, 4):        # adt_calc, res_calc, bres_calc, update
            app._loop(i)
        seen = between(app)
        for i in after:
            app._loop(i)
        got = app.fetch()
        op2.op_exit()
        op2.op_init()
        return seen, got

    def res_now(app):
        return app.fetch()["res"]

    def res_after_adt(app):
        app._loop(1)
        return app.fetch()["res"]

    def res_after_res_calc(app):
        app._loop(1)
        app._loop(2)
        return app.fetch()["res"]

    def new_eps(app):
        app._loop(1)
        op2.op_decl_const(1, "double", 0.07, "eps")
        return None

    def res_calc_then_update(app):   # bres_calc skipped
        app._loop(1)
        app._loop(2)
        return None

    cases = [(res_now, (1, 2, 3, 4)), (res_after_adt, (2, 3, 4)),
             (res_after_res_calc, (3, 4)), (new_eps, (2, 3, 4)),
             (res_calc_then_update, (4, 1, 2, 3))]
    for between, after in cases:
        s0, g0 = run(0, between, after)
        s1, g1 = run(1, between, after)
        if s0 is not None:
            assert np.array_equal(s0, s1), between.__name__
        for k in ("q", "qold", "adt", "res"):
            assert np.array_equal(g0[k], g1[k]), (between.__name__, k)
    assert np.all(run(1, res_now, ())[0] == 0)


def test_fused_loop_pairs_are_bit_identical_to_separate_loops(op2):
    """The runtime defers save_soln and res_calc and fuses them with the
    adt_calc / bres_calc that follow; with fusion off every loop launches on
    its own.  q, adt, res, rms, maxerr and errloc agree bit for bit, in both
    precisions, and a deferred loop is launched before anything observes it."""
    m = M.channel_bump(96, 48, seed=12)
    for dtype in (np.float64, np.float32):
        out, hists, stats = [], [], []
        for fuse in (0, 1):
            op2.set_option("fuse", fuse)
            op2.set_option("speculate_adt", 0)  # every adt_calc computed, fused or not
            op2.set_option("rename_save", 0)    # save_soln copies (into the adt_calc)
            op2.load().op2b_reset_stats()
            app = Airfoil(m, dtype=dtype)
            hists.append(app.iterate(4))
            out.append(app.fetch())
            stats.append({n: op2.loop_stats(n) for n in
                          ("save_soln", "res_calc", "save_soln+adt_calc", "res_calc+bres_calc")})
            op2.op_exit()
            op2.op_init()
        assert hists[0] == hists[1], dtype
        for k in ("q", "qold", "adt", "res"):
            assert np.array_equal(out[0][k], out[1][k]), (dtype, k)
        assert stats[0]["res_calc+bres_calc"] is None and stats[1]["res_calc+bres_calc"]
        assert stats[1]["save_soln+adt_calc"]["calls"] == 4
    # a deferred save_soln / res_calc is launched before a fetch observes it
    op2.set_option("speculate_adt", 0)
    op2.set_option("rename_save", 0)
    app = Airfoil(m)
    app.iterate(1)
    app._loop(0)                                    # save_soln, deferred
    q = app.fetch()["q"]
    assert np.array_equal(app.fetch()["qold"], q)
    app._loop(1)                                    # adt_calc
    app._loop(2)                                    # res_calc, deferred
    r_deferred = app.fetch()["res"]
    op2.set_option("fuse", 0)
    app2 = Airfoil(m)
    app2.iterate(1)
    for i in (0, 1, 2):
        app2._loop(i)
    assert np.array_equal(r_deferred, app2.fetch()["res"])


def test_renamed_save_soln_is_bit_identical_and_invisible(op2):
    """save_soln by renaming: no copy; the update that next reads qold and
    writes q reads q's array and writes qold's, and the two dats swap arrays.
    Against rename_save 0, in both precisions: the same history and fields,
    and no save_soln launch at all inside the iterations.  Every observer
    sees qold = q after save_soln: a fetch, another loop writing q, a loop
    reading qold."""
    m = M.channel_bump(96, 48, seed=13)
    for dtype in (np.float64, np.float32):
        out, hists, launches = [], [], []
        for rename in (0, 1):
            op2.set_option("rename_save", rename)
            op2.load().op2b_reset_stats()
            app = Airfoil(m, dtype=dtype)
            hists.append(app.iterate(5))
            out.append(app.fetch())
            launches.append(op2.loop_stats("save_soln"))
            renamed = op2.loop_stats("save_soln(renamed)")
            op2.op_exit()
            op2.op_init()
        assert hists[0] == hists[1], dtype
        for k in ("q", "qold", "adt", "res"):
            assert np.array_equal(out[0][k], out[1][k]), (dtype, k)
        # copying: the first save_soln goes out fused with the first adt_calc
        assert launches[0]["calls"] == 4 and launches[1] is None and renamed["calls"] == 5
    # observers of a renamed save_soln
    app = Airfoil(m)
    app.iterate(2)
    app._loop(0)                                    # save_soln, renamed
    assert np.array_equal(app.fetch()["qold"], app.fetch()["q"])
    q_saved = app.fetch()["q"]
    app._loop(0)
    app._loop(1)                                    # adt_calc, reads q
    # a loop that writes q (not the update) makes the copy first
    L.op_par_loop("save_soln", app.cells,
                  L.op_arg_dat(app.p_qold, -1, L.OP_ID, 4, "double", L.OP_READ),
                  L.op_arg_dat(app.p_q, -1, L.OP_ID, 4, "double", L.OP_WRITE))  # qold -> q
    assert np.array_equal(app.fetch()["qold"], q_saved)
    assert np.array_equal(app.fetch()["q"], q_saved)
    app3 = Airfoil(m)
    app3.iterate(2)
    app3._loop(0)
    # a device pointer handed out for q before the update: no renaming is
    # done for it, the results stay those of the copying path
    L.load().op2b_dat_device_ptr(app3.p_q)
    for i in (1, 2, 3, 4):
        app3._loop(i)
    op2.set_option("rename_save", 0)
    app4 = Airfoil(m)
    app4.iterate(2)
    app4._loop(0)
    for i in (1, 2, 3, 4):
        app4._loop(i)
    assert np.array_equal(app3.fetch()["q"], app4.fetch()["q"])
    assert np.array_equal(app3.fetch()["qold"], app4.fetch()["qold"])


@pytest.mark.parametrize("adt", [6, 8])
def test_adt_calc_variants_are_bit_identical(op2, adt):
    """adt_calc under a register cap (6 or 8 CTAs per SM) against the default
    kernel, in both precisions."""
    m = M.channel_bump(120, 60, seed=8)
    for dtype in (np.float64, np.float32):
        out = []
        for v in (0, adt):
            op2.set_option("adt_minblocks", v)
            app = Airfoil(m, dtype=dtype)
            app.iterate(3)
            out.append(app.fetch())
        for k in ("q", "adt", "res"):
            assert np.array_equal(out[0][k], out[1][k]), (dtype, k)


def test_corner_kernel_falls_back_when_edges_are_not_cell_corners(op2):
    """Corner records need a cell's edges to touch at most four nodes; with
    the edges' node pairs shuffled they touch up to eight, and gather_kernel 6
    must serve the loop through the slot-record pipeline, bit-identically."""
    m = M.channel_bump(48, 24, seed=9)
    rng = np.random.default_rng(3)
    m.edge = np.ascontiguousarray(m.edge[rng.permutation(m.nedge)])
    out = []
    for gk in (3, 6):
        op2.set_option("gather_kernel", gk)
        app = Airfoil(m)
        app.iterate(3)
        out.append(app.fetch())
    for k in ("q", "adt", "res"):
        assert np.array_equal(out[0][k], out[1][k]), k


def test_options_return_to_defaults_at_exit(op2):
    defaults = {k: op2.get_option(k) for k in ("inc_mode", "gather_kernel", "bres_kernel",
                                                "adt_minblocks", "pipe_block")}
    op2.set_option("inc_mode", L.OP2B_INC_ATOMIC)
    op2.set_option("gather_kernel", 3)
    op2.set_option("bres_kernel", 0)
    op2.set_option("adt_minblocks", 6)
    op2.set_option("pipe_block", 256)
    op2.op_exit()
    op2.op_init()
    assert {k: op2.get_option(k) for k in defaults} == defaults
    with pytest.raises(L.Op2Error):
        op2.set_option("gather_kernel", 8)


def test_large_mesh_one_iteration_against_oracle(op2):
    """The full 2400x1200 configuration: GPU vs oracle after 2 iterations, plus
    conservation of the interior flux (sum of res_calc's increments is 0)."""
    m = M.channel_bump(2400, 1200, seed=1)
    c = M.airfoil_constants()
    st, rms_o, _, _ = O.airfoil_run(m, c, 2)
    app = Airfoil(m, c)
    hist = app.iterate(2)
    assert np.max(np.abs(np.array([h[0] for h in hist]) / rms_o - 1)) < 1e-12
    assert _close(app.fetch()["q"], st.q, 1e-12)
    # res_calc alone on the converged-ish state: increments cancel pairwise
    app._loop(1)
    app._loop(2)
    r = app.fetch()["res"]
    assert np.all(np.abs(r.sum(axis=0)) <= 1e-9 * np.abs(r).sum(axis=0))


@pytest.mark.parametrize("kernel", [3, 4, 5, 6, 7])
def test_mixed_precision_against_fp32_restatement(op2, kernel):
    op2.set_option("gather_kernel", kernel)
    m = M.channel_bump(120, 60, seed=4)
    c = M.airfoil_constants()
    st32, rms32 = O.airfoil_run_mixed(m, c, 50)
    _, rms64, _, _ = O.airfoil_run(m, c, 50)
    app = Airfoil(m, c, dtype=np.float32)
    hist = app.iterate(50)
    rms = np.array([h[0] for h in hist])
    q = app.fetch()["q"]
    # float increments in a different order: agreement at float rounding level
    assert np.max(np.abs(rms / rms32 - 1)) < 1e-4
    assert _close(q, st32.q, 1e-5)
    # and the stated error of the form against the FP64 oracle
    assert np.max(np.abs(rms / rms64 - 1)) < 1e-3


def test_errors_are_reported_not_run_on_host(op2):
    m = M.channel_bump(8, 4, seed=1)
    app = Airfoil(m)
    with pytest.raises(L.Op2Error, match="no device implementation"):
        L.op_par_loop("not_a_loop", app.cells, *app.a_save)
    with pytest.raises(L.Op2Error, match="argument"):
        L.op_par_loop("res_calc", app.edges, *app.a_res[:7])
    bad = L.op_arg_dat(app.p_q, -1, L.OP_ID, 4, "double", L.OP_WRITE)
    with pytest.raises(L.Op2Error, match="OP_READ"):
        L.op_par_loop("save_soln", app.cells, bad, app.a_save[1])
    with pytest.raises(L.Op2Error, match="invalid data for map"):
        L.op_decl_map(app.edges, app.cells, 2, np.full(2 * m.nedge, m.ncell), "bad")
    launches = L.load().op2b_kernel_launches()
    assert launches >= 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_reversed_update_changes_only_the_rms_summation_order(op2, dtype):
    """Option update_reverse (the default) walks the update's cells from the
    last down, for the L2: q, res, adt, maxerr and errloc are the same bits as
    walking upwards (errloc: the lowest cell on ties either way), and rms
    differs only by the order of its sum."""
    m = M.channel_bump(240, 120, seed=2)
    out = {}
    for rev in (1, 0):
        L.op_exit()
        L.op_init()
        L.set_option("update_reverse", rev)
        app = Airfoil(m, dtype=dtype)
        app.renumber(stats=False)
        hist = app.iterate(20)
        f = app.fetch()
        out[rev] = (hist, f)
    (h1, f1), (h0, f0) = out[1], out[0]
    for k in ("q", "res", "adt", "qold"):
        assert np.array_equal(f1[k], f0[k]), k
    for (r1, m1, e1), (r0, m0, e0) in zip(h1, h0):
        assert m1 == m0 and e1 == e0
        assert abs(r1 / r0 - 1) < 1e-12
