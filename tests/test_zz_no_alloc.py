"""op2b_update_noalloc against op_par_loop("update", ...), through the C ABI.

Some callers cannot let a library allocate device memory: applications that
hand all of it to their own pool at start-up, and latency-critical paths that
must not pay cudaMalloc's device-wide synchronisation.  op2b_update_noalloc
serves them with a fixed scratch array inside the library.  This test runs it
twice in a row on the library's own device arrays and checks each call
against the regular update loop on the same state and against the oracle's
restated update (update.h:1-19): q bit for bit (same arithmetic), res
cleared, rms within 1e-14 relative (the per-block partial sums are grouped
differently), maxerr and errloc equal.  The second call also shows that the
shared scratch left by the first call does no harm.  A misaligned array is
refused on the host, before any launch.

The file name sorts last so a run stopping at the first failure has run every
other test before this one.
"""
import numpy as np
import pytest

from op2b import lib as L
from op2b import mesh as M
from op2b.airfoil import Airfoil
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _state(m, c, scale):
    st, *_ = O.airfoil_run(m, c, 3)
    for name in ("adt_calc", "res_calc", "bres_calc"):
        O.loop(name, m, c, st)
    st.res *= scale
    return st


def _upload(lib, dat, arr):
    a = np.ascontiguousarray(arr, dtype=np.float64 if arr.dtype != np.int32 else np.int32)
    assert lib.op2b_dat_upload(dat, a.ctypes.data, a.nbytes) == 0, L.last_error()


def test_update_noalloc_matches_update_loop_twice(op2):
    lib = L.load()
    m = M.channel_bump(120, 60, seed=5)
    c = M.airfoil_constants()
    ref = Airfoil(m, c)          # the existing entry point runs here
    alt = Airfoil(m, c)          # the allocation-free entry point runs here
    one = L.op_decl_set(1, "one")
    out_d = L.op_decl_dat(one, 2, "double", np.zeros((1, 2)), "rms_maxerr")
    out_i = L.op_decl_dat(one, 1, "int", np.zeros((1, 1), np.int32), "errloc")
    dptr = lambda d: lib.op2b_dat_device_ptr(d)
    stream = lib.op2b_get_stream()
    for call, scale in enumerate((1.0, 3.0)):
        st = _state(m, c, scale)
        want = st.copy()
        o_rms, o_max, o_loc = O.loop("update", m, c, want)
        for app in (ref, alt):
            _upload(lib, app.p_q, st.q)
            _upload(lib, app.p_qold, st.qold)
            _upload(lib, app.p_adt, st.adt)
            _upload(lib, app.p_res, st.res)
        ref.rms[0] = 0.0
        ref.maxerr[0] = 0.0
        ref.errloc[0] = 0
        ref._loop(4)
        _upload(lib, out_d, np.zeros((1, 2)))
        _upload(lib, out_i, np.zeros((1, 1), np.int32))
        base = dptr(out_d)
        rc = lib.op2b_update_noalloc(m.ncell, dptr(alt.p_qold), dptr(alt.p_q), dptr(alt.p_res),
                                     dptr(alt.p_adt), base, base + 8, dptr(out_i), stream)
        assert rc == 0, L.last_error()
        L.synchronize()
        g_ref, g_alt = ref.fetch(), alt.fetch()
        rms_maxerr = L.op_fetch_data(out_d)[0]
        errloc = int(L.op_fetch_data(out_i)[0, 0])
        assert np.array_equal(g_alt["q"], g_ref["q"]), f"call {call}: q differs"
        assert not g_alt["res"].any(), f"call {call}: res not cleared"
        assert abs(rms_maxerr[0] / ref.rms[0] - 1) < 1e-14, f"call {call}: rms"
        assert rms_maxerr[1] == ref.maxerr[0], f"call {call}: maxerr"
        assert errloc == ref.errloc[0], f"call {call}: errloc"
        # and directly against the oracle's update on the same state
        assert np.array_equal(g_alt["q"], want.q), f"call {call}: q differs from the oracle"
        assert abs(rms_maxerr[0] / o_rms - 1) < 1e-14, f"call {call}: rms vs oracle"
        assert rms_maxerr[1] == o_max and errloc == o_loc, f"call {call}: maxerr/errloc vs oracle"


def test_update_noalloc_refuses_misaligned_arrays_before_launch(op2):
    lib = L.load()
    m = M.channel_bump(16, 8, seed=2)
    app = Airfoil(m)
    one = L.op_decl_set(1, "one")
    out_d = L.op_decl_dat(one, 2, "double", np.zeros((1, 2)), "rms_maxerr")
    out_i = L.op_decl_dat(one, 1, "int", np.zeros((1, 1), np.int32), "errloc")
    dptr = lambda d: lib.op2b_dat_device_ptr(d)
    L.synchronize()
    before = lib.op2b_kernel_launches()
    base = dptr(out_d)
    # q shifted by one double: still device memory, no longer 16-byte aligned
    rc = lib.op2b_update_noalloc(m.ncell - 1, dptr(app.p_qold), dptr(app.p_q) + 8,
                                 dptr(app.p_res), dptr(app.p_adt), base, base + 8,
                                 dptr(out_i), lib.op2b_get_stream())
    assert rc == -1
    assert "aligned" in L.last_error() and "q" in L.last_error()
    assert lib.op2b_kernel_launches() == before


def test_update_noalloc_rejects_sizes_beyond_its_scratch(op2):
    lib = L.load()
    rc = lib.op2b_update_noalloc(4_194_305, None, None, None, None, None, None, None, None)
    assert rc == -1
    assert "4194304" in L.last_error()
