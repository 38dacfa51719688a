"""HDF5 mesh I/O through the OP2 API (include/op_hdf5.h; the reference's
op2/src/externlib/op_hdf5.cpp): op_dump_to_hdf5 / op_write_const_hdf5 write
what the library holds, a new session declares it back with
op_decl_{set,map,dat}_hdf5 and op_get_const_hdf5, op_fetch_data_hdf5_file
writes a dat in its declared order; the reference's error cases; and the
reference's own airfoil_hdf5 programs (convert_mesh.cpp, airfoil.cpp),
unmodified, writing and reading their mesh file through libop2b."""
import math
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from op2b import lib as L
from op2b import mesh as M
from op2b.airfoil import Airfoil
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CONSTS = ("gam", "gm1", "cfl", "eps", "mach", "alpha")


def _map_host(m, n, dim):
    return np.ctypeslib.as_array(m.contents.map, shape=(n * dim,)).reshape(n, dim).copy()


def test_dump_then_declare_from_the_file(op2, tmp_path):
    m = M.channel_bump(60, 30, seed=2)
    app = Airfoil(m)
    app.iterate(3)
    f = str(tmp_path / "mesh.h5")
    L.op_dump_to_hdf5(f)
    for k in CONSTS:
        L.op_write_const_hdf5(k, 1, "double", [app.c[k]], f)
    L.op_write_const_hdf5("qinf", 4, "double", app.c["qinf"], f)
    q = L.op_fetch_data(app.p_q)
    adt = L.op_fetch_data(app.p_adt)
    # the file as the reference lays it out
    names = set(L.h5_list(f))
    assert {"/nodes", "/cells", "/edges", "/bedges", "/pedge", "/pecell", "/pcell", "/p_q",
            "/p_x", "/p_res", "/qinf", "/gam"} <= names
    assert int(L.h5_read(f, "cells")[0]) == m.ncell
    np.testing.assert_array_equal(L.h5_read(f, "pecell"), m.ecell)
    np.testing.assert_array_equal(L.h5_read(f, "p_q"), q)
    assert (L.h5_get_attr(f, "pecell", "size"), L.h5_get_attr(f, "pecell", "dim"),
            L.h5_get_attr(f, "pecell", "type")) == (str(m.nedge), "2", "int")
    # a dat's "size" attribute is its bytes per element (dat->size), as written
    # by the reference
    assert (L.h5_get_attr(f, "p_q", "size"), L.h5_get_attr(f, "p_q", "dim"),
            L.h5_get_attr(f, "p_q", "type")) == ("32", "4", "double")
    assert (L.h5_get_attr(f, "qinf", "dim"), L.h5_get_attr(f, "qinf", "type")) == ("4", "double")
    # a new session declares everything back from the file
    L.op_exit()
    L.op_init()
    nodes = L.op_decl_set_hdf5(f, "nodes")
    cells = L.op_decl_set_hdf5(f, "cells")
    edges = L.op_decl_set_hdf5_infer_size(f, "edges", "pecell")
    assert (L.op_get_size(nodes), L.op_get_size(cells), L.op_get_size(edges)) == \
        (m.nnode, m.ncell, m.nedge)
    pecell = L.op_decl_map_hdf5(edges, cells, 2, f, "pecell")
    pcell = L.op_decl_map_hdf5(cells, nodes, 4, f, "pcell")
    np.testing.assert_array_equal(_map_host(pecell, m.nedge, 2), m.ecell)
    np.testing.assert_array_equal(_map_host(pcell, m.ncell, 4), m.cell)
    p_q = L.op_decl_dat_hdf5(cells, 4, "double", f, "p_q")
    p_adt = L.op_decl_dat_hdf5(cells, 1, "double", f, "p_adt")
    p_x = L.op_decl_dat_hdf5(nodes, 2, "double", f, "p_x")
    np.testing.assert_array_equal(L.op_fetch_data(p_q), q)
    np.testing.assert_array_equal(L.op_fetch_data(p_adt), adt)
    np.testing.assert_array_equal(L.op_fetch_data(p_x), m.x)
    # converted on reading when the requested type differs
    p_xf = L.op_decl_dat_hdf5(nodes, 2, "float", f, "p_x")
    np.testing.assert_array_equal(L.op_fetch_data(p_xf), m.x.astype(np.float32))
    for k in CONSTS:
        assert L.op_get_const_hdf5(k, 1, "double", f)[0] == app.c[k]
    np.testing.assert_array_equal(L.op_get_const_hdf5("qinf", 4, "double", f), app.c["qinf"])


def test_fetch_to_file_writes_the_declared_order(op2, tmp_path):
    m = M.channel_bump(60, 30, seed=4)
    app = Airfoil(m)
    app.iterate(2)
    app.renumber(stats=False)
    app.iterate(1)
    f = str(tmp_path / "q.h5")
    L.op_fetch_data_hdf5_file(app.p_q, f)
    L.op_fetch_data_hdf5_file(app.p_q, f, "/results/states_0000001")
    q1 = app.fetch_original()
    np.testing.assert_array_equal(L.h5_read(f, "p_q"), q1)
    np.testing.assert_array_equal(L.h5_read(f, "/results/states_0000001"), q1)
    assert L.h5_list(f) == ["/p_q", "/results/", "/results/states_0000001"]
    # an existing dataset is overwritten after its attributes are checked
    app.iterate(1)
    L.op_fetch_data_hdf5_file(app.p_q, f)
    np.testing.assert_array_equal(L.h5_read(f, "p_q"), app.fetch_original())
    np.testing.assert_array_equal(L.h5_read(f, "/results/states_0000001"), q1)
    L.h5_write(f, "wrong", np.zeros((m.ncell, 4)))
    L.h5_set_attr(f, "wrong", "size", [32])
    L.h5_set_attr(f, "wrong", "dim", [4])
    L.h5_set_attr(f, "wrong", "type", "float", "string")
    with pytest.raises(L.Op2Error, match="do not match"):
        L.op_fetch_data_hdf5_file(app.p_q, f, "wrong")
    L.h5_write(f, "noattr", np.zeros((m.ncell, 4)))
    with pytest.raises(L.Op2Error, match="does not have attribute 'size'"):
        L.op_fetch_data_hdf5_file(app.p_q, f, "noattr")


def test_the_reference_error_cases(op2, tmp_path):
    f = str(tmp_path / "e.h5")
    L.h5_write(f, "cells", np.array([6], np.int32))
    L.h5_write(f, "nodes", np.array([9], np.int32))
    L.h5_write(f, "pcell", np.arange(24, dtype=np.int32).reshape(6, 4) % 9)
    L.h5_write(f, "q", np.ones((6, 4)))
    with pytest.raises(L.Op2Error, match="does not exist"):
        L.op_decl_set_hdf5(str(tmp_path / "missing.h5"), "cells")
    cells = L.op_decl_set_hdf5(f, "cells")
    nodes = L.op_decl_set_hdf5(f, "nodes")
    with pytest.raises(L.Op2Error, match="not found"):
        L.op_decl_map_hdf5(cells, nodes, 4, f, "m_test")
    with pytest.raises(L.Op2Error, match="do not match"):
        L.op_decl_map_hdf5(cells, nodes, 2, f, "pcell")
    with pytest.raises(L.Op2Error, match="do not match"):
        L.op_decl_map_hdf5(nodes, cells, 4, f, "pcell")       # from-set size
    with pytest.raises(L.Op2Error, match="not found"):
        L.op_decl_dat_hdf5(cells, 4, "double", f, "p_test")
    with pytest.raises(L.Op2Error, match="do not match"):
        L.op_decl_dat_hdf5(cells, 2, "double", f, "q")
    L.op_write_const_hdf5("gam", 1, "double", [1.4], f)
    with pytest.raises(L.Op2Error, match="already holds"):
        L.op_write_const_hdf5("gam", 1, "double", [1.5], f)
    with pytest.raises(L.Op2Error, match="do not match"):
        L.op_get_const_hdf5("gam", 2, "double", f)
    assert L.op_get_const_hdf5("gam", 1, "double", f)[0] == 1.4
    assert L.op_get_const_hdf5("gam", 1, "float", f)[0] == np.float32(1.4)
    assert L.op_decl_map_hdf5(cells, nodes, 4, f, "pcell")


def _run(binary, cwd):
    r = subprocess.run([binary], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


@pytest.mark.skipif(not (O.ref_binary("airfoil_hdf5_convert_dropin") and
                         O.ref_binary("airfoil_hdf5_dropin")),
                    reason="airfoil_hdf5 drop-in binaries not built")
def test_reference_airfoil_hdf5_programs_run_on_libop2b():
    """convert_mesh writes new_grid_out.h5 (every set, map and dat, two of them
    under nested groups, and the constants) and test.h5 (a dat at three
    paths); airfoil.cpp, given that file as new_grid.h5, declares its mesh from
    it (two datasets it asks for are absent: their declarations fail as in
    the reference), dumps it again, runs 1000 iterations and writes q to
    file_name.h5.  libop2b runs the application's loops with its built-in
    Airfoil kernels, whose arithmetic is airfoil_plain's (this application's
    adt_calc multiplies by 1/cfl where airfoil_plain's divides by cfl), so q
    equals the restated airfoil_plain's bit for bit."""
    m = M.channel_bump(240, 120, seed=1)
    c = M.airfoil_constants()
    with tempfile.TemporaryDirectory() as tmp:
        M.write_grid_dat(m, os.path.join(tmp, "new_grid.dat"))
        _run(O.ref_binary("airfoil_hdf5_convert_dropin"), tmp)
        g = os.path.join(tmp, "new_grid_out.h5")
        for s, n in (("nodes", m.nnode), ("cells", m.ncell), ("edges", m.nedge),
                     ("bedges", m.nbedge)):
            assert int(L.h5_read(g, s)[0]) == n
        for name, want in (("pedge", m.edge), ("pecell", m.ecell), ("pbedge", m.bedge),
                           ("pcell", m.cell), ("/group3/pedge_test", m.edge)):
            np.testing.assert_array_equal(L.h5_read(g, name), want)
        np.testing.assert_array_equal(L.h5_read(g, "pbecell").ravel(), m.becell)
        np.testing.assert_array_equal(L.h5_read(g, "p_bound").ravel(), m.bound)
        np.testing.assert_array_equal(L.h5_read(g, "p_x"), m.x)
        np.testing.assert_array_equal(L.h5_read(g, "/group3/group2/group1/p_x_test"), m.x)
        np.testing.assert_array_equal(L.h5_read(g, "p_q"), np.tile(c["qinf"], (m.ncell, 1)))
        for k in ("gam", "gm1", "cfl", "eps", "mach"):
            assert L.h5_read(g, k)[0] == c[k], k
        assert abs(L.h5_read(g, "alpha")[0] - math.pi / 60) < 1e-7
        np.testing.assert_array_equal(L.h5_read(g, "qinf"), c["qinf"])
        t = os.path.join(tmp, "test.h5")
        for p in ("/group3/group2/group1/p_x_test", "/states_0000000",
                  "/results/states_0000000"):
            np.testing.assert_array_equal(L.h5_read(t, p), m.x)
        shutil.move(g, os.path.join(tmp, "new_grid.h5"))
        out = _run(O.ref_binary("airfoil_hdf5_dropin"), tmp)
        hist = [(int(i), float(v)) for i, v in
                re.findall(r"^\s*(\d+)\s+([0-9.]+e[-+]\d+)\s*$", out, flags=re.M)]
        st, rms, _, _ = O.airfoil_run(m, c, 1000)
        assert [i for i, _ in hist] == list(range(100, 1001, 100)), out[-2000:]
        for i, v in hist:
            assert abs(v / rms[i - 1] - 1) < 2e-5      # printed with 6 digits
        np.testing.assert_array_equal(L.h5_read(os.path.join(tmp, "file_name.h5"), "p_q"),
                                      st.q)
        # the application's own dump of what it declared from new_grid.h5
        src, dump = os.path.join(tmp, "new_grid.h5"), os.path.join(tmp, "new_grid_out.h5")
        for name in ("nodes", "cells", "edges", "bedges", "pedge", "pecell", "pbedge",
                     "pbecell", "pcell", "p_bound", "p_x", "gam", "qinf"):
            np.testing.assert_array_equal(L.h5_read(dump, name), L.h5_read(src, name))


def test_full_size_mesh_round_trip(op2, tmp_path):
    """The benchmark's 2400x1200 mesh (2.88M cells, 484 MB in the file):
    dumped after renumbering, declared back in a new session, every map and
    dat equal; the times are printed (host file I/O)."""
    import time
    m = M.channel_bump(2400, 1200, seed=1)
    app = Airfoil(m)
    app.renumber(stats=False)
    app.iterate(1)
    f = str(tmp_path / "big.h5")
    want = {n: L.op_fetch_data(d) for n, d in (("p_q", app.p_q), ("p_x", app.p_x),
                                                 ("p_adt", app.p_adt), ("p_bound", app.p_bound))}
    t0 = time.perf_counter()
    L.op_dump_to_hdf5(f)
    t1 = time.perf_counter()
    size = os.path.getsize(f)
    L.op_exit()
    L.op_init()
    t2 = time.perf_counter()
    nodes = L.op_decl_set_hdf5(f, "nodes")
    cells = L.op_decl_set_hdf5(f, "cells")
    edges = L.op_decl_set_hdf5(f, "edges")
    bedges = L.op_decl_set_hdf5(f, "bedges")
    maps = {n: L.op_decl_map_hdf5(fr, to, d, f, n) for n, fr, to, d in (
        ("pedge", edges, nodes, 2), ("pecell", edges, cells, 2), ("pbedge", bedges, nodes, 2),
        ("pbecell", bedges, cells, 1), ("pcell", cells, nodes, 4))}
    got = {"p_q": L.op_decl_dat_hdf5(cells, 4, "double", f, "p_q"),
           "p_x": L.op_decl_dat_hdf5(nodes, 2, "double", f, "p_x"),
           "p_adt": L.op_decl_dat_hdf5(cells, 1, "double", f, "p_adt"),
           "p_bound": L.op_decl_dat_hdf5(bedges, 1, "int", f, "p_bound")}
    t3 = time.perf_counter()
    print(f"2400x1200 mesh: {size / 1e6:.0f} MB, op_dump_to_hdf5 {1e3 * (t1 - t0):.0f} ms, "
          f"declared back {1e3 * (t3 - t2):.0f} ms")
    assert size > 450e6
    for n, d in got.items():
        assert np.array_equal(L.op_fetch_data(d), want[n]), n
    # the maps as the library held them (renumbered), through the file
    assert np.array_equal(_map_host(maps["pecell"], m.nedge, 2), L.h5_read(f, "pecell"))
    assert np.array_equal(_map_host(maps["pcell"], m.ncell, 4), L.h5_read(f, "pcell"))
