"""Loops without a hand-written kernel: the application's kernel source
compiled at run time (NVRTC, sm_100a) into a generated loop, against numpy.

Tolerances: direct arguments and OP_MIN/OP_MAX are exact (each element's
arithmetic is the kernel's, compiled without FMA contraction, as numpy
computes it); OP_INC increments and OP_INC globals are summed by atomics in
no fixed order: within 1e-12 relative of the sequential sum.  Loops with
indirect OP_RW/OP_WRITE run colour by colour; their test sums integers, so
any order is exact.
"""
import os

import numpy as np
import pytest

from op2b import lib as L

pytestmark = pytest.mark.gpu

DIRECT = """
inline void gen_scale(const double *a, double *b, const int *i, double *s, double *mx,
                      double *mn, const double *g) {
  *b = fac * (*a) + g[0] * (*i) + g[1];
  *s += *b;
  *mx = (*b > *mx) ? *b : *mx;
  *mn = (*b < *mn) ? *b : *mn;
}
"""

EDGES = """
inline void gen_scatter(const double *A, const double *u, double *du, const double *beta,
                        const int *e, const int *n0) {
  du[0] += (*beta) * (*A) * u[0];
  du[1] += (*beta) * u[1] - (double)(*e) + 0.5 * (*n0);
}
"""


def _rng_mesh(n_nodes=5000, n_edges=16000, seed=0):
    rng = np.random.default_rng(seed)
    pp = rng.integers(0, n_nodes, size=(n_edges, 2)).astype(np.int32)
    return rng, pp


def test_direct_loop_with_globals_index_and_constant(op2):
    op2.register_kernel("gen_scale", DIRECT)
    rng = np.random.default_rng(1)
    n = 20000
    a = rng.standard_normal(n)
    s = op2.op_decl_set(n, "cells")
    pa = op2.op_decl_dat(s, 1, "double", a, "a")
    pb = op2.op_decl_dat(s, 1, "double", None, "b")
    op2.op_decl_const(1, "double", 2.5, "fac")
    tot = np.array([10.0])
    mx = np.array([-1e300])
    mn = np.array([1e300])
    g = np.array([1e-3, -0.25])
    for _ in range(2):  # the second call runs the cached module
        tot[0] = 10.0
        op2.op_par_loop("gen_scale", s,
                        op2.op_arg_dat(pa, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                        op2.op_arg_dat(pb, -1, op2.OP_ID, 1, "double", op2.OP_WRITE),
                        op2.op_arg_idx(-1, op2.OP_ID),
                        op2.op_arg_gbl(tot, 1, "double", op2.OP_INC),
                        op2.op_arg_gbl(mx, 1, "double", op2.OP_MAX),
                        op2.op_arg_gbl(mn, 1, "double", op2.OP_MIN),
                        op2.op_arg_gbl(g, 2, "double", op2.OP_READ))
    b = 2.5 * a + g[0] * np.arange(n) + g[1]
    got = op2.op_fetch_data(pb)[:, 0]
    assert np.array_equal(got, b)
    assert abs(tot[0] - (10.0 + b.sum())) <= 1e-12 * np.abs(b).sum()
    assert mx[0] == b.max() and mn[0] == b.min()
    # a changed constant reaches the compiled module
    op2.op_decl_const(1, "double", -1.0, "fac")
    op2.op_par_loop("gen_scale", s,
                    op2.op_arg_dat(pa, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_dat(pb, -1, op2.OP_ID, 1, "double", op2.OP_WRITE),
                    op2.op_arg_idx(-1, op2.OP_ID),
                    op2.op_arg_gbl(np.zeros(1), 1, "double", op2.OP_INC),
                    op2.op_arg_gbl(np.array([-1e300]), 1, "double", op2.OP_MAX),
                    op2.op_arg_gbl(np.array([1e300]), 1, "double", op2.OP_MIN),
                    op2.op_arg_gbl(g, 2, "double", op2.OP_READ))
    assert np.array_equal(op2.op_fetch_data(pb)[:, 0], -a + g[0] * np.arange(n) + g[1])


def test_indirect_increment_and_read_through_a_map(op2):
    op2.register_kernel("gen_scatter", EDGES)
    rng, pp = _rng_mesh()
    nn, ne = 5000, pp.shape[0]
    A = rng.standard_normal(ne)
    u = rng.standard_normal((nn, 2))
    nodes = op2.op_decl_set(nn, "nodes")
    edges = op2.op_decl_set(ne, "edges")
    m = op2.op_decl_map(edges, nodes, 2, pp, "ppedge")
    pA = op2.op_decl_dat(edges, 1, "double", A, "A")
    pu = op2.op_decl_dat(nodes, 2, "double", u, "u")
    pdu = op2.op_decl_dat(nodes, 2, "double", None, "du")
    beta = np.array([0.75])
    op2.op_par_loop("gen_scatter", edges,
                    op2.op_arg_dat(pA, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_dat(pu, 1, m, 2, "double", op2.OP_READ),
                    op2.op_arg_dat(pdu, 0, m, 2, "double", op2.OP_INC),
                    op2.op_arg_gbl(beta, 1, "double", op2.OP_READ),
                    op2.op_arg_idx(-1, op2.OP_ID),
                    op2.op_arg_idx(0, m))
    ref = np.zeros((nn, 2))
    e = np.arange(ne)
    np.add.at(ref[:, 0], pp[:, 0], 0.75 * A * u[pp[:, 1], 0])
    np.add.at(ref[:, 1], pp[:, 0], 0.75 * u[pp[:, 1], 1] - e + 0.5 * pp[:, 0])
    got = op2.op_fetch_data(pdu)
    scale = np.abs(ref).max(axis=0)
    assert np.all(np.abs(got - ref).max(axis=0) <= 1e-12 * scale)


def test_float_and_int_and_kernel_file_with_prelude(op2, tmp_path):
    (tmp_path / "user_types.h").write_text(
        "#include <math.h>\nstatic inline float gen_sq(float v) { return v * v; }\n")
    (tmp_path / "gen_norm.h").write_text(
        "inline void gen_norm(const float *x, float *y, int *cnt, int *top) {\n"
        "  *y = sqrtf(gen_sq(x[0]) + gen_sq(x[1]));\n"
        "  *cnt += 1;\n"
        "  *top = (int)(*y) > *top ? (int)(*y) : *top;\n"
        "}\n")
    old = os.environ.get("OP2B_KERNEL_PATH")
    os.environ["OP2B_KERNEL_PATH"] = str(tmp_path)
    try:
        rng = np.random.default_rng(2)
        n = 7777
        x = (rng.standard_normal((n, 2)) * 10).astype(np.float32)
        s = op2.op_decl_set(n, "pts")
        px = op2.op_decl_dat(s, 2, "float", x, "x")
        py = op2.op_decl_dat(s, 1, "float", None, "y")
        cnt = np.array([3], np.int32)
        top = np.array([-5], np.int32)
        op2.op_par_loop("gen_norm", s,
                        op2.op_arg_dat(px, -1, op2.OP_ID, 2, "float", op2.OP_READ),
                        op2.op_arg_dat(py, -1, op2.OP_ID, 1, "float", op2.OP_WRITE),
                        op2.op_arg_gbl(cnt, 1, "int", op2.OP_INC),
                        op2.op_arg_gbl(top, 1, "int", op2.OP_MAX))
        y = np.sqrt(x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1])
        assert np.array_equal(op2.op_fetch_data(py)[:, 0], y)
        assert cnt[0] == 3 + n and top[0] == int(y.astype(np.int32).max())
    finally:
        if old is None:
            os.environ.pop("OP2B_KERNEL_PATH")
        else:
            os.environ["OP2B_KERNEL_PATH"] = old


def test_unsupported_forms_and_compile_errors_are_reported(op2):
    op2.register_kernel("gen_rw", "inline void gen_rw(double *v) { *v += 1.0; }\n")
    op2.register_kernel("gen_bad", "inline void gen_bad(double *v) { *v = undeclared; }\n")
    rng, pp = _rng_mesh(100, 300)
    nodes = op2.op_decl_set(100, "nodes")
    edges = op2.op_decl_set(300, "edges")
    m = op2.op_decl_map(edges, nodes, 2, pp, "ppedge")
    pv = op2.op_decl_dat(nodes, 1, "double", None, "v")
    with pytest.raises(L.Op2Error, match="does not fit a map of dimension 2"):
        op2.op_par_loop("gen_rw", edges, op2.op_arg_dat(pv, 2, m, 1, "double", op2.OP_READ))
    with pytest.raises(L.Op2Error, match="does not fit a map of dimension 2"):
        op2.op_par_loop("gen_rw", edges, op2.op_arg_dat(pv, -3, m, 1, "double", op2.OP_READ))
    with pytest.raises(L.Op2Error, match="compiling the kernel failed"):
        op2.op_par_loop("gen_bad", nodes, op2.op_arg_dat(pv, -1, op2.OP_ID, 1, "double",
                                                         op2.OP_RW))
    with pytest.raises(L.Op2Error, match="no device implementation"):
        op2.op_par_loop("gen_missing", nodes, op2.op_arg_dat(pv, -1, op2.OP_ID, 1, "double",
                                                             op2.OP_RW))


def test_indirect_rw_and_write_run_colour_by_colour(op2):
    """Indirect OP_RW and OP_WRITE arguments: the loop runs one launch per
    colour of the device-built OP_COLOR2 plan, so no two elements of a launch
    share a target.  Integer-valued increments make any order exact."""
    op2.register_kernel("gen_rw2", """
inline void gen_rw2(double *a, double *b, const double *w, const int *e) {
  *a += *w;
  *b += 2.0 * (*w) + (*e % 3);
}
""")
    op2.register_kernel("gen_pin", "inline void gen_pin(double *v, const int *i) { *v = 100.0 + *i; }\n")
    rng, pp = _rng_mesh(3000, 12000, seed=4)
    pp = pp[pp[:, 0] != pp[:, 1]]
    nn, ne = 3000, pp.shape[0]
    w = rng.integers(-50, 50, size=ne).astype(np.float64)
    v0 = rng.integers(-1000, 1000, size=nn).astype(np.float64)
    nodes = op2.op_decl_set(nn, "nodes")
    edges = op2.op_decl_set(ne, "edges")
    m = op2.op_decl_map(edges, nodes, 2, pp, "ppedge")
    pv = op2.op_decl_dat(nodes, 1, "double", v0, "v")
    pw = op2.op_decl_dat(edges, 1, "double", w, "w")
    before = L.load().op2b_kernel_launches()
    for _ in range(2):  # the second call reuses the cached colouring
        op2.op_par_loop("gen_rw2", edges,
                        op2.op_arg_dat(pv, 0, m, 1, "double", op2.OP_RW),
                        op2.op_arg_dat(pv, 1, m, 1, "double", op2.OP_RW),
                        op2.op_arg_dat(pw, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                        op2.op_arg_idx(-1, op2.OP_ID))
    ref = v0.copy()
    for _ in range(2):
        np.add.at(ref, pp[:, 0], w)
        np.add.at(ref, pp[:, 1], 2.0 * w + np.arange(ne) % 3)
    assert np.array_equal(op2.op_fetch_data(pv)[:, 0], ref)
    # one launch per colour; a colour needs at least the largest degree
    deg = np.bincount(pp.reshape(-1), minlength=nn).max()
    assert L.load().op2b_kernel_launches() - before >= 2 * deg
    # indirect OP_WRITE through a one-to-one map (boundary pinning)
    nb = 500
    bn = rng.permutation(nn)[:nb].astype(np.int32)
    bset = op2.op_decl_set(nb, "bnodes")
    bm = op2.op_decl_map(bset, nodes, 1, bn.reshape(-1, 1), "pbnode")
    op2.op_par_loop("gen_pin", bset, op2.op_arg_dat(pv, 0, bm, 1, "double", op2.OP_WRITE),
                    op2.op_arg_idx(-1, op2.OP_ID))
    ref[bn] = 100.0 + np.arange(nb)
    assert np.array_equal(op2.op_fetch_data(pv)[:, 0], ref)


def test_vector_map_arguments(op2):
    """Vector map arguments (op_arg_dat with idx = -k): the kernel gets k
    pointers, one per map entry (op_seq.h op_arg_copy_in) -- OP_READ through
    a const T ** parameter, OP_INC into per-entry locals added atomically,
    OP_RW run colour by colour.  Integer-valued data keep every order exact."""
    op2.register_kernel("gen_vcell", """
inline void gen_vcell(const double **x, double **r, const double *w) {
  for (int j = 0; j < 4; j++) {
    r[j][0] += (*w) * x[j][0];
    r[j][1] += x[(j + 1) % 4][1] - x[j][1];
  }
}
""")
    op2.register_kernel("gen_vrw", """
inline void gen_vrw(double **v, const int *e) {
  v[0][0] += 1.0 + (*e % 5);
  v[1][0] -= 2.0;
}
""")
    rng = np.random.default_rng(6)
    nn, nc = 4000, 9000
    cell = np.stack([rng.permutation(nn)[:4] for _ in range(nc)]).astype(np.int32)
    x = rng.integers(-100, 100, size=(nn, 2)).astype(np.float64)
    w = rng.integers(-9, 9, size=nc).astype(np.float64)
    nodes = op2.op_decl_set(nn, "nodes")
    cells = op2.op_decl_set(nc, "cells")
    pcell = op2.op_decl_map(cells, nodes, 4, cell, "pcell")
    px = op2.op_decl_dat(nodes, 2, "double", x, "x")
    pr = op2.op_decl_dat(nodes, 2, "double", None, "r")
    pw = op2.op_decl_dat(cells, 1, "double", w, "w")
    op2.op_par_loop("gen_vcell", cells,
                    op2.op_arg_dat(px, -4, pcell, 2, "double", op2.OP_READ),
                    op2.op_arg_dat(pr, -4, pcell, 2, "double", op2.OP_INC),
                    op2.op_arg_dat(pw, -1, op2.OP_ID, 1, "double", op2.OP_READ))
    ref = np.zeros((nn, 2))
    for j in range(4):
        np.add.at(ref[:, 0], cell[:, j], w * x[cell[:, j], 0])
        np.add.at(ref[:, 1], cell[:, j], x[cell[:, (j + 1) % 4], 1] - x[cell[:, j], 1])
    assert np.array_equal(op2.op_fetch_data(pr), ref)
    # RW through a vector argument of two entries (edge endpoints)
    pp = cell[:, :2].copy()
    edges = op2.op_decl_set(nc, "edges")
    pe = op2.op_decl_map(edges, nodes, 2, pp, "ppedge")
    v0 = rng.integers(-50, 50, size=nn).astype(np.float64)
    pv = op2.op_decl_dat(nodes, 1, "double", v0, "v")
    op2.op_par_loop("gen_vrw", edges, op2.op_arg_dat(pv, -2, pe, 1, "double", op2.OP_RW),
                    op2.op_arg_idx(-1, op2.OP_ID))
    ref_v = v0.copy()
    np.add.at(ref_v, pp[:, 0], 1.0 + np.arange(nc) % 5)
    np.add.at(ref_v, pp[:, 1], -2.0)
    assert np.array_equal(op2.op_fetch_data(pv)[:, 0], ref_v)


def test_optional_arguments_switched_off(op2):
    """op_opt_arg_dat / op_opt_arg_gbl with opt = 0: the kernel still gets a
    pointer (to scratch) and must not use it; the dat and the caller's
    global stay as they were.  With opt = 1 the same loop uses them."""
    op2.register_kernel("gen_opt", """
inline void gen_opt(const double *a, double *b, double *extra, double *gsum) {
  *b = 2.0 * (*a);
  if (gen_use) { *extra += *a; *gsum += *a; }
}
""")
    rng = np.random.default_rng(7)
    n = 3000
    a = rng.integers(-20, 20, size=n).astype(np.float64)
    s = op2.op_decl_set(n, "s")
    pa = op2.op_decl_dat(s, 1, "double", a, "a")
    pb = op2.op_decl_dat(s, 1, "double", None, "b")
    pe = op2.op_decl_dat(s, 1, "double", np.full(n, 5.0), "extra")
    for use in (0, 1):
        op2.op_decl_const(1, "int", np.array([use], np.int32), "gen_use")
        g = np.array([100.0])
        op2.op_par_loop("gen_opt", s,
                        op2.op_arg_dat(pa, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                        op2.op_arg_dat(pb, -1, op2.OP_ID, 1, "double", op2.OP_WRITE),
                        op2.op_opt_arg_dat(use, pe, -1, op2.OP_ID, 1, "double", op2.OP_INC),
                        op2.op_opt_arg_gbl(use, g, 1, "double", op2.OP_INC))
        assert np.array_equal(op2.op_fetch_data(pb)[:, 0], 2.0 * a)
        if use:
            assert np.array_equal(op2.op_fetch_data(pe)[:, 0], 5.0 + a)
            assert g[0] == 100.0 + a.sum()
        else:
            assert np.all(op2.op_fetch_data(pe) == 5.0) and g[0] == 100.0


def test_arg_info_follows_the_best_element(op2):
    """op_arg_info in a run-time compiled loop: the payload the kernel
    writes where its OP_MAX (or OP_MIN) global improves ends at the element
    with the best value, the lowest such element on ties, as the reference's
    CUDA reductions give it; a loop that never beats the caller's value
    leaves the payload alone."""
    op2.register_kernel("gen_argmax", """
inline void gen_argmax(const double *v, const int *i, double *best, int *where) {
  if (*v > *best) { *best = *v; where[0] = *i; where[1] = 7 * (*i); }
}
""")
    op2.register_kernel("gen_argmin", """
inline void gen_argmin(const double *v, const int *i, double *low, int *where) {
  if (*v < *low) { *low = *v; *where = *i; }
}
""")
    rng = np.random.default_rng(8)
    n = 200000
    v = rng.integers(-1000, 1000, size=n).astype(np.float64)
    v[[5000, 123456, 199999]] = 5000.0       # ties for the maximum
    v[[77, 150000]] = -9000.0                 # and for the minimum
    s = op2.op_decl_set(n, "s")
    pv = op2.op_decl_dat(s, 1, "double", v, "v")
    best = np.array([-1e300])
    where = np.array([-1, -1], np.int32)
    op2.op_par_loop("gen_argmax", s, op2.op_arg_dat(pv, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_idx(-1, op2.OP_ID), op2.op_arg_gbl(best, 1, "double", op2.OP_MAX),
                    op2.op_arg_info(where, 2, "int", 2))
    assert best[0] == 5000.0 and list(where) == [5000, 35000]
    low = np.array([1e300])
    w1 = np.array([-1], np.int32)
    op2.op_par_loop("gen_argmin", s, op2.op_arg_dat(pv, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_idx(-1, op2.OP_ID), op2.op_arg_gbl(low, 1, "double", op2.OP_MIN),
                    op2.op_arg_info(w1, 1, "int", 2))
    assert low[0] == -9000.0 and w1[0] == 77
    # the caller's value already better: the payload stays
    best2 = np.array([6000.0])
    w2 = np.array([-5, -6], np.int32)
    op2.op_par_loop("gen_argmax", s, op2.op_arg_dat(pv, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_idx(-1, op2.OP_ID), op2.op_arg_gbl(best2, 1, "double", op2.OP_MAX),
                    op2.op_arg_info(w2, 2, "int", 2))
    assert best2[0] == 6000.0 and list(w2) == [-5, -6]


def test_arg_info_payload_starts_from_the_callers(op2):
    """Each thread's op_arg_info payload starts as the caller's (the
    sequential build copies the caller's payload in before the loop): a
    kernel that writes only part of the payload leaves the rest as the caller
    had it.  A kernel that also writes on ties (>=) returns the payload of
    one element that reaches the best value, never a mix of elements."""
    op2.register_kernel("gen_argmax_part", """
inline void gen_argmax_part(const double *v, const int *i, double *best, int *where) {
  if (*v > *best) { *best = *v; where[0] = *i; }
}
""")
    op2.register_kernel("gen_argmax_ge", """
inline void gen_argmax_ge(const double *v, const int *i, double *best, int *where) {
  if (*v >= *best) { *best = *v; where[0] = *i; where[1] = 3 * (*i); }
}
""")
    rng = np.random.default_rng(4)
    n = 1_000_000                      # more elements than threads: each runs several
    v = rng.integers(0, 100, size=n).astype(np.float64)
    v[654321] = 500.0
    s = op2.op_decl_set(n, "s")
    pv = op2.op_decl_dat(s, 1, "double", v, "v")
    best = np.array([-1.0])
    where = np.array([-1, 42], np.int32)
    op2.op_par_loop("gen_argmax_part", s,
                    op2.op_arg_dat(pv, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_idx(-1, op2.OP_ID), op2.op_arg_gbl(best, 1, "double", op2.OP_MAX),
                    op2.op_arg_info(where, 2, "int", 2))
    assert best[0] == 500.0 and list(where) == [654321, 42]
    # ties everywhere: the value 99 is reached by ~10,000 elements
    v2 = np.minimum(v, 99.0)
    pv2 = op2.op_decl_dat(s, 1, "double", v2, "v2")
    best = np.array([-1.0])
    where = np.array([-1, -1], np.int32)
    op2.op_par_loop("gen_argmax_ge", s,
                    op2.op_arg_dat(pv2, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_idx(-1, op2.OP_ID), op2.op_arg_gbl(best, 1, "double", op2.OP_MAX),
                    op2.op_arg_info(where, 2, "int", 2))
    assert best[0] == 99.0
    assert 0 <= where[0] < n and v2[where[0]] == 99.0 and where[1] == 3 * where[0]


def test_arg_info_payload_too_large_for_the_block_reduction_is_refused(op2):
    op2.register_kernel("gen_argmax_big", """
inline void gen_argmax_big(const double *v, double *best, double *where) {
  if (*v > *best) { *best = *v; where[0] = *v; }
}
""")
    s = op2.op_decl_set(100, "s")
    pv = op2.op_decl_dat(s, 1, "double", np.arange(100.0), "v")
    best = np.array([-1.0])
    where = np.zeros(32)                # 256 bytes a thread: 64 KiB a block
    with pytest.raises(op2.Op2Error, match="shared memory"):
        op2.op_par_loop("gen_argmax_big", s,
                        op2.op_arg_dat(pv, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                        op2.op_arg_gbl(best, 1, "double", op2.OP_MAX),
                        op2.op_arg_info(where, 32, "double", 1))


def test_work_global_is_reloaded_for_every_element(op2):
    """OP_WORK scratch holds the caller's values at the start of every
    element's call, also for the second and later elements a thread runs."""
    op2.register_kernel("gen_work_rd", """
inline void gen_work_rd(const double *a, double *b, double *w) {
  *b = w[0] + w[1];
  w[0] = *a;
}
""")
    n = 1_000_000
    a = np.arange(n, dtype=np.float64)
    s = op2.op_decl_set(n, "s")
    pa = op2.op_decl_dat(s, 1, "double", a, "a")
    pb = op2.op_decl_dat(s, 1, "double", None, "b")
    w = np.array([0.25, 0.5])
    op2.op_par_loop("gen_work_rd", s, op2.op_arg_dat(pa, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_dat(pb, -1, op2.OP_ID, 1, "double", op2.OP_WRITE),
                    op2.op_arg_gbl(w, 2, "double", op2.OP_WORK))
    assert np.all(op2.op_fetch_data(pb)[:, 0] == 0.75)
    assert list(w) == [0.25, 0.5]


def test_work_global_is_per_thread_scratch(op2):
    """An OP_WORK global (op_lib_core.h:114) is scratch: each thread gets
    the caller's values to work in, and nothing is written back."""
    op2.register_kernel("gen_work", """
inline void gen_work(const double *a, double *b, double *w) {
  w[0] = 2.0 * (*a);
  w[1] = w[0] + w[2];
  *b = w[1];
}
""")
    n = 10000
    a = np.arange(n, dtype=np.float64)
    s = op2.op_decl_set(n, "s")
    pa = op2.op_decl_dat(s, 1, "double", a, "a")
    pb = op2.op_decl_dat(s, 1, "double", None, "b")
    w = np.array([0.0, 0.0, 0.5])
    op2.op_par_loop("gen_work", s, op2.op_arg_dat(pa, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_dat(pb, -1, op2.OP_ID, 1, "double", op2.OP_WRITE),
                    op2.op_arg_gbl(w, 3, "double", op2.OP_WORK))
    assert np.array_equal(op2.op_fetch_data(pb)[:, 0], 2.0 * a + 0.5)
    assert list(w) == [0.0, 0.0, 0.5]


def test_application_loop_sharing_an_airfoil_name(op2):
    """An application's own 'update' (jac1's signature) is not Airfoil's: its
    source is compiled and run instead of the hand-written update loop."""
    op2.register_kernel("update", """
inline void update(const double *r, double *du, double *u, int *index, double *u_sum,
                   double *u_max) {
  *u += *du + gen_alpha * (*r);
  *du = 0.0f;
  *u_sum += (*u) * (*u);
  *u_max = (*u_max > *u) ? *u_max : *u;
}
""")
    try:
        rng = np.random.default_rng(3)
        n = 4096
        r_, du, u = (rng.standard_normal(n) for _ in range(3))
        s = op2.op_decl_set(n, "nodes")
        pr = op2.op_decl_dat(s, 1, "double", r_, "r")
        pdu = op2.op_decl_dat(s, 1, "double", du, "du")
        pu = op2.op_decl_dat(s, 1, "double", u, "u")
        op2.op_decl_const(1, "double", 1.0, "gen_alpha")
        usum = np.zeros(1)
        umax = np.zeros(1)
        op2.op_par_loop("update", s,
                        op2.op_arg_dat(pr, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                        op2.op_arg_dat(pdu, -1, op2.OP_ID, 1, "double", op2.OP_RW),
                        op2.op_arg_dat(pu, -1, op2.OP_ID, 1, "double", op2.OP_INC),
                        op2.op_arg_idx(-1, op2.OP_ID),
                        op2.op_arg_gbl(usum, 1, "double", op2.OP_INC),
                        op2.op_arg_gbl(umax, 1, "double", op2.OP_MAX))
        ref = u + (du + 1.0 * r_)  # *u += *du + alpha * (*r)
        assert np.array_equal(op2.op_fetch_data(pu)[:, 0], ref)
        assert np.all(op2.op_fetch_data(pdu) == 0)
        assert abs(usum[0] - (ref * ref).sum()) <= 1e-12 * (ref * ref).sum()
        assert umax[0] == max(0.0, ref.max())
    finally:
        op2.register_kernel("update", None)  # leave no source under an Airfoil name


def test_temporary_and_overlay_dats(op2):
    """op_decl_dat_temp: zeroed, a second one of the same name is refused,
    op_free_dat_temp returns 1 then -1 (op_lib_core.cpp:638-680).
    op_decl_dat_overlay / _ptr: a dat on a smaller set sharing the storage of
    another, host copy and device array (op_lib_core.cpp:581-636)."""
    op2.register_kernel("gen_fill", "inline void gen_fill(double *v, const int *i) { v[0] = *i; v[1] = -(*i); }\n")
    n, m = 1000, 600
    big = op2.op_decl_set(n, "big")
    small = op2.op_decl_set(m, "small")
    t = op2.op_decl_dat_temp(big, 2, "double", "tmp")
    assert np.all(op2.op_fetch_data(t) == 0)
    with pytest.raises(L.Op2Error, match="already exists"):
        op2.op_decl_dat_temp(big, 2, "double", "tmp")
    src = np.arange(2 * n, dtype=np.float64).reshape(n, 2) * 0.5
    d = op2.op_decl_dat(big, 2, "double", src, "d")
    ov = op2.op_decl_dat_overlay(small, d)
    ov2 = op2.op_decl_dat_overlay_ptr(small, src)
    assert ov2.contents.data_d == d.contents.data_d == ov.contents.data_d
    assert ov.contents.data == d.contents.data and ov.contents.set.contents.size == m
    with pytest.raises(L.Op2Error, match="bigger than overlayed"):
        op2.op_decl_dat_overlay(big, op2.op_decl_dat(small, 1, "double", None, "s1"))
    # a loop over the small set through the overlay writes the first m rows of d
    op2.op_par_loop("gen_fill", small, op2.op_arg_dat(ov, -1, op2.OP_ID, 2, "double", op2.OP_WRITE),
                    op2.op_arg_idx(-1, op2.OP_ID))
    got = op2.op_fetch_data(d)
    i = np.arange(m, dtype=np.float64)
    assert np.array_equal(got[:m], np.stack([i, -i], axis=1))
    assert np.array_equal(got[m:], src[m:])
    assert np.array_equal(op2.op_fetch_data(ov), got[:m])
    assert op2.op_free_dat_temp(t) == 1
    assert op2.op_free_dat_temp(t) == -1
    # overlays share storage across sets: renumbering is refused while they exist
    mp = op2.op_decl_map(small, big, 1, np.arange(m, dtype=np.int32).reshape(m, 1), "pm")
    with pytest.raises(L.Op2Error, match="overlay"):
        op2.op_renumber(mp)


ROWS = """
inline void gen_rows(const double *a, double *b, float *c, int *d, const double *x1,
                     const double *x2, double *acc, float **vacc) {
  for (int k = 0; k < 3; k++) b[k] += a[k] * x1[k % 2] - x2[1];
  c[0] = 2.0f * c[1] + (float)a[0];
  c[1] = c[1] - 1.0f;
  d[0] += d[1];
  for (int k = 0; k < 4; k++) acc[k] += a[k % 3] * 0.5 + k;
  for (int j = 0; j < 3; j++) { vacc[j][0] += 1.0f; vacc[j][1] += (float)j; }
}
"""


@pytest.mark.parametrize("n", [1, 31, 33, 1000, 40963])
def test_coalesced_rows_gathers_and_warp_combined_increments(op2, n):
    """The generated loop's warp mode (option jit_warp, the default): direct
    rows read through shared memory (OP_READ, OP_RW, direct OP_INC of double,
    float and int rows), a write-only row stored by the kernel, read-only
    gathers by vector loads, increments combined per warp -- with sets that
    end inside a warp, every element of a warp incrementing the same target,
    and a vector map whose entries repeat within an element.  Equal to numpy
    (exact where no sum is reordered), and to the same loop with jit_warp 0."""
    op2.register_kernel("gen_rows", ROWS)
    rng = np.random.default_rng(n)
    m = 7
    a = rng.standard_normal((n, 3))
    b0 = rng.standard_normal((n, 3))
    c0 = rng.standard_normal((n, 2)).astype(np.float32)
    d0 = rng.integers(-50, 50, size=(n, 2)).astype(np.int32)
    x = rng.standard_normal((m, 2))
    tgt = np.zeros((n, 2), np.int32)            # x1 by map 0; x2 by map 1
    tgt[:, 0] = rng.integers(0, m, n)
    tgt[:, 1] = rng.integers(0, m, n)
    ends = np.zeros((n, 1), np.int32)           # every element increments target 0
    vmap = np.stack([rng.integers(0, m, n)] * 2 + [rng.integers(0, m, n)], 1).astype(np.int32)
    out = {}
    for warp in (1, 0):
        op2.set_option("jit_warp", warp)
        s = op2.op_decl_set(n, f"e{warp}")
        t = op2.op_decl_set(m, f"t{warp}")
        pa = op2.op_decl_dat(s, 3, "double", a, f"a{warp}")
        pb = op2.op_decl_dat(s, 3, "double", b0, f"b{warp}")
        pc = op2.op_decl_dat(s, 2, "float", c0, f"c{warp}")
        pd = op2.op_decl_dat(s, 2, "int", d0, f"d{warp}")
        px = op2.op_decl_dat(t, 2, "double", x, f"x{warp}")
        pacc = op2.op_decl_dat(t, 4, "double", None, f"acc{warp}")
        pv = op2.op_decl_dat(t, 2, "float", None, f"v{warp}")
        mt = op2.op_decl_map(s, t, 2, tgt, f"mt{warp}")
        me = op2.op_decl_map(s, t, 1, ends, f"me{warp}")
        mv = op2.op_decl_map(s, t, 3, vmap, f"mv{warp}")
        A, R, RW, INC, W = op2.op_arg_dat, op2.OP_READ, op2.OP_RW, op2.OP_INC, op2.OP_WRITE
        op2.op_par_loop("gen_rows", s, A(pa, -1, op2.OP_ID, 3, "double", R),
                        A(pb, -1, op2.OP_ID, 3, "double", RW),
                        A(pc, -1, op2.OP_ID, 2, "float", RW),
                        A(pd, -1, op2.OP_ID, 2, "int", INC),
                        A(px, 0, mt, 2, "double", R), A(px, 1, mt, 2, "double", R),
                        A(pacc, 0, me, 4, "double", INC), A(pv, -3, mv, 2, "float", INC))
        out[warp] = [op2.op_fetch_data(p) for p in (pb, pc, pd, pacc, pv)]
    x1, x2 = x[tgt[:, 0]], x[tgt[:, 1]]
    b = b0 + (a * x1[:, [0, 1, 0]] - x2[:, [1]])
    c = np.stack([np.float32(2) * c0[:, 1] + a[:, 0].astype(np.float32),
                  c0[:, 1] - np.float32(1)], 1)
    d = d0.copy()
    d[:, 0] += d0[:, 1]
    acc = np.zeros((m, 4))
    acc[0] = (a[:, [0, 1, 2, 0]] * 0.5 + np.arange(4)).sum(0)
    v = np.zeros((m, 2), np.float32)
    for j in range(3):
        np.add.at(v[:, 0], vmap[:, j], 1.0)
        np.add.at(v[:, 1], vmap[:, j], float(j))
    for warp in (1, 0):
        gb, gc, gd, gacc, gv = out[warp]
        assert np.array_equal(gb, b) and np.array_equal(gc, c) and np.array_equal(gd, d)
        np.testing.assert_allclose(gacc, acc, rtol=1e-12, atol=1e-12 * n)
        assert np.array_equal(gv, v)             # small integers: exact in any order


def test_arg_info_beside_staged_rows_and_combined_increments(op2):
    """A loop with a large op_arg_info payload (16 doubles: 36 KB of the
    block's shared memory for its reduction) beside a read-write direct row
    and an indirect increment: the rows staged through shared memory get only
    what the reduction leaves, and the loop compiles and gives the numpy
    result (argmax payload, rows, increments)."""
    op2.register_kernel("gen_info_rows", """
inline void gen_info_rows(double *r, const int *i, double *acc, double *best, double *pay) {
  r[0] += 1.0; r[1] *= 2.0; r[2] -= r[0];
  for (int k = 0; k < 4; k++) acc[k] += r[k % 3];
  if (r[1] > *best) { *best = r[1]; for (int k = 0; k < 16; k++) pay[k] = k + *i; }
}
""")
    rng = np.random.default_rng(21)
    n, m = 50001, 9
    r0 = rng.standard_normal((n, 3))
    tgt = rng.integers(0, m, size=(n, 1)).astype(np.int32)
    s = op2.op_decl_set(n, "s")
    t = op2.op_decl_set(m, "t")
    pr = op2.op_decl_dat(s, 3, "double", r0, "r")
    pacc = op2.op_decl_dat(t, 4, "double", None, "acc")
    mp = op2.op_decl_map(s, t, 1, tgt, "mp")
    best = np.array([-1e300])
    pay = np.full(16, -1.0)
    op2.op_par_loop("gen_info_rows", s, op2.op_arg_dat(pr, -1, op2.OP_ID, 3, "double", op2.OP_RW),
                    op2.op_arg_idx(-1, op2.OP_ID),
                    op2.op_arg_dat(pacc, 0, mp, 4, "double", op2.OP_INC),
                    op2.op_arg_gbl(best, 1, "double", op2.OP_MAX),
                    op2.op_arg_info(pay, 16, "double", 3))
    r = r0.copy()
    r[:, 0] += 1.0
    r[:, 1] *= 2.0
    r[:, 2] -= r[:, 0]
    assert np.array_equal(op2.op_fetch_data(pr), r)
    acc = np.zeros((m, 4))
    for k in range(4):
        np.add.at(acc[:, k], tgt[:, 0], r[:, k % 3])
    np.testing.assert_allclose(op2.op_fetch_data(pacc), acc, rtol=1e-12, atol=1e-9)
    e = int(np.argmax(r[:, 1]))
    assert best[0] == r[e, 1] and np.array_equal(pay, np.arange(16) + e)


def test_exact_increments_are_the_sequential_loops(op2):
    """Option jit_exact: a generated loop whose only effect is incrementing
    one dat runs owner-computes (each target re-runs the kernel for the
    elements that increment it, in element order, adding into its own sum),
    so the result is the sequential loop's bit for bit: the scatter above
    against numpy's in-order np.add.at, and Airfoil's res_calc and bres_calc
    written as user kernels (op2b.jit_bench's restatement) against the C
    restatement of the reference's sequential loops."""
    from op2b import jit_bench as JB
    from op2b import mesh as M
    from op2b.airfoil import Airfoil
    from oracle import oracle as O
    op2.set_option("jit_exact", 1)
    op2.register_kernel("gen_scatter", EDGES)
    rng, pp = _rng_mesh()
    nn, ne = 5000, pp.shape[0]
    A = rng.standard_normal(ne)
    u = rng.standard_normal((nn, 2))
    du0 = rng.standard_normal((nn, 2))
    nodes = op2.op_decl_set(nn, "nodes")
    edges = op2.op_decl_set(ne, "edges")
    m = op2.op_decl_map(edges, nodes, 2, pp, "ppedge")
    pA = op2.op_decl_dat(edges, 1, "double", A, "A")
    pu = op2.op_decl_dat(nodes, 2, "double", u, "u")
    pdu = op2.op_decl_dat(nodes, 2, "double", du0, "du")
    op2.op_par_loop("gen_scatter", edges,
                    op2.op_arg_dat(pA, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_dat(pu, 1, m, 2, "double", op2.OP_READ),
                    op2.op_arg_dat(pdu, 0, m, 2, "double", op2.OP_INC),
                    op2.op_arg_gbl(np.array([0.75]), 1, "double", op2.OP_READ),
                    op2.op_arg_idx(-1, op2.OP_ID),
                    op2.op_arg_idx(0, m))
    ref = du0.copy()
    e = np.arange(ne)
    np.add.at(ref[:, 0], pp[:, 0], 0.75 * A * u[pp[:, 1], 0])
    np.add.at(ref[:, 1], pp[:, 0], 0.75 * u[pp[:, 1], 1] - e + 0.5 * pp[:, 0])
    assert np.array_equal(op2.op_fetch_data(pdu), ref)
    # Airfoil's increment loops, generated
    mesh = M.channel_bump(60, 30, seed=3)
    app = Airfoil(mesh)
    app.iterate(2)
    for k in ("jres", "jbres"):
        op2.register_kernel(k, JB.KERNELS)
    t, R, INC = "double", op2.OP_READ, op2.OP_INC
    Ad = op2.op_arg_dat
    op2.op_par_loop("jres", app.edges, Ad(app.p_x, 0, app.pedge, 2, t, R),
                    Ad(app.p_x, 1, app.pedge, 2, t, R), Ad(app.p_q, 0, app.pecell, 4, t, R),
                    Ad(app.p_q, 1, app.pecell, 4, t, R), Ad(app.p_adt, 0, app.pecell, 1, t, R),
                    Ad(app.p_adt, 1, app.pecell, 1, t, R), Ad(app.p_res, 0, app.pecell, 4, t, INC),
                    Ad(app.p_res, 1, app.pecell, 4, t, INC))
    op2.op_par_loop("jbres", app.bedges, Ad(app.p_x, 0, app.pbedge, 2, t, R),
                    Ad(app.p_x, 1, app.pbedge, 2, t, R), Ad(app.p_q, 0, app.pbecell, 4, t, R),
                    Ad(app.p_adt, 0, app.pbecell, 1, t, R), Ad(app.p_res, 0, app.pbecell, 4, t, INC),
                    Ad(app.p_bound, -1, op2.OP_ID, 1, "int", R))
    f = app.fetch()
    st = O.State(mesh.ncell, app.c["qinf"])
    st.q[:] = f["q"]
    st.adt[:] = f["adt"]
    st.res[:] = 0.0
    O.loop("res_calc", mesh, app.c, st)
    O.loop("bres_calc", mesh, app.c, st)
    assert np.array_equal(f["res"], st.res)
