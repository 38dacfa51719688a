"""Empty sets through the API: declarations of size 0 (maps and dats without
data), loops over them (direct, indirect increments, reductions: the
globals keep their initial values, as zero iterations of the reference's
sequential loop leave them), loops over non-empty sets with an empty
indirect target range untouched, and fetches of empty dats."""
import numpy as np
import pytest

from op2b import lib as L

pytestmark = pytest.mark.gpu

DIRECT = """
inline void edge_scale(const double *a, double *b, double *s, double *mx, double *mn) {
  *b = 2.0 * (*a);
  *s += *b;
  *mx = (*b > *mx) ? *b : *mx;
  *mn = (*b < *mn) ? *b : *mn;
}
"""

SCATTER = """
inline void edge_scatter(const double *w, double *acc) {
  acc[0] += w[0];
}
"""


def test_loops_over_empty_sets(op2):
    op2.register_kernel("edge_scale", DIRECT)
    op2.register_kernel("edge_scatter", SCATTER)
    empty = op2.op_decl_set(0, "none")
    nodes = op2.op_decl_set(10, "nodes")
    pa = op2.op_decl_dat(empty, 1, "double", None, "a")
    pb = op2.op_decl_dat(empty, 1, "double", None, "b")
    tot, mx, mn = np.array([3.5]), np.array([-7.0]), np.array([7.0])
    op2.op_par_loop("edge_scale", empty,
                    op2.op_arg_dat(pa, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_dat(pb, -1, op2.OP_ID, 1, "double", op2.OP_WRITE),
                    op2.op_arg_gbl(tot, 1, "double", op2.OP_INC),
                    op2.op_arg_gbl(mx, 1, "double", op2.OP_MAX),
                    op2.op_arg_gbl(mn, 1, "double", op2.OP_MIN))
    assert tot[0] == 3.5 and mx[0] == -7.0 and mn[0] == 7.0
    # an indirect increment from an empty set into a non-empty one
    m = op2.op_decl_map(empty, nodes, 1, np.zeros((0, 1), np.int32), "m")
    pw = op2.op_decl_dat(empty, 1, "double", None, "w")
    acc0 = np.arange(10, dtype=np.float64)
    pacc = op2.op_decl_dat(nodes, 1, "double", acc0, "acc")
    op2.op_par_loop("edge_scatter", empty,
                    op2.op_arg_dat(pw, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                    op2.op_arg_dat(pacc, 0, m, 1, "double", op2.OP_INC))
    assert np.array_equal(op2.op_fetch_data(pacc)[:, 0], acc0)
    assert op2.op_fetch_data(pb).shape == (0, 1)


def test_direct_loop_on_a_set_smaller_than_a_warp(op2):
    op2.register_kernel("edge_scale", DIRECT)
    for n in (1, 3, 31, 33):
        s = op2.op_decl_set(n, f"s{n}")
        a = np.linspace(-1.0, 2.0, n)
        pa = op2.op_decl_dat(s, 1, "double", a, f"a{n}")
        pb = op2.op_decl_dat(s, 1, "double", None, f"b{n}")
        tot, mx, mn = np.array([0.0]), np.array([-1e300]), np.array([1e300])
        op2.op_par_loop("edge_scale", s,
                        op2.op_arg_dat(pa, -1, op2.OP_ID, 1, "double", op2.OP_READ),
                        op2.op_arg_dat(pb, -1, op2.OP_ID, 1, "double", op2.OP_WRITE),
                        op2.op_arg_gbl(tot, 1, "double", op2.OP_INC),
                        op2.op_arg_gbl(mx, 1, "double", op2.OP_MAX),
                        op2.op_arg_gbl(mn, 1, "double", op2.OP_MIN))
        b = 2.0 * a
        assert np.array_equal(op2.op_fetch_data(pb)[:, 0], b)
        assert abs(tot[0] - b.sum()) <= 1e-14 * max(1.0, np.abs(b).sum())
        assert mx[0] == b.max() and mn[0] == b.min()


def test_map_with_data_on_an_empty_set_is_refused_only_when_entries_are_out_of_range(op2):
    empty = op2.op_decl_set(0, "none")
    nodes = op2.op_decl_set(4, "nodes")
    # no entries: nothing to check
    assert op2.op_decl_map(empty, nodes, 2, np.zeros((0, 2), np.int32), "m0")
    # a non-empty map with an entry outside the target set is refused
    cells = op2.op_decl_set(2, "cells")
    with pytest.raises(L.Op2Error, match="invalid data for map"):
        op2.op_decl_map(cells, nodes, 2, np.array([[0, 1], [2, 4]], np.int32), "bad")
