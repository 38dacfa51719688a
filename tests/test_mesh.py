"""The seeded channel-with-bump generator: sizes, orientation, closure, file formats."""
import os
import tempfile

import numpy as np
import pytest

from op2b import mesh as M


@pytest.mark.parametrize("I,J", [(24, 12), (240, 120)])
def test_sizes(I, J):
    m = M.channel_bump(I, J, seed=1)
    assert m.nnode == (I + 1) * (J + 1)
    assert m.ncell == I * J
    assert m.nedge == (J - 1) * I + (I - 1) * J
    assert m.nbedge == 2 * (I + J)
    M.check_mesh(m)


def test_orientation_and_closure():
    m = M.channel_bump(30, 15, seed=4)
    x = m.x
    d = x[m.edge[:, 0]] - x[m.edge[:, 1]]
    n = np.stack([d[:, 1], -d[:, 0]], 1)
    cen = x[m.cell].mean(1)
    # normal (dy, -dx) points from c1 into c2 (res_calc.h sign convention)
    assert (np.einsum("ij,ij->i", n, cen[m.ecell[:, 1]] - cen[m.ecell[:, 0]]) > 0).all()
    db = x[m.bedge[:, 0]] - x[m.bedge[:, 1]]
    nb = np.stack([db[:, 1], -db[:, 0]], 1)
    mid = 0.5 * (x[m.bedge[:, 0]] + x[m.bedge[:, 1]])
    assert (np.einsum("ij,ij->i", nb, mid - cen[m.becell]) > 0).all()
    # every cell is closed: outward normals sum to zero
    s = np.zeros((m.ncell, 2))
    np.add.at(s, m.ecell[:, 0], n)
    np.add.at(s, m.ecell[:, 1], -n)
    np.add.at(s, m.becell, nb)
    assert np.abs(s).max() < 1e-15
    assert (np.bincount(m.ecell.ravel(), minlength=m.ncell)
            + np.bincount(m.becell, minlength=m.ncell) == 4).all()
    assert set(np.unique(m.bound)) == {1, 2}
    assert (m.bound == 1).sum() == 60 and (m.bound == 2).sum() == 30


def test_seeded_and_permuted():
    a = M.channel_bump(20, 10, seed=7)
    b = M.channel_bump(20, 10, seed=7)
    c = M.channel_bump(20, 10, seed=8)
    assert np.array_equal(a.ecell, b.ecell) and np.array_equal(a.x, b.x)
    assert not np.array_equal(a.ecell, c.ecell)
    s = M.channel_bump(20, 10, seed=7, permute=False)
    assert not np.array_equal(s.ecell, a.ecell)


def test_file_round_trips():
    m = M.channel_bump(16, 8, seed=2)
    with tempfile.TemporaryDirectory() as tmp:
        pb = os.path.join(tmp, "m.bin")
        pt = os.path.join(tmp, "new_grid.dat")
        M.write_grid_bin(m, pb)
        M.write_grid_dat(m, pt)
        for r in (M.read_grid_bin(pb), M.read_grid_dat(pt)):
            for k in ("x", "cell", "edge", "ecell", "bedge", "becell", "bound"):
                assert np.array_equal(getattr(r, k), getattr(m, k)), k


def test_constants_match_reference_literals():
    c = M.airfoil_constants()
    assert c["gam"] == float(np.float32(1.4)) and c["cfl"] == float(np.float32(0.9))
    assert c["gm1"] == c["gam"] - 1.0 and c["eps"] == float(np.float32(0.05))
    assert c["qinf"][2] == 0.0 and c["qinf"][0] == 1.0


def test_fe_grid_for_aero():
    """FE_grid.dat as the reference's aero reads it (aero.cpp:79-117): the
    header, the nodes, each cell's nodes in the bilinear element's tensor
    order (the corner opposite node 0 last) and the far-field nodes."""
    m = M.channel_bump(12, 6, seed=3)
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "FE_grid.dat")
        M.write_fe_grid_dat(m, p)
        lines = open(p).read().split("\n")
    nnode, ncell, nb = (int(v) for v in lines[0].split())
    bnode = np.unique(m.bedge[m.bound == 2].reshape(-1))
    assert (nnode, ncell, nb) == (m.nnode, m.ncell, bnode.size)
    x = np.array([[float(v) for v in ln.split()] for ln in lines[1:1 + nnode]])
    assert np.array_equal(x, m.x)
    cells = np.array([[int(v) for v in ln.split()] for ln in lines[1 + nnode:1 + nnode + ncell]])
    assert np.array_equal(cells, m.cell[:, [0, 1, 3, 2]])
    # tensor order: node 3 is the corner diagonal to node 0 (no shared edge)
    e = {tuple(sorted(p)) for p in m.edge.tolist()} | {tuple(sorted(p)) for p in m.bedge.tolist()}
    for c in cells[:50]:
        assert tuple(sorted((c[0], c[1]))) in e and tuple(sorted((c[0], c[2]))) in e
        assert tuple(sorted((c[0], c[3]))) not in e
    got = np.array([int(v) for v in lines[1 + nnode + ncell:1 + nnode + ncell + nb]])
    assert np.array_equal(got, bnode)
