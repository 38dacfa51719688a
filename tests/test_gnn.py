"""CPU checks of the learned warm start: the oracle's gradients against
finite differences, the product's parameter layout against the oracle's, and
the mesh graph and features the network reads."""
import numpy as np

from op2b import gnn as G
from op2b import mesh as M
from oracle import gnn_oracle as O


def _small(I=6, J=3, seed=1, bump=0.08):
    m = M.channel_bump(I, J, seed=seed, bump=bump)
    g = G.cell_graph(m)
    return m, g, G.node_features(m, 0.5, 2.0, bump), G.edge_features(m, g)


def test_layout_is_the_oracles():
    for steps in (1, 2, 8):
        assert G.layout(steps=steps) == O.layout(steps=steps)
        assert G.offsets(G.layout(steps=steps)) == O.offsets(O.layout(steps=steps))
    _, n = G.offsets(G.layout(steps=8))
    assert n == 1_289_224


def test_oracle_gradient_matches_finite_differences():
    m, g, ni, ei = _small()
    steps = 2
    lay = O.layout(steps=steps)
    p = G.init_params(lay, seed=3, resid_scale=1.0).astype(np.float64)
    rng = np.random.default_rng(0)
    t = rng.standard_normal((m.ncell, 4))
    loss, grad, _ = O.loss_and_grad(p, lay, g, ni.astype(np.float64), ei.astype(np.float64), t,
                                    steps, rnd=False)
    off, _ = O.offsets(lay)
    which = []
    for key in [("enc_node", 0), ("enc_edge", 1), ("edge0", 0), ("edge1", 2), ("node0", 1),
                ("node1", 0), ("dec", 2), ("dec", 0)]:
        w0, b0, kin, nout = off[key]
        which += [w0 + int(rng.integers(kin * min(nout, 4))), b0 + int(rng.integers(min(nout, 4)))]
    fd = O.finite_difference(p, lay, g, ni.astype(np.float64), ei.astype(np.float64), t, steps,
                             which)
    err = np.abs(grad[which] - fd)
    assert np.all(err <= 1e-4 * np.abs(fd) + 1e-9), np.c_[grad[which], fd]


def test_planted_gradient_mistake_is_caught():
    """A wrong sign in one backward term of the oracle must fail the check."""
    m, g, ni, ei = _small()
    steps = 1
    lay = O.layout(steps=steps)
    p = G.init_params(lay, seed=4, resid_scale=1.0).astype(np.float64)
    t = np.random.default_rng(1).standard_normal((m.ncell, 4))
    good = O.silu_grad
    try:
        O.silu_grad = lambda z: -good(z)
        _, grad, _ = O.loss_and_grad(p, lay, g, ni.astype(np.float64), ei.astype(np.float64), t,
                                     steps, rnd=False)
    finally:
        O.silu_grad = good
    off, _ = O.offsets(lay)
    w0, _, kin, _ = off[("node0", 1)]   # one flipped factor (layer 0 gets two)
    which = [w0 + 3, w0 + kin + 5]
    fd = O.finite_difference(p, lay, g, ni.astype(np.float64), ei.astype(np.float64), t, steps,
                             which)
    assert np.any(np.abs(grad[which] - fd) > 1e-3 * np.abs(fd))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38, 1e-40])
    got = O.bf16(x)
    assert got[0] == 1.0 and got[1] == 1.0            # tie -> even
    assert got[2] == 1.0 + 2 ** -6                      # tie -> even (up)
    assert got[3] == -2.5


def test_cell_graph_is_symmetric_csr():
    m, g, _, _ = _small(12, 6)
    assert g["E"] == 2 * m.nedge
    assert np.array_equal(g["src"][g["rev"]], g["dst"])
    assert np.array_equal(g["dst"][g["rev"]], g["src"])
    for n in range(m.ncell):
        ks = g["idx"][g["off"][n]:g["off"][n + 1]]
        assert np.all(g["dst"][ks] == n) and np.all(np.diff(ks) > 0)
    # interior cells have 4 neighbours
    deg = np.diff(g["off"])
    assert deg.max() == 4 and deg.min() == 2
    b = G.replicate_graph(g, 3)
    assert b["N"] == 3 * g["N"] and b["off"][-1] == 3 * g["E"]
    assert np.array_equal(b["dst"][b["idx"][b["off"][g["N"]]:b["off"][g["N"] + 1]]],
                          np.full(deg[0], g["N"]))


def test_features_do_not_depend_on_resolution():
    """Edge features are unit vectors and a length ratio; node features are
    physical positions and flow parameters -- the same scale on any mesh."""
    for I, J in ((20, 10), (80, 40)):
        m = M.channel_bump(I, J, seed=2, bump=0.06)
        g = G.cell_graph(m)
        ef = G.edge_features(m, g)
        assert np.allclose(np.linalg.norm(ef[:, 0:2], axis=1), 1.0, atol=1e-6)
        assert 0.6 < ef[:, 4].min() and ef[:, 4].max() < 1.6
        nf = G.node_features(m, 0.5, 2.0, 0.06)
        assert nf[:, 0].min() > -1.0 and nf[:, 0].max() < 1.0
        assert nf[:, 5].min() > -1.0 and nf[:, 5].max() < 1.0
        # face normal points from the source cell towards the destination cell
        cen = m.x[m.cell].mean(axis=1)
        d = cen[g["dst"]] - cen[g["src"]]
        assert np.all(np.einsum("ij,ij->i", ef[:, 0:2], d) > 0)
