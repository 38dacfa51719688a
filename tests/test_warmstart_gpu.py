"""What the learned warm start gains over the freestream start.

* A small end-to-end run: converged fields solved by the batched solver on a
  40x20 family, a network trained on them with the library's kernels (its
  validation error must fall tenfold), and on an unseen mesh and flow the
  plain FP64 iteration from the prediction reaches the freestream run's
  tolerance in at most 85% of the iterations.
* The committed network (op2b/data/gnn_airfoil_200x100.npz: trained on 2,000
  fields at 200x100 by `python -m op2b.warmstart --samples 2000 --val 64
  --steps 4000 --out ...`) at 480x240, a resolution it never saw: at most 80%
  of the freestream iterations to rms < 1e-5 rms0.
* The fallback: a prediction whose first residual exceeds freestream's is
  dropped, and the answer is the freestream solve.
"""
import os

import numpy as np
import pytest

from op2b import gnn as G
from op2b import lib as L
from op2b import warmstart as W
from op2b.mesh import channel_bump

pytestmark = pytest.mark.gpu

DATA = os.path.join(os.path.dirname(G.__file__), "data", "gnn_airfoil_200x100.npz")


@pytest.fixture
def lib():
    from op2b import build
    build.build()
    L.load()
    yield L


def test_small_pipeline_learns_and_beats_freestream(lib):
    fam = W.MeshFamily(40, 20, seed=0)
    flows = W.sample_flows(80, seed=11)
    q, iters, rel = W.solve_family(fam, flows, tol=1e-5, max_iter=40000)
    assert np.all(rel < 1e-5)
    tr = W.Dataset(fam, flows[:64], q[:64])
    va = W.Dataset(fam, flows[64:], q[64:], norm=tr.norm)
    net = G.GraphNet(steps=8, seed=0, norm=tr.norm)
    before = W.evaluate(net, va)
    W.train(net, tr, va, steps=400, batch=8, lr=1e-3, log=lambda s: None)
    after = W.evaluate(net, va)
    assert after < 0.1 * before, (before, after)
    flow = W.sample_flows(1, seed=12)[0]
    mesh = channel_bump(40, 20, seed=5, bump=flow["bump"])
    r = W.warm_vs_freestream(net, mesh, flow, tol_rel=1e-5, log=lambda s: None)
    assert r["warm"]["converged"] and r["free"]["converged"] and not r["fallback"]
    assert r["warm"]["iterations"] <= 0.85 * r["free"]["iterations"], r


def test_committed_network_beats_freestream_at_480x240(lib):
    net = G.GraphNet.load(DATA)
    assert net.n == 1_289_224 and net.steps == 8
    flow = dict(mach=0.45, alpha=2.0, bump=0.06)
    mesh = channel_bump(480, 240, seed=21, bump=flow["bump"])
    r = W.warm_vs_freestream(net, mesh, flow, tol_rel=1e-5, log=lambda s: None)
    assert r["warm"]["converged"] and r["free"]["converged"] and not r["fallback"]
    assert r["warm"]["rms"] < r["tol_abs"]
    assert r["warm"]["iterations"] <= 0.8 * r["free"]["iterations"], r


def test_fallback_to_freestream(lib):
    # an untrained network with an absurd output scale predicts nonsense
    net = G.GraphNet(steps=2, seed=3, norm=[0, 0, 0, 0, 0.5, 0.5, 0.5, 0.5])
    flow = dict(mach=0.5, alpha=1.0, bump=0.05)
    mesh = channel_bump(24, 12, seed=2, bump=flow["bump"])
    r = W.warm_vs_freestream(net, mesh, flow, tol_rel=1e-4, log=lambda s: None)
    assert r["fallback"]
    assert r["warm"]["iterations"] == r["free"]["iterations"] + 1
