"""Batched Airfoil (include/op2b_batch.h) against the oracle.

Every instance of a batch is an independent Airfoil problem with its own
mesh, Mach number, angle of attack and bump: after a fixed number of FP64
iterations its q must match the oracle run of that instance alone (1e-12,
the plain path's tolerance).  The mixed batch must bring every instance to
rms < tol * rms0 through its FP32-then-FP64 phases.  Graph replay and eager
launches give bit-identical q; the autotuner picks a candidate and reports.
"""
import numpy as np
import pytest

from op2b import lib as L
from op2b import mesh as M
from op2b.batch import AirfoilBatch, sample_instances
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPECS = [dict(I=24, J=12, mach=0.4, alpha=2.0, bump=0.05, seed=1),
         dict(I=40, J=20, mach=0.6, alpha=-3.0, bump=0.08, seed=2),
         dict(I=30, J=16, mach=0.3, alpha=5.0, bump=0.0, seed=3)]


def _oracle_q(spec, niter):
    m = M.channel_bump(spec["I"], spec["J"], seed=spec["seed"], bump=spec["bump"])
    c = M.airfoil_constants(mach=spec["mach"], alpha_deg=spec["alpha"])
    st, rms, _, _ = O.airfoil_run(m, c, niter)
    return st.q, rms


@pytest.mark.parametrize("graph,res_kernel,part", [(True, 0, 2048), (False, 0, 2048),
                                                   (True, 1, 512), (True, 2, 256),
                                                   (False, 2, 8192)])
def test_fp64_batch_matches_each_instance(op2, graph, res_kernel, part):
    """Every res_calc strategy of the batch engine (owner computes, atomics,
    edges by colour without atomics) and partition size."""
    b = AirfoilBatch(SPECS, fp32=False)
    b.set("tol", 0.0)
    b.set("res_kernel", res_kernel)
    b.set("part_size", part)
    active, _ = b.run(40, check_every=10, graph=graph)
    assert active == len(SPECS)
    st = b.stats()
    assert list(st["iters"]) == [40] * len(SPECS)
    for i, spec in enumerate(SPECS):
        q_ref, rms = _oracle_q(spec, 40)
        q = b.q_instance(i)
        scale = np.abs(q_ref).max(axis=0)
        assert np.all(np.abs(q - q_ref).max(axis=0) <= 1e-12 * scale), i
        assert abs(st["rms_last"][i] / rms[-1] - 1) < 1e-12
        assert abs(st["rms0"][i] / rms[0] - 1) < 1e-12
    b.close()


def test_graph_and_eager_are_identical(op2):
    qs = []
    for graph in (True, False):
        b = AirfoilBatch(SPECS, fp32=True)
        b.set("tol", 0.0)
        b.run(30, check_every=30, graph=graph)
        qs.append([b.q_instance(i, "fp32") for i in range(len(SPECS))])
        b.close()
        L.op_exit()
        L.op_init()
    for a, c in zip(*qs):
        assert np.array_equal(a, c)


def test_mixed_batch_converges_through_promotion(op2):
    specs = sample_instances(6, seed=4, cells=(300, 2000))
    b = AirfoilBatch(specs, fp32=True)
    b.set("tol", 1e-6)
    b.set("promote_tol", 1e-4)
    active, ms = b.run(200000, check_every=500)
    st = b.stats()
    assert active == 0, st
    assert np.all(st["phase"] == 2)
    assert np.all(st["rms_last"] < 1e-6 * st["rms0"])
    # every instance spent iterations in FP32 storage before finishing in FP64
    assert np.all(st["iters32"] > 0) and np.all(st["iters"] > st["iters32"])
    b.close()


def test_autotuner_picks_and_keeps_state(op2):
    b = AirfoilBatch(SPECS, fp32=True)
    rep = b.tune(iters=5)
    # res_calc strategy (gather, atomic, colour) x block size x partition size
    assert "chosen:" in rep and rep.count("ms/iter") == 27
    for word in ("gather", "atomic", "colour", "part_size=512", "part_size=8192"):
        assert word in rep
    b.set("tol", 0.0)
    b.run(10, check_every=10)
    st = b.stats()
    assert list(st["iters"]) == [10] * len(SPECS)   # tuning did not advance the solve
    b.close()
