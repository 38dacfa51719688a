"""Pins of the oracle (the C restatement in oracle/airfoil_oracle.c).

* against the golden fixtures made by the reference's own sequential build
  (tests/golden/make_golden.py): bit-for-bit rms, maxerr, errloc and fields;
* against the reference builds themselves when oracle/_ref is present;
* the reference's own known-answer tests (tests/functional/{gbl,
  dat_reductions,idx}) built from its sources must print their PASSED lines;
* the size of the increment-order effect the GPU parity tolerance allows for.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN
from op2b import mesh as M
from oracle import oracle as O


def _digest(m):
    import hashlib
    h = hashlib.sha256()
    for a in (m.x, m.cell, m.edge, m.ecell, m.bedge, m.becell, m.bound):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.mark.parametrize("fixture", ["airfoil_24x12_s3.npz", "airfoil_240x120_s1.npz"])
def test_restatement_matches_reference_golden(fixture):
    g = _golden(fixture)
    m = M.channel_bump(int(g["I"]), int(g["J"]), seed=int(g["seed"]))
    assert _digest(m) == str(g["digest"]), "mesh generator drifted from the golden mesh"
    st, rms, mx, el = O.airfoil_run(m, M.airfoil_constants(), int(g["niter"]))
    assert np.array_equal(rms, g["rms"])
    assert np.array_equal(mx, g["maxerr"])
    assert np.array_equal(el, g["errloc"])
    if "q" in g:
        assert np.array_equal(st.q, g["q"])
        assert np.array_equal(st.qold, g["qold"])
        assert np.array_equal(st.res, g["res"])
        assert np.array_equal(st.adt, g["adt"])
    else:
        assert np.array_equal(st.q[g["q_sample_idx"]], g["q_sample"])
        assert np.array_equal(st.adt[g["q_sample_idx"]], g["adt_sample"])
    assert np.array_equal(st.q.sum(axis=0), g["q_sum"])


@pytest.mark.skipif(not O.ref_binary("ref_airfoil_seq_strict"), reason="reference not built")
def test_restatement_matches_reference_build_live():
    m = M.channel_bump(40, 20, seed=11)
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "m.bin")
        M.write_grid_bin(m, p)
        _, a = O.run_reference_airfoil(O.ref_binary("ref_airfoil_seq_strict"), p, 30, m.ncell)
    st, rms, mx, el = O.airfoil_run(m, M.airfoil_constants(), 30)
    assert np.array_equal(a["q"], st.q) and np.array_equal(a["rms"], rms)
    assert np.array_equal(a["maxerr"], mx) and np.array_equal(a["errloc"], el)


@pytest.mark.skipif(not O.ref_binary("ref_airfoil_openmp"), reason="reference not built")
@pytest.mark.parametrize("build", ["ref_airfoil_seq", "ref_airfoil_genseq", "ref_airfoil_openmp"])
def test_reference_builds_agree_with_restatement(build):
    """The reference's -O3 builds (FMA contraction allowed) stay within 1e-13 of the strict one."""
    m = M.channel_bump(40, 20, seed=12)
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "m.bin")
        M.write_grid_bin(m, p)
        _, a = O.run_reference_airfoil(O.ref_binary(build), p, 50, m.ncell,
                                       env={"OMP_NUM_THREADS": "4"})
    st, rms, _, _ = O.airfoil_run(m, M.airfoil_constants(), 50)
    assert np.max(np.abs(a["rms"] / rms - 1)) < 1e-13
    scale = np.abs(st.q).max(axis=0)
    assert np.all(np.abs(a["q"] - st.q).max(axis=0) <= 1e-13 * scale)


@pytest.mark.skipif(not O.ref_binary("gbl_tests"), reason="reference not built")
@pytest.mark.parametrize("kat", ["gbl_tests", "reduc_tests", "idx_tests"])
def test_reference_known_answer_tests_pass(kat):
    out = subprocess.run([O.ref_binary(kat)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "passed" in out.stdout.lower()
    assert "ERROR" not in out.stdout


def test_increment_order_effect_is_far_below_tolerance():
    """Reordering edges (hence res increments) moves rms by ~1e-15 after 100 iterations:
    the 1e-12 relative bound of the GPU parity tests has three orders of headroom."""
    m = M.channel_bump(120, 60, seed=2)
    c = M.airfoil_constants()
    _, r1, _, _ = O.airfoil_run(m, c, 100)
    rng = np.random.default_rng(9)
    m2 = M.renumber_mesh(m, np.arange(m.nnode), np.arange(m.ncell),
                         rng.permutation(m.nedge), rng.permutation(m.nbedge))
    _, r2, _, _ = O.airfoil_run(m2, c, 100)
    assert np.max(np.abs(r2 / r1 - 1)) < 1e-13


def test_planted_mistake_is_caught():
    """A perturbed oracle input (one flipped edge orientation) must break the golden pin."""
    g = _golden("airfoil_24x12_s3.npz")
    m = M.channel_bump(24, 12, seed=3)
    m.edge[5] = m.edge[5][::-1].copy()
    _, rms, _, _ = O.airfoil_run(m, M.airfoil_constants(), 5)
    assert not np.array_equal(rms, g["rms"][:5])
