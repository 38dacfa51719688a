"""Regenerate the golden fixtures in this directory from the reference's own builds.

Runs the reference's sequential Airfoil build (oracle/_ref/ref_airfoil_seq_strict,
made by oracle/Makefile from the reference sources with -ffp-contract=off) and
its plan builder (oracle/_ref/ref_plan_dump) on seeded meshes from
op2b.mesh.channel_bump, and stores the results as small .npz files.  The
reference tree is not available where the GPU tests run; these files carry its
answers there.

The large case (2400x1200, seed 1) is run on the mesh renumbered by the
restated reverse Cuthill-McKee order (oracle/renumber_oracle.c, the order the
library's op_renumber builds), the numbering the benchmark solves on.  Its
fixture holds SHA-256 digests of the whole q field after 100 and after 1000
iterations in the declared cell order (bit-exact comparison without shipping
92 MB) and the 1000-iteration rms history of the same build on the same mesh.

usage: python tests/golden/make_golden.py [small|plans|large]...
       (needs `make -C oracle` first; no argument runs every group)
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "op2-common_b200"))
sys.path.insert(0, REPO)

from op2b import mesh as M  # noqa: E402
from oracle import oracle as O  # noqa: E402

# (I, J, seed, niter, store full fields?)
AIRFOIL_CASES = [(24, 12, 3, 100, True), (240, 120, 1, 100, False)]
# (I, J, seed, niter, trajectory length): on the RCM-renumbered mesh
AIRFOIL_RCM_CASES = [(2400, 1200, 1, 100, 1000)]
# (I, J, seed, staging, part_size)
PLAN_CASES = [(24, 12, 3, 2, 0), (24, 12, 3, 2, 64), (24, 12, 3, 1, 64), (24, 12, 3, 3, 64),
              (24, 12, 3, 4, 0), (60, 30, 5, 2, 128), (60, 30, 5, 2, 0)]


def mesh_digest(m: M.Mesh) -> str:
    h = hashlib.sha256()
    for a in (m.x, m.cell, m.edge, m.ecell, m.bedge, m.becell, m.bound):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def airfoil_case(I, J, seed, niter, full, tmp):
    m = M.channel_bump(I, J, seed=seed)
    path = os.path.join(tmp, f"m{I}x{J}.bin")
    M.write_grid_bin(m, path)
    summary, a = O.run_reference_airfoil(O.ref_binary("ref_airfoil_seq_strict"), path, niter,
                                         m.ncell)
    out = dict(I=I, J=J, seed=seed, niter=niter, digest=mesh_digest(m), rms=a["rms"],
               maxerr=a["maxerr"], errloc=a["errloc"])
    q = a["q"]
    out["q_sum"] = q.sum(axis=0)
    out["q_sumsq"] = (q * q).sum(axis=0)
    if full:
        out.update(q=q, qold=a["qold"], res=a["res"], adt=a["adt"])
    else:
        sel = np.arange(0, m.ncell, 97)
        out.update(q_sample_idx=sel, q_sample=q[sel], adt_sample=a["adt"][sel])
    np.savez_compressed(os.path.join(HERE, f"airfoil_{I}x{J}_s{seed}.npz"), **out)
    print("airfoil", I, J, summary)


def q_digest(q: np.ndarray) -> str:
    """SHA-256 of a q field as little-endian float64, row-major (cell, component)."""
    return hashlib.sha256(np.ascontiguousarray(q, dtype="<f8").tobytes()).hexdigest()


def airfoil_rcm_case(I, J, seed, niter, niter_traj, tmp):
    m = M.channel_bump(I, J, seed=seed)
    mr, perms = O.rcm_mesh(m)   # the restated op_renumber(pecell)
    pc = perms["cells"]
    path = os.path.join(tmp, f"r{I}x{J}.bin")
    M.write_grid_bin(mr, path)
    binary = O.ref_binary("ref_airfoil_seq_strict")
    summary, a = O.run_reference_airfoil(binary, path, niter, m.ncell)
    q = a["q"][pc]                       # back to the declared cell order
    sel = np.arange(0, m.ncell, 9973)
    out = dict(I=I, J=J, seed=seed, niter=niter, digest=mesh_digest(m),
               rcm_digest=mesh_digest(mr), rms=a["rms"], maxerr=a["maxerr"],
               errloc_rcm=a["errloc"], q_digest=q_digest(q), q_sum=q.sum(axis=0),
               q_sumsq=(q * q).sum(axis=0), q_sample_idx=sel, q_sample=q[sel],
               adt_sample=a["adt"][pc][sel])
    print("airfoil rcm", I, J, niter, summary, flush=True)
    s2, a2 = O.run_reference_airfoil(binary, path, niter_traj, m.ncell)
    assert np.array_equal(a2["rms"][:niter], a["rms"])
    q2 = a2["q"][pc]
    out.update(niter_traj=niter_traj, rms_traj=a2["rms"], maxerr_traj=a2["maxerr"],
               errloc_traj_rcm=a2["errloc"], q_digest_traj=q_digest(q2),
               q_sum_traj=q2.sum(axis=0))
    np.savez_compressed(os.path.join(HERE, f"airfoil_{I}x{J}_s{seed}_rcm.npz"), **out)
    print("airfoil rcm", I, J, niter_traj, s2, flush=True)


def plan_case(I, J, seed, staging, part, tmp):
    m = M.channel_bump(I, J, seed=seed)
    path = os.path.join(tmp, f"m{I}x{J}.bin")
    M.write_grid_bin(m, path)
    prefix = os.path.join(tmp, "plan")
    subprocess.run([O.ref_binary("ref_plan_dump"), path, str(staging), str(part), prefix],
                   check=True, capture_output=True)
    for loop in ("adt_calc", "res_calc", "bres_calc"):
        d = O.read_plan_dump(f"{prefix}.{loop}.plan")
        d["digest"] = np.array(mesh_digest(m))
        np.savez_compressed(os.path.join(HERE, f"plan_{loop}_{I}x{J}_s{seed}_st{staging}_p{part}.npz"),
                            **d)
    print("plan", I, J, staging, part)


def main():
    if not O.ref_binary("ref_airfoil_seq_strict"):
        sys.exit("build the reference first: make -C oracle")
    groups = set(sys.argv[1:]) or {"small", "plans", "large"}
    with tempfile.TemporaryDirectory() as tmp:
        if "small" in groups:
            for c in AIRFOIL_CASES:
                airfoil_case(*c, tmp)
        if "plans" in groups:
            for c in PLAN_CASES:
                plan_case(*c, tmp)
        if "large" in groups:
            for c in AIRFOIL_RCM_CASES:
                airfoil_rcm_case(*c, tmp)


if __name__ == "__main__":
    main()
