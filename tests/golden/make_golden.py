"""Regenerate the golden fixtures in this directory from the reference's own builds.

Runs the reference's sequential Airfoil build (oracle/_ref/ref_airfoil_seq_strict,
made by oracle/Makefile from the reference sources with -ffp-contract=off) and
its plan builder (oracle/_ref/ref_plan_dump) on seeded meshes from
op2b.mesh.channel_bump, and stores the results as small .npz files.  The
reference tree is not available where the GPU tests run; these files carry its
answers there.

usage: python tests/golden/make_golden.py      (needs `make -C oracle` first)
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
    with tempfile.TemporaryDirectory() as tmp:
        for c in AIRFOIL_CASES:
            airfoil_case(*c, tmp)
        for c in PLAN_CASES:
            plan_case(*c, tmp)


if __name__ == "__main__":
    main()
