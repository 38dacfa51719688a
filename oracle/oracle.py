"""ORACLE -- test infrastructure only.

ctypes access to the C restatement (liboracle.so, built from airfoil_oracle.c
and plan_oracle.c by oracle/Makefile) and runners for the reference's own
builds under oracle/_ref/ (made by the same Makefile from the reference
sources).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
import this module, always as the checker or the timed CPU baseline; the
product never does.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


def build(quiet: bool = True) -> None:
    """Compile the restatement (and the reference builds when the reference is present)."""
    out = subprocess.run(["make", "-C", HERE, "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", HERE, "restatement"], check=True, capture_output=True)
        _LIB = ctypes.CDLL(path)
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


def consts_vector(c: dict, dtype=np.float64) -> np.ndarray:
    """k = {gam, gm1, cfl, eps, qinf[0..3]} as the restatement takes it."""
    return np.array([c["gam"], c["gm1"], c["cfl"], c["eps"], *c["qinf"]], dtype=dtype)


class State:
    """AoS Airfoil state: q/qold/res (4 per cell), adt (1 per cell)."""

    def __init__(self, ncell: int, qinf, dtype=np.float64):
        self.q = np.tile(np.asarray(qinf, dtype), (ncell, 1))
        self.qold = np.zeros((ncell, 4), dtype)
        self.res = np.zeros((ncell, 4), dtype)
        self.adt = np.zeros(ncell, dtype)

    def copy(self):
        s = State.__new__(State)
        s.q, s.qold, s.res, s.adt = (a.copy() for a in (self.q, self.qold, self.res, self.adt))
        return s


def _maps(mesh):
    return {k: np.ascontiguousarray(getattr(mesh, k), np.int32)
            for k in ("cell", "edge", "ecell", "bedge", "becell", "bound")}


def airfoil_run(mesh, consts: dict, niter: int, state: State | None = None):
    """Run the restated Airfoil driver; returns (state, rms, maxerr, errloc) histories."""
    L = lib()
    k = consts_vector(consts)
    st = state if state is not None else State(mesh.ncell, consts["qinf"])
    m = _maps(mesh)
    x = np.ascontiguousarray(mesh.x, np.float64)
    rms = np.zeros(max(niter, 1))
    mx = np.zeros(max(niter, 1))
    el = np.zeros(max(niter, 1), np.int32)
    L.orc_airfoil_run(mesh.nnode, mesh.ncell, mesh.nedge, mesh.nbedge, _p(x, _dp),
                      _p(m["cell"], _ip), _p(m["edge"], _ip), _p(m["ecell"], _ip),
                      _p(m["bedge"], _ip), _p(m["becell"], _ip), _p(m["bound"], _ip),
                      _p(st.q, _dp), _p(st.qold, _dp), _p(st.adt, _dp), _p(st.res, _dp),
                      _p(k, _dp), niter, _p(rms, _dp), _p(mx, _dp), _p(el, _ip))
    return st, rms[:niter], mx[:niter], el[:niter]


def airfoil_run_mixed(mesh, consts: dict, niter: int):
    """The mixed-precision restatement: float storage and fluxes, double update/rms."""
    L = lib()
    k = consts_vector(consts, np.float32)
    st = State(mesh.ncell, np.asarray(consts["qinf"], np.float32), np.float32)
    m = _maps(mesh)
    x = np.ascontiguousarray(mesh.x, np.float32)
    rms = np.zeros(max(niter, 1))
    L.orc_airfoil_run_mixed(mesh.ncell, mesh.nedge, mesh.nbedge, _p(x, _fp),
                            _p(m["cell"], _ip), _p(m["edge"], _ip), _p(m["ecell"], _ip),
                            _p(m["bedge"], _ip), _p(m["becell"], _ip), _p(m["bound"], _ip),
                            _p(st.q, _fp), _p(st.qold, _fp), _p(st.adt, _fp), _p(st.res, _fp),
                            _p(k, _fp), niter, _p(rms, _dp))
    return st, rms[:niter]


def loop(name: str, mesh, consts: dict, st: State, dtype=np.float64):
    """Run one restated loop on state ``st`` in place (update returns rms, maxerr, errloc)."""
    L = lib()
    f32 = dtype == np.float32
    P = _fp if f32 else _dp
    sfx = "_f32" if f32 else ""
    k = consts_vector(consts, dtype)
    m = _maps(mesh)
    x = np.ascontiguousarray(mesh.x, dtype)
    if name == "save_soln":
        getattr(L, "orc_save_soln" + sfx)(mesh.ncell, _p(st.q, P), _p(st.qold, P))
    elif name == "adt_calc":
        getattr(L, "orc_adt_calc" + sfx)(mesh.ncell, _p(m["cell"], _ip), _p(x, P), _p(st.q, P),
                                         _p(st.adt, P), _p(k, P))
    elif name == "res_calc":
        getattr(L, "orc_res_calc" + sfx)(mesh.nedge, _p(m["edge"], _ip), _p(m["ecell"], _ip),
                                         _p(x, P), _p(st.q, P), _p(st.adt, P), _p(st.res, P),
                                         _p(k, P))
    elif name == "bres_calc":
        getattr(L, "orc_bres_calc" + sfx)(mesh.nbedge, _p(m["bedge"], _ip), _p(m["becell"], _ip),
                                          _p(m["bound"], _ip), _p(x, P), _p(st.q, P),
                                          _p(st.adt, P), _p(st.res, P), _p(k, P))
    elif name == "update":
        rms = ctypes.c_double(0.0)
        mx = ctypes.c_double(0.0)
        el = ctypes.c_int(0)
        fn = L.orc_update_mixed if f32 else L.orc_update
        fn(mesh.ncell, _p(st.qold, P), _p(st.q, P), _p(st.res, P), _p(st.adt, P),
           ctypes.byref(rms), ctypes.byref(mx), ctypes.byref(el))
        return rms.value, mx.value, el.value
    else:
        raise KeyError(name)
    return None


def airfoil_maps(mesh):
    """Airfoil's sets and maps in the reference's declaration order
    (airfoil.cpp:175-189): sets nodes, edges, bedges, cells; maps pedge,
    pecell, pbedge, pbecell, pcell."""
    sizes = [mesh.nnode, mesh.nedge, mesh.nbedge, mesh.ncell]
    maps = [(1, 0, 2, mesh.edge), (1, 3, 2, mesh.ecell), (2, 0, 2, mesh.bedge),
            (2, 3, 1, mesh.becell), (3, 0, 4, mesh.cell)]
    return sizes, maps


def renumber(sizes, maps, base: int):
    """Restated renumbering: returns [perm or None per set], perm[i] = new index."""
    L = lib()
    nsets, nmaps = len(sizes), len(maps)
    set_size = np.array(sizes, np.int32)
    flat = np.array([[f, t, d] for f, t, d, _ in maps], np.int32).ravel()
    datas = [np.ascontiguousarray(m, np.int32).ravel() for *_, m in maps]
    ptrs = (ctypes.POINTER(ctypes.c_int) * nmaps)(*[_p(d, _ip) for d in datas])
    outs = [np.zeros(max(s, 1), np.int32) for s in sizes]
    optrs = (ctypes.POINTER(ctypes.c_int) * nsets)(*[_p(o, _ip) for o in outs])
    has = np.zeros(nsets, np.int32)
    L.orc_renumber(nsets, _p(set_size, _ip), nmaps, _p(flat, _ip), ptrs, base, optrs,
                   _p(has, _ip))
    return [outs[s][:sizes[s]] if has[s] else None for s in range(nsets)]


def rcm_mesh(mesh):
    """The mesh renumbered by the restated op_renumber(pecell): reverse
    Cuthill-McKee on cells, propagated to edges, boundary edges and nodes (the
    permutations the library's GPU renumbering builds).  Returns (renumbered
    mesh, per-set permutations {nodes, edges, bedges, cells}, perm[i] = new
    index of element i)."""
    from op2b import mesh as M
    sizes, maps = airfoil_maps(mesh)
    pn, pe, pb, pc = renumber(sizes, maps, 1)
    new2old = [np.argsort(p) for p in (pn, pc, pe, pb)]
    return M.renumber_mesh(mesh, *new2old), dict(nodes=pn, edges=pe, bedges=pb, cells=pc)


# ---------------------------------------------------------------- reference builds

def ref_binary(name: str) -> str | None:
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None


def run_reference_airfoil(binary: str, mesh_bin: str, niter: int, ncell: int,
                          env: dict | None = None, outdir: str | None = None):
    """Run one of the reference's Airfoil builds; returns (json summary, arrays)."""
    tmp = outdir or tempfile.mkdtemp(prefix="op2b_ref_")
    prefix = os.path.join(tmp, "run")
    e = dict(os.environ)
    if env:
        e.update(env)
    out = subprocess.run([binary, mesh_bin, str(niter), prefix], capture_output=True,
                         text=True, env=e)
    if out.returncode != 0:
        raise RuntimeError(f"{binary} failed: {out.stdout[-2000:]} {out.stderr[-2000:]}")
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1]
    summary = json.loads(line)
    arrays = {}
    for suffix, dt, shape in (("rms", np.float64, (niter,)), ("maxerr", np.float64, (niter,)),
                              ("errloc", np.int32, (niter,)), ("q", np.float64, (ncell, 4)),
                              ("qold", np.float64, (ncell, 4)), ("res", np.float64, (ncell, 4)),
                              ("adt", np.float64, (ncell,))):
        path = f"{prefix}.{suffix}"
        if os.path.exists(path):
            arrays[suffix] = np.fromfile(path, dtype=dt).reshape(shape)
    return summary, arrays


def run_reference_airfoil_timed(binary: str, mesh_bin: str, niter: int, skip: int,
                                env: dict | None = None):
    """Run a reference Airfoil build for `niter` iterations, timing all but the
    first `skip`; returns (json summary, rms history)."""
    e = dict(os.environ)
    if env:
        e.update(env)
    with tempfile.TemporaryDirectory(prefix="op2b_ref_") as tmp:
        out = subprocess.run([binary, mesh_bin, str(niter), os.path.join(tmp, "run"), str(skip)],
                             capture_output=True, text=True, env=e)
        rp = os.path.join(tmp, "run.rms")
        rms = np.fromfile(rp, dtype=np.float64) if os.path.exists(rp) else None
    if out.returncode != 0:
        raise RuntimeError(f"{binary} failed: {out.stdout[-2000:]} {out.stderr[-2000:]}")
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1]
    return json.loads(line), rms


def read_plan_dump(path: str) -> dict:
    """Parse a plan file written by ref_plan_dump (records of int32/int16/float32 arrays)."""
    out = {}
    with open(path, "rb") as f:
        while True:
            hdr = f.read(4)
            if len(hdr) < 4:
                break
            n = int(np.frombuffer(hdr, np.int32)[0])
            name = f.read(n).decode()
            kind = int(np.frombuffer(f.read(4), np.int32)[0])
            count = int(np.frombuffer(f.read(8), np.int64)[0])
            dt = {0: np.int32, 1: np.int16, 2: np.float32}[kind]
            out[name] = np.frombuffer(f.read(count * np.dtype(dt).itemsize), dt).copy()
    return out
