"""Batched Airfoil through the C ABI of include/op2b_batch.h.

Instances (meshes of uneven size, each with its own Mach number, angle of
attack and bump height) are concatenated into one OP2 mesh, declared once
(sets and maps) with the Airfoil dats in float and in double, renumbered
(op_renumber: every instance then owns contiguous ranges), and solved together:
one persistent launch per loop stage, one CUDA graph per iteration, FP32
storage until an instance's rms falls below promote_tol * rms0 (or stalls),
FP64 to tol * rms0.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import lib as L
from .mesh import Mesh, airfoil_constants, channel_bump


class op2b_airfoil_dats(ctypes.Structure):
    _fields_ = [("pcell", L.op_map), ("pedge", L.op_map), ("pecell", L.op_map),
                ("pbedge", L.op_map), ("pbecell", L.op_map), ("p_x", L.op_dat),
                ("p_q", L.op_dat), ("p_qold", L.op_dat), ("p_adt", L.op_dat),
                ("p_res", L.op_dat), ("p_bound", L.op_dat)]


_BATCH_SIGS = {
    "op2b_batch_create": (ctypes.c_void_p, [ctypes.POINTER(op2b_airfoil_dats),
                                            ctypes.POINTER(op2b_airfoil_dats), ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "op2b_batch_set": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]),
    "op2b_batch_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                                       ctypes.c_int]),
    "op2b_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_double)]),
    "op2b_batch_stats": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 5),
    "op2b_batch_destroy": (None, [ctypes.c_void_p]),
}


def _lib():
    lib = L.load()
    if not getattr(lib, "_batch_sigs", False):
        for name, (res, args) in _BATCH_SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        lib._batch_sigs = True
    return lib


def sample_instances(n: int, seed: int = 0, cells=(10_000, 500_000)):
    """Config-4 style instances: cells log-uniform in `cells` (aspect 2:1), Mach
    uniform in [0.3, 0.7], angle of attack uniform in [-4, 6] degrees, bump
    height uniform in [0, 0.1] of the channel height."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        c = math.exp(rng.uniform(math.log(cells[0]), math.log(cells[1])))
        J = max(2, int(round(math.sqrt(c / 2.0))))
        out.append(dict(I=2 * J, J=J, mach=float(rng.uniform(0.3, 0.7)),
                        alpha=float(rng.uniform(-4.0, 6.0)), bump=float(rng.uniform(0.0, 0.1)),
                        seed=int(seed * 1000 + i)))
    return out


def concat(meshes):
    """One mesh with every instance's elements and maps offset; offsets per set."""
    off = {k: [0] for k in ("n", "c", "e", "b")}
    xs, cells, edges, ecells, bedges, becells, bounds = [], [], [], [], [], [], []
    for m in meshes:
        n0, c0 = off["n"][-1], off["c"][-1]
        xs.append(m.x)
        cells.append(m.cell + n0)
        edges.append(m.edge + n0)
        ecells.append(m.ecell + c0)
        bedges.append(m.bedge + n0)
        becells.append(m.becell + c0)
        bounds.append(m.bound)
        off["n"].append(n0 + m.nnode)
        off["c"].append(c0 + m.ncell)
        off["e"].append(off["e"][-1] + m.nedge)
        off["b"].append(off["b"][-1] + m.nbedge)
    cat = lambda a: np.ascontiguousarray(np.concatenate(a))
    mesh = Mesh(x=cat(xs), cell=cat(cells).astype(np.int32), edge=cat(edges).astype(np.int32),
                ecell=cat(ecells).astype(np.int32), bedge=cat(bedges).astype(np.int32),
                becell=cat(becells).astype(np.int32), bound=cat(bounds).astype(np.int32))
    return mesh, {k: np.array(v) for k, v in off.items()}


class AirfoilBatch:
    def __init__(self, specs, fp32: bool = True, renumber: bool = True, meshes=None):
        """specs: per instance I, J, mach, alpha, bump, seed; `meshes` (optional)
        supplies the instances' meshes instead of generating them from I, J, seed."""
        self.specs = list(specs)
        if meshes is None:
            meshes = [channel_bump(s["I"], s["J"], seed=s["seed"], bump=s["bump"]) for s in specs]
        if len(meshes) != len(self.specs):
            raise L.Op2Error("one mesh per instance")
        self.meshes = meshes
        mesh, off = concat(meshes)
        self.mesh = mesh
        k0 = airfoil_constants()
        consts = [airfoil_constants(mach=s["mach"], alpha_deg=s["alpha"]) for s in specs]
        qinf = np.array([c["qinf"] for c in consts])
        q0 = np.repeat(qinf, np.diff(off["c"]), axis=0)
        s_nodes = L.op_decl_set(mesh.nnode, "nodes")
        s_edges = L.op_decl_set(mesh.nedge, "edges")
        s_bedges = L.op_decl_set(mesh.nbedge, "bedges")
        s_cells = L.op_decl_set(mesh.ncell, "cells")
        self.sets = (s_nodes, s_edges, s_bedges, s_cells)
        pedge = L.op_decl_map(s_edges, s_nodes, 2, mesh.edge, "pedge")
        pecell = L.op_decl_map(s_edges, s_cells, 2, mesh.ecell, "pecell")
        pbedge = L.op_decl_map(s_bedges, s_nodes, 2, mesh.bedge, "pbedge")
        pbecell = L.op_decl_map(s_bedges, s_cells, 1, mesh.becell, "pbecell")
        pcell = L.op_decl_map(s_cells, s_nodes, 4, mesh.cell, "pcell")
        bound = L.op_decl_dat(s_bedges, 1, "int", mesh.bound, "p_bound")
        nc = mesh.ncell

        def dats(dt, t, sfx):
            return op2b_airfoil_dats(
                pcell, pedge, pecell, pbedge, pbecell,
                L.op_decl_dat(s_nodes, 2, t, mesh.x.astype(dt), "p_x" + sfx),
                L.op_decl_dat(s_cells, 4, t, q0.astype(dt), "p_q" + sfx),
                L.op_decl_dat(s_cells, 4, t, np.zeros((nc, 4), dt), "p_qold" + sfx),
                L.op_decl_dat(s_cells, 1, t, np.zeros(nc, dt), "p_adt" + sfx),
                L.op_decl_dat(s_cells, 4, t, np.zeros((nc, 4), dt), "p_res" + sfx), bound)

        self.d64 = dats(np.float64, "double", "")
        self.d32 = dats(np.float32, "float", "32") if fp32 else None
        for name in ("gam", "gm1", "cfl", "eps"):
            L.op_decl_const(1, "double", k0[name], name)
        L.op_decl_const(4, "double", k0["qinf"], "qinf")
        order = np.arange(len(specs))
        cell_off, edge_off = off["c"], off["e"]
        self.renumber_stats = None
        if renumber:
            self.renumber_stats = L.op_renumber(pecell)
            pc = L.set_permutation(s_cells)
            pe = L.set_permutation(s_edges)
            starts, cranges, eranges = [], [], []
            for i in range(len(specs)):
                cs = pc[cell_off[i]:cell_off[i + 1]]
                es = pe[edge_off[i]:edge_off[i + 1]]
                if cs.max() - cs.min() + 1 != cs.size or es.max() - es.min() + 1 != es.size:
                    raise L.Op2Error("renumbering did not keep instances contiguous")
                starts.append(cs.min())
                cranges.append((cs.min(), cs.size))
                eranges.append((es.min(), es.size))
            order = np.argsort(starts)
            cell_off = np.concatenate([[0], np.cumsum([cranges[i][1] for i in order])])
            edge_off = np.concatenate([[0], np.cumsum([eranges[i][1] for i in order])])
            if not all(cranges[i][0] == cell_off[k] for k, i in enumerate(order)):
                raise L.Op2Error("cell ranges are not consecutive")
            if not all(eranges[i][0] == edge_off[k] for k, i in enumerate(order)):
                raise L.Op2Error("edge ranges are not consecutive")
        self.order = order               # batch slot k holds instance order[k]
        self.cell_off = np.ascontiguousarray(cell_off, np.int32)
        self.edge_off = np.ascontiguousarray(edge_off, np.int32)
        qinf_sorted = np.ascontiguousarray(qinf[order], np.float64)
        lib = _lib()
        h = lib.op2b_batch_create(ctypes.byref(self.d32) if self.d32 else None,
                                  ctypes.byref(self.d64), len(specs),
                                  self.cell_off.ctypes.data, self.edge_off.ctypes.data,
                                  qinf_sorted.ctypes.data)
        if not h:
            raise L.Op2Error(L.last_error())
        self.h = h

    def set(self, key: str, value: float):
        if _lib().op2b_batch_set(self.h, key.encode(), float(value)) != 0:
            raise L.Op2Error(L.last_error())

    def tune(self, iters: int = 10) -> str:
        buf = ctypes.create_string_buffer(4096)
        if _lib().op2b_batch_tune(self.h, iters, buf, 4096) != 0:
            raise L.Op2Error(L.last_error())
        return buf.value.decode()

    def run(self, max_iterations: int, check_every: int = 100, graph: bool = True):
        ms = ctypes.c_double(0.0)
        n = _lib().op2b_batch_run(self.h, max_iterations, check_every, int(graph),
                                  ctypes.byref(ms))
        if n < 0:
            raise L.Op2Error(L.last_error())
        return n, ms.value

    def stats(self):
        n = len(self.specs)
        it = np.zeros(n, np.int32)
        it32 = np.zeros(n, np.int32)
        r0 = np.zeros(n)
        rl = np.zeros(n)
        ph = np.zeros(n, np.int32)
        if _lib().op2b_batch_stats(self.h, it.ctypes.data, it32.ctypes.data, r0.ctypes.data,
                                   rl.ctypes.data, ph.ctypes.data) != 0:
            raise L.Op2Error(L.last_error())
        inv = np.argsort(self.order)     # back to the caller's instance order
        return dict(iters=it[inv], iters32=it32[inv], rms0=r0[inv], rms_last=rl[inv],
                    phase=ph[inv])

    def q_instance(self, i: int, precision: str = "fp64") -> np.ndarray:
        """q of instance i (caller's order) in its declared cell order."""
        full = self.q_all(precision)
        c0 = sum(m.ncell for m in self.meshes[:i])
        return full[c0:c0 + self.meshes[i].ncell]

    def q_all(self, precision: str = "fp64") -> np.ndarray:
        """q of every instance, concatenated in the caller's order, declared cell order."""
        d = self.d64 if precision == "fp64" else self.d32
        return L.op_fetch_data_idx(d.p_q, 0, self.mesh.ncell - 1)

    def q_final(self) -> list:
        """Each instance's q from the precision it finished in (FP32 if it never
        left the FP32 phase, FP64 otherwise), as float64 arrays."""
        st = self.stats()
        need32 = bool(np.any(st["iters32"] == st["iters"])) and self.d32 is not None
        q64 = self.q_all("fp64")
        q32 = self.q_all("fp32").astype(np.float64) if need32 else None
        out, c0 = [], 0
        for i, m in enumerate(self.meshes):
            src = q32 if (need32 and st["iters32"][i] == st["iters"][i]) else q64
            out.append(src[c0:c0 + m.ncell].copy())
            c0 += m.ncell
        return out

    def close(self):
        if getattr(self, "h", None):
            _lib().op2b_batch_destroy(self.h)
            self.h = None
