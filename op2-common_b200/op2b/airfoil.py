"""The Airfoil application on libop2b, through the OP2 API.

Declarations and the time-marching loop follow
apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:175-297 call for call: sets
nodes/edges/bedges/cells, maps pedge/pecell/pbedge/pbecell/pcell, dats
p_bound/p_x/p_q/p_qold/p_adt/p_res, constants gam/gm1/cfl/eps/mach/alpha/qinf,
then per iteration save_soln and two rounds of adt_calc, res_calc, bres_calc,
update, with rms = sqrt(rms/ncell) of the second round.

The op_arg lists are built once and reused every iteration (they do not change
between iterations), so a Python iteration costs nine C calls.
``dtype=np.float32`` declares x/q/qold/adt/res as float: the mixed-precision
form (float storage and fluxes, double update, rms and maxerr).
"""
from __future__ import annotations

import math

import numpy as np

from . import lib as L
from .mesh import Mesh, airfoil_constants


class Airfoil:
    def __init__(self, mesh: Mesh, consts: dict | None = None, dtype=np.float64,
                 rms_only: bool = False, q0: np.ndarray | None = None):
        self.mesh = mesh
        self.c = consts or airfoil_constants()
        self.dtype = np.dtype(dtype)
        t = "double" if self.dtype == np.float64 else "float"
        self.t = t
        ncell = mesh.ncell
        self.nodes = L.op_decl_set(mesh.nnode, "nodes")
        self.edges = L.op_decl_set(mesh.nedge, "edges")
        self.bedges = L.op_decl_set(mesh.nbedge, "bedges")
        self.cells = L.op_decl_set(ncell, "cells")
        self.pedge = L.op_decl_map(self.edges, self.nodes, 2, mesh.edge, "pedge")
        self.pecell = L.op_decl_map(self.edges, self.cells, 2, mesh.ecell, "pecell")
        self.pbedge = L.op_decl_map(self.bedges, self.nodes, 2, mesh.bedge, "pbedge")
        self.pbecell = L.op_decl_map(self.bedges, self.cells, 1, mesh.becell, "pbecell")
        self.pcell = L.op_decl_map(self.cells, self.nodes, 4, mesh.cell, "pcell")
        qinf = np.asarray(self.c["qinf"], np.float64)
        if q0 is None:
            q = np.empty((ncell, 4), self.dtype)
            q[:] = qinf.astype(self.dtype)
        else:
            q = np.ascontiguousarray(q0, dtype=self.dtype)
        self.p_bound = L.op_decl_dat(self.bedges, 1, "int", mesh.bound, "p_bound")
        self.p_x = L.op_decl_dat(self.nodes, 2, t, np.ascontiguousarray(mesh.x, dtype=self.dtype),
                                 "p_x")
        self.p_q = L.op_decl_dat(self.cells, 4, t, q, "p_q")
        # qold, adt and res start at zero, as airfoil.cpp's arrays do: declared
        # without data they are zeroed on the device instead of uploaded
        self.p_qold = L.op_decl_dat(self.cells, 4, t, None, "p_qold")
        self.p_adt = L.op_decl_dat(self.cells, 1, t, None, "p_adt")
        self.p_res = L.op_decl_dat(self.cells, 4, t, None, "p_res")
        for name in ("gam", "gm1", "cfl", "eps", "mach", "alpha"):
            L.op_decl_const(1, "double", self.c[name], name)
        L.op_decl_const(4, "double", qinf, "qinf")
        self.rms = np.zeros(1, np.float64)
        self.maxerr = np.zeros(1, np.float64)
        self.errloc = np.zeros(1, np.int32)
        self.rms_only = rms_only
        self._build_args()

    def _build_args(self):
        t, R, W, RW, INC = self.t, L.OP_READ, L.OP_WRITE, L.OP_RW, L.OP_INC
        A = L.op_arg_dat
        self.a_save = [A(self.p_q, -1, L.OP_ID, 4, t, R), A(self.p_qold, -1, L.OP_ID, 4, t, W)]
        self.a_adt = [A(self.p_x, i, self.pcell, 2, t, R) for i in range(4)] + [
            A(self.p_q, -1, L.OP_ID, 4, t, R), A(self.p_adt, -1, L.OP_ID, 1, t, W)]
        self.a_res = [A(self.p_x, 0, self.pedge, 2, t, R), A(self.p_x, 1, self.pedge, 2, t, R),
                      A(self.p_q, 0, self.pecell, 4, t, R), A(self.p_q, 1, self.pecell, 4, t, R),
                      A(self.p_adt, 0, self.pecell, 1, t, R),
                      A(self.p_adt, 1, self.pecell, 1, t, R),
                      A(self.p_res, 0, self.pecell, 4, t, INC),
                      A(self.p_res, 1, self.pecell, 4, t, INC)]
        self.a_bres = [A(self.p_x, 0, self.pbedge, 2, t, R), A(self.p_x, 1, self.pbedge, 2, t, R),
                       A(self.p_q, 0, self.pbecell, 4, t, R),
                       A(self.p_adt, 0, self.pbecell, 1, t, R),
                       A(self.p_res, 0, self.pbecell, 4, t, INC),
                       A(self.p_bound, -1, L.OP_ID, 1, "int", R)]
        upd = [A(self.p_qold, -1, L.OP_ID, 4, t, R), A(self.p_q, -1, L.OP_ID, 4, t, W),
               A(self.p_res, -1, L.OP_ID, 4, t, RW), A(self.p_adt, -1, L.OP_ID, 1, t, R),
               L.op_arg_gbl(self.rms, 1, "double", L.OP_INC)]
        if not self.rms_only:
            upd += [L.op_arg_gbl(self.maxerr, 1, "double", L.OP_MAX), L.op_arg_idx(-1, L.OP_ID),
                    L.op_arg_info(self.errloc, 1, "int", 5)]
        self.a_upd = upd
        mk = lambda args: (L.op_arg * len(args))(*args)
        self._c = [(b"save_soln", self.cells, mk(self.a_save), 2),
                   (b"adt_calc", self.cells, mk(self.a_adt), 6),
                   (b"res_calc", self.edges, mk(self.a_res), 8),
                   (b"bres_calc", self.bedges, mk(self.a_bres), 6),
                   (b"update", self.cells, mk(self.a_upd), len(upd))]

    def _loop(self, i):
        name, s, arr, n = self._c[i]
        if L.load().op_par_loop_c(name, s, n, arr) != 0:
            raise L.Op2Error(L.last_error())

    def iterate(self, niter: int, history: bool = True):
        """Run `niter` outer iterations; returns [(rms, maxerr, errloc)] per iteration."""
        hist = []
        ncell = self.mesh.ncell
        for _ in range(niter):
            self._loop(0)
            for _k in range(2):
                self._loop(1)
                self._loop(2)
                self._loop(3)
                self.rms[0] = 0.0
                self.maxerr[0] = 0.0
                self.errloc[0] = 0
                self._loop(4)
            r = math.sqrt(self.rms[0] / ncell)
            if history:
                hist.append((r, float(self.maxerr[0]), int(self.errloc[0])))
        return hist

    def renumber(self, stats: bool = True):
        """op_renumber(pecell): RCM on the cell graph, propagated to edges,
        boundary edges and nodes (the call the reference's MPI Airfoil makes);
        returns the bandwidth statistics unless stats is False."""
        return L.op_renumber(self.pecell, stats)

    def fetch_original(self):
        """q in the order the cells were declared (op_fetch_data_idx)."""
        return L.op_fetch_data_idx(self.p_q, 0, self.mesh.ncell - 1)

    def fetch(self):
        return dict(q=L.op_fetch_data(self.p_q), qold=L.op_fetch_data(self.p_qold),
                    res=L.op_fetch_data(self.p_res), adt=L.op_fetch_data(self.p_adt)[:, 0])
