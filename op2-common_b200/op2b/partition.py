"""Partitioned single-mesh Airfoil: one mesh split over ranks (one GPU each),
with halo exchanges -- the reference's distributed-memory model
(op2/src/mpi/op_mpi_core.cpp:560 op_halo_create, the exchanges of
op2/src/mpi/op_mpi_rt_support.cpp:61-200) on libop2b.

Model (owner computes, as the reference's MPI back end):

* Every cell is owned by one partition (recursive coordinate bisection of
  the cell centroids, `rcb_partition`).  A partition's interior edges are
  those that touch an owned cell; an edge between two partitions is computed
  by both (the reference's redundantly executed "exec halo").  Its boundary
  edges are those of owned cells.
* A partition's local cells are its owned cells, in global order, followed by
  its import halo (the other ends of its edges), grouped by owner rank and in
  global order within a group, so each neighbour's contribution is one
  contiguous slice.  Local edges, boundary edges and nodes keep the global
  order.
* Per outer iteration: save_soln and update run on the owned cells (through
  overlay dats on an owned-cell set, op_decl_dat_overlay); adt_calc runs on
  every local cell (the halo's time steps are needed by the edges on the
  partition boundary); res_calc and bres_calc run on the local edges; after
  each update the owned rows of q that neighbours import are sent to them
  (op2b_dat_pack / op2b_dat_unpack around the transfer).  rms is the sum of
  the partitions' sums.
* An owned cell's residual adds the fluxes of its edges in the local edge
  order, which is the global order: q on the owned cells equals, bit for
  bit, the single-mesh owner-computes run on the same numbering.

`PartAirfoil` is one partition on this process's GPU.  `run_partitioned`
drives several partitions in one process (the transfers are device copies;
no kernel of one partition waits for another) or one partition per rank of a
torch.distributed group (NCCL between GPUs; the transfers use
torch.distributed send/recv of device buffers).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import lib as L
from .mesh import Mesh, airfoil_constants


# ------------------------------------------------------------------ partitioning

def cell_centroids(mesh: Mesh) -> np.ndarray:
    return mesh.x[mesh.cell].mean(axis=1)


def rcb_partition(points: np.ndarray, nparts: int) -> np.ndarray:
    """Recursive coordinate bisection: part id per point.  A group of points
    for k parts is split across its longer extent at the rank that gives the
    two halves floor(k/2) and ceil(k/2) parts' worth of points."""
    part = np.zeros(len(points), np.int32)

    def split(idx, first, k):
        if k == 1 or idx.size == 0:
            part[idx] = first
            return
        p = points[idx]
        ext = p.max(axis=0) - p.min(axis=0)
        axis = int(np.argmax(ext))
        k0 = k // 2
        cut = int(round(idx.size * k0 / k))
        order = np.argsort(p[:, axis], kind="stable")
        split(idx[order[:cut]], first, k0)
        split(idx[order[cut:]], first + k0, k - k0)

    split(np.arange(len(points)), 0, nparts)
    return part


@dataclass
class Part:
    rank: int
    nparts: int
    cells: np.ndarray        # local -> global cell: owned (ascending), then the import halo
    nowned: int
    edges: np.ndarray        # local -> global interior edge (ascending)
    bedges: np.ndarray       # local -> global boundary edge (of owned cells, ascending)
    nodes: np.ndarray        # local -> global node (ascending)
    mesh: Mesh               # the local mesh, maps in local numbering
    imports: dict = field(default_factory=dict)   # owner rank -> (first local row, count)
    exports: dict = field(default_factory=dict)   # rank -> local owned rows it imports

    @property
    def nhalo(self) -> int:
        return int(self.cells.size - self.nowned)


def partition(mesh: Mesh, nparts: int, cell_part: np.ndarray | None = None) -> list[Part]:
    """Split `mesh` into `nparts` partitions (cell_part: owner of each cell;
    default: recursive coordinate bisection of the centroids)."""
    if nparts < 1:
        raise ValueError("nparts must be at least 1")
    if cell_part is None:
        cell_part = rcb_partition(cell_centroids(mesh), nparts)
    cell_part = np.asarray(cell_part, np.int32)
    if cell_part.shape != (mesh.ncell,) or cell_part.min() < 0 or cell_part.max() >= nparts:
        raise ValueError("cell_part must give every cell a part in [0, nparts)")
    parts = []
    owner_e = cell_part[mesh.ecell]                      # (nedge, 2)
    for p in range(nparts):
        owned = np.flatnonzero(cell_part == p).astype(np.int64)
        edges = np.flatnonzero((owner_e == p).any(axis=1)).astype(np.int64)
        ends = mesh.ecell[edges].ravel()
        halo = np.unique(ends[cell_part[ends] != p])
        halo = halo[np.lexsort((halo, cell_part[halo]))]  # by owner, then global id
        cells = np.concatenate([owned, halo]).astype(np.int64)
        bedges = np.flatnonzero(cell_part[mesh.becell] == p).astype(np.int64)
        nodes = np.unique(np.concatenate([mesh.cell[cells].ravel(), mesh.edge[edges].ravel(),
                                          mesh.bedge[bedges].ravel()]))
        g2l_cell = np.full(mesh.ncell, -1, np.int64)
        g2l_cell[cells] = np.arange(cells.size)
        g2l_node = lambda a: np.searchsorted(nodes, a).astype(np.int32)
        local = Mesh(x=np.ascontiguousarray(mesh.x[nodes]),
                     cell=g2l_node(mesh.cell[cells]),
                     edge=g2l_node(mesh.edge[edges]),
                     ecell=g2l_cell[mesh.ecell[edges]].astype(np.int32),
                     bedge=g2l_node(mesh.bedge[bedges]),
                     becell=g2l_cell[mesh.becell[bedges]].astype(np.int32),
                     bound=np.ascontiguousarray(mesh.bound[bedges]).astype(np.int32),
                     meta=dict(mesh.meta, part=p, nparts=nparts))
        imports = {}
        if halo.size:
            owners = cell_part[halo]
            for r in np.unique(owners):
                sel = np.flatnonzero(owners == r)
                imports[int(r)] = (int(owned.size + sel[0]), int(sel.size))
        parts.append(Part(rank=p, nparts=nparts, cells=cells, nowned=int(owned.size),
                          edges=edges, bedges=bedges, nodes=nodes, mesh=local, imports=imports))
    # exports: what each neighbour imports from p, as p's local (owned) rows
    for q in parts:
        for p, (first, n) in q.imports.items():
            src = parts[p]
            g = q.cells[first:first + n]
            pos = np.searchsorted(src.cells[:src.nowned], g)
            assert np.array_equal(src.cells[pos], g)
            src.exports[q.rank] = pos.astype(np.int32)
    return parts


# ------------------------------------------------------------------ one partition on the GPU

class PartAirfoil:
    """One partition of the Airfoil mesh on this process's GPU, through the
    OP2 API (apps/c/airfoil/airfoil_plain/dp/airfoil.cpp's sets, maps, dats
    and loops), with an owned-cell set whose overlay dats carry save_soln and
    update."""

    def __init__(self, part: Part, consts: dict | None = None, dtype=np.float64):
        import torch
        self.part = part
        self.c = consts or airfoil_constants()
        m = part.mesh
        t = "double" if np.dtype(dtype) == np.float64 else "float"
        self.t, self.dtype = t, np.dtype(dtype)
        self.nodes = L.op_decl_set(m.nnode, "nodes")
        self.edges = L.op_decl_set(m.nedge, "edges")
        self.bedges = L.op_decl_set(m.nbedge, "bedges")
        self.cells = L.op_decl_set(m.ncell, "cells")
        self.owned = L.op_decl_set(part.nowned, "cells_owned")
        self.pedge = L.op_decl_map(self.edges, self.nodes, 2, m.edge, "pedge")
        self.pecell = L.op_decl_map(self.edges, self.cells, 2, m.ecell, "pecell")
        self.pbedge = L.op_decl_map(self.bedges, self.nodes, 2, m.bedge, "pbedge")
        self.pbecell = L.op_decl_map(self.bedges, self.cells, 1, m.becell, "pbecell")
        self.pcell = L.op_decl_map(self.cells, self.nodes, 4, m.cell, "pcell")
        qinf = np.asarray(self.c["qinf"], np.float64)
        q = np.empty((m.ncell, 4), self.dtype)
        q[:] = qinf.astype(self.dtype)
        self.p_bound = L.op_decl_dat(self.bedges, 1, "int", m.bound, "p_bound")
        self.p_x = L.op_decl_dat(self.nodes, 2, t, np.ascontiguousarray(m.x, dtype=self.dtype),
                                 "p_x")
        self.p_q = L.op_decl_dat(self.cells, 4, t, q, "p_q")
        self.p_qold = L.op_decl_dat(self.cells, 4, t, None, "p_qold")
        self.p_adt = L.op_decl_dat(self.cells, 1, t, None, "p_adt")
        self.p_res = L.op_decl_dat(self.cells, 4, t, None, "p_res")
        # the owned rows (the first nowned) of q, qold, res and adt
        ov = lambda d: L.load().op_decl_dat_overlay(self.owned, d)
        self.q_o, self.qold_o, self.res_o, self.adt_o = (ov(d) for d in (
            self.p_q, self.p_qold, self.p_res, self.p_adt))
        if not all((self.q_o, self.qold_o, self.res_o, self.adt_o)):
            raise L.Op2Error(L.last_error())
        for name in ("gam", "gm1", "cfl", "eps", "mach", "alpha"):
            L.op_decl_const(1, "double", self.c[name], name)
        L.op_decl_const(4, "double", qinf, "qinf")
        self.rms = np.zeros(1, np.float64)
        self.maxerr = np.zeros(1, np.float64)
        self.errloc = np.zeros(1, np.int32)
        self._build_args()
        # export rows on the device, and transfer buffers per neighbour
        dev = torch.device("cuda", torch.cuda.current_device())
        tdt = torch.float64 if self.dtype == np.float64 else torch.float32
        self.export_rows = {r: torch.from_numpy(rows).to(dev) for r, rows in part.exports.items()}
        self.send_buf = {r: torch.empty((rows.size, 4), dtype=tdt, device=dev)
                         for r, rows in part.exports.items()}
        self.recv_buf = {r: torch.empty((n, 4), dtype=tdt, device=dev)
                         for r, (_, n) in part.imports.items()}

    def _build_args(self):
        t, R, W, RW, INC = self.t, L.OP_READ, L.OP_WRITE, L.OP_RW, L.OP_INC
        A = L.op_arg_dat
        mk = lambda args: (L.op_arg * len(args))(*args)
        save = [A(self.q_o, -1, L.OP_ID, 4, t, R), A(self.qold_o, -1, L.OP_ID, 4, t, W)]
        adt = [A(self.p_x, i, self.pcell, 2, t, R) for i in range(4)] + [
            A(self.p_q, -1, L.OP_ID, 4, t, R), A(self.p_adt, -1, L.OP_ID, 1, t, W)]
        res = [A(self.p_x, 0, self.pedge, 2, t, R), A(self.p_x, 1, self.pedge, 2, t, R),
               A(self.p_q, 0, self.pecell, 4, t, R), A(self.p_q, 1, self.pecell, 4, t, R),
               A(self.p_adt, 0, self.pecell, 1, t, R), A(self.p_adt, 1, self.pecell, 1, t, R),
               A(self.p_res, 0, self.pecell, 4, t, INC), A(self.p_res, 1, self.pecell, 4, t, INC)]
        bres = [A(self.p_x, 0, self.pbedge, 2, t, R), A(self.p_x, 1, self.pbedge, 2, t, R),
                A(self.p_q, 0, self.pbecell, 4, t, R), A(self.p_adt, 0, self.pbecell, 1, t, R),
                A(self.p_res, 0, self.pbecell, 4, t, INC),
                A(self.p_bound, -1, L.OP_ID, 1, "int", R)]
        upd = [A(self.qold_o, -1, L.OP_ID, 4, t, R), A(self.q_o, -1, L.OP_ID, 4, t, W),
               A(self.res_o, -1, L.OP_ID, 4, t, RW), A(self.adt_o, -1, L.OP_ID, 1, t, R),
               L.op_arg_gbl(self.rms, 1, "double", L.OP_INC),
               L.op_arg_gbl(self.maxerr, 1, "double", L.OP_MAX), L.op_arg_idx(-1, L.OP_ID),
               L.op_arg_info(self.errloc, 1, "int", 5)]
        self._loops = [(b"save_soln", self.owned, mk(save), 2),
                       (b"adt_calc", self.cells, mk(adt), 6),
                       (b"res_calc", self.edges, mk(res), 8),
                       (b"bres_calc", self.bedges, mk(bres), 6),
                       (b"update", self.owned, mk(upd), 8)]

    def loop(self, i):
        name, s, arr, n = self._loops[i]
        if L.load().op_par_loop_c(name, s, n, arr) != 0:
            raise L.Op2Error(L.last_error())

    def pack(self, rank):
        rows, buf = self.export_rows[rank], self.send_buf[rank]
        if L.load().op2b_dat_pack(self.p_q, rows.data_ptr(), rows.numel(), buf.data_ptr()) != 0:
            raise L.Op2Error(L.last_error())
        return buf

    def unpack(self, rank, buf):
        first, n = self.part.imports[rank]
        if L.load().op2b_dat_unpack(self.p_q, None, first, n, buf.data_ptr()) != 0:
            raise L.Op2Error(L.last_error())

    def fetch_owned(self) -> np.ndarray:
        return L.op_fetch_data_idx(self.p_q, 0, self.part.nowned - 1)


def _exchange_local(parts: list[PartAirfoil]):
    """Halo transfers between partitions held by this process: each
    neighbour's export rows packed into its buffer, then unpacked into the
    importer's halo slice (device copies on the library's stream)."""
    for p in parts:
        for r in p.part.imports:
            p.unpack(r, parts[r].pack(p.part.rank))


def _exchange_dist(p: PartAirfoil, dist):
    """Halo transfer of this rank's partition with its neighbours over a
    torch.distributed group (device buffers; NCCL between GPUs)."""
    import torch
    for r in p.part.exports:
        p.pack(r)
    L.synchronize()
    ops = [dist.P2POp(dist.isend, p.send_buf[r], r) for r in p.part.exports]
    ops += [dist.P2POp(dist.irecv, p.recv_buf[r], r) for r in p.part.imports]
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    torch.cuda.synchronize()
    for r in p.part.imports:
        p.unpack(r, p.recv_buf[r])


def run_partitioned(parts: list[PartAirfoil], niter: int, ncell_total: int, dist=None):
    """Outer iterations of the partitioned Airfoil (airfoil.cpp:221-297 with a
    halo exchange after each update).  `parts`: the partitions this process
    holds (all of them, or this rank's one with `dist` given).  Returns
    [(rms, maxerr, global errloc)] per iteration."""
    hist = []
    for _ in range(niter):
        for p in parts:
            p.loop(0)
        for _k in range(2):
            for p in parts:
                p.loop(1)
                p.loop(2)
                p.loop(3)
                p.rms[0] = 0.0
                p.maxerr[0] = 0.0
                p.errloc[0] = 0
                p.loop(4)
            if dist is None:
                _exchange_local(parts)
            else:
                _exchange_dist(parts[0], dist)
        rms = sum(float(p.rms[0]) for p in parts)
        best = max(parts, key=lambda p: (float(p.maxerr[0]), -int(p.part.cells[p.errloc[0]])))
        mx, loc = float(best.maxerr[0]), int(best.part.cells[best.errloc[0]])
        if dist is not None:
            import torch
            t = torch.tensor([rms, mx, -loc], dtype=torch.float64, device="cuda")
            tot = t.clone()
            dist.all_reduce(tot[:1])
            rms = float(tot[0])
            allm = [torch.zeros(2, dtype=torch.float64, device="cuda")
                    for _ in range(dist.get_world_size())]
            dist.all_gather(allm, t[1:].contiguous())
            mx, neg = max((float(a[0]), float(a[1])) for a in allm)
            loc = int(-neg)
        hist.append((math.sqrt(rms / ncell_total), mx, loc))
    return hist
