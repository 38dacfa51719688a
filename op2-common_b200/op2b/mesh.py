"""Seeded synthetic Airfoil meshes: a 2-D channel with a bump on its lower wall.

The reference Airfoil driver reads its unstructured quad mesh from
``new_grid.dat`` (apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:94-141): a header
``nnode ncell nedge nbedge``, then ``x y`` per node, four node ids per cell,
``n1 n2 c1 c2`` per interior edge and ``n1 n2 c bound`` per boundary edge.
That mesh is not shipped with the reference, so this module generates meshes of
the same shape from a seed and writes them in the same text layout (and in a
compact binary layout used by the oracle harnesses and the benchmark).

Geometry: channel ``length x height`` (2 x 1), lower wall with a sin^2 bump of
height ``bump*height`` on ``[0.25, 0.75]*length``; ``I x J`` quads; interior
node coordinates perturbed uniformly by ``+-perturb`` of the local spacing.
Boundary flag: 1 = wall (lower and upper), 2 = far field (inlet and outlet),
the two values bres_calc distinguishes (apps/c/airfoil/airfoil_plain/dp/
bres_calc.h:12).

Orientation follows the flux convention of res_calc.h:4-7 and bres_calc.h:4-5:
with ``(dx, dy) = x(n1) - x(n2)`` the normal ``(dy, -dx)`` points from ``c1``
into ``c2`` for an interior edge, and out of the cell for a boundary edge.

Numbering: with ``permute=True`` nodes, cells, edges and boundary edges are
each shuffled by a seeded permutation, so every map is unstructured.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

_BIN_MAGIC = 0x4F503242  # "OP2B"


@dataclass
class Mesh:
    x: np.ndarray        # (nnode, 2) float64 node coordinates
    cell: np.ndarray     # (ncell, 4) int32 nodes of each cell, counter-clockwise
    edge: np.ndarray     # (nedge, 2) int32 nodes of each interior edge
    ecell: np.ndarray    # (nedge, 2) int32 cells either side of each interior edge
    bedge: np.ndarray    # (nbedge, 2) int32 nodes of each boundary edge
    becell: np.ndarray   # (nbedge,) int32 cell of each boundary edge
    bound: np.ndarray    # (nbedge,) int32 1 = wall, 2 = far field
    meta: dict = field(default_factory=dict)

    @property
    def nnode(self) -> int:
        return int(self.x.shape[0])

    @property
    def ncell(self) -> int:
        return int(self.cell.shape[0])

    @property
    def nedge(self) -> int:
        return int(self.edge.shape[0])

    @property
    def nbedge(self) -> int:
        return int(self.bedge.shape[0])

    def sizes(self):
        return self.nnode, self.ncell, self.nedge, self.nbedge


def _orient(x, a, b, ref_from, ref_to):
    """Swap (a, b) where the normal (dy, -dx) of x[a]-x[b] points against ref_to-ref_from."""
    d = x[a] - x[b]
    nrm = np.stack([d[:, 1], -d[:, 0]], axis=1)
    flip = np.einsum("ij,ij->i", nrm, ref_to - ref_from) < 0
    a2 = np.where(flip, b, a)
    b2 = np.where(flip, a, b)
    return a2.astype(np.int32), b2.astype(np.int32)


def channel_bump(I: int, J: int, seed: int = 0, length: float = 2.0,
                 height: float = 1.0, bump: float = 0.05, perturb: float = 0.10,
                 permute: bool = True) -> Mesh:
    """Generate the I x J channel-with-bump quad mesh described in the module docstring."""
    if I < 1 or J < 1:
        raise ValueError("mesh needs at least one cell in each direction")
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(I + 1), np.arange(J + 1), indexing="ij")
    xs = length * ii / I
    lo, hi = 0.25 * length, 0.75 * length
    inside = (xs >= lo) & (xs <= hi)
    ylow = np.where(inside, bump * height * np.sin(math.pi * (xs - lo) / (hi - lo)) ** 2, 0.0)
    ys = ylow + (height - ylow) * jj / J
    interior = (ii > 0) & (ii < I) & (jj > 0) & (jj < J)
    du = rng.uniform(-perturb, perturb, size=xs.shape)
    dv = rng.uniform(-perturb, perturb, size=xs.shape)
    xs = np.where(interior, xs + du * (length / I), xs)
    ys = np.where(interior, ys + dv * (height - ylow) / J, ys)
    x = np.stack([xs.ravel(), ys.ravel()], axis=1).astype(np.float64)

    def nid(i, j):
        return i * (J + 1) + j

    def cid(i, j):
        return i * J + j

    ci, cj = np.meshgrid(np.arange(I), np.arange(J), indexing="ij")
    ci, cj = ci.ravel(), cj.ravel()
    cell = np.stack([nid(ci, cj), nid(ci + 1, cj), nid(ci + 1, cj + 1), nid(ci, cj + 1)],
                    axis=1).astype(np.int32)
    cen = x[cell].mean(axis=1)

    # interior edges between cell (i-1, j) and (i, j)
    vi, vj = np.meshgrid(np.arange(1, I), np.arange(J), indexing="ij")
    vi, vj = vi.ravel(), vj.ravel()
    # interior edges between cell (i, j-1) and (i, j)
    hi_, hj = np.meshgrid(np.arange(I), np.arange(1, J), indexing="ij")
    hi_, hj = hi_.ravel(), hj.ravel()
    ea = np.concatenate([nid(vi, vj), nid(hi_, hj)])
    eb = np.concatenate([nid(vi, vj + 1), nid(hi_ + 1, hj)])
    c1 = np.concatenate([cid(vi - 1, vj), cid(hi_, hj - 1)])
    c2 = np.concatenate([cid(vi, vj), cid(hi_, hj)])
    ea, eb = _orient(x, ea, eb, cen[c1], cen[c2])
    edge = np.stack([ea, eb], axis=1)
    ecell = np.stack([c1, c2], axis=1).astype(np.int32)

    bi = np.arange(I)
    bj = np.arange(J)
    ba = np.concatenate([nid(bi, 0), nid(bi, J), nid(0, bj), nid(I, bj)])
    bb = np.concatenate([nid(bi + 1, 0), nid(bi + 1, J), nid(0, bj + 1), nid(I, bj + 1)])
    bc = np.concatenate([cid(bi, 0), cid(bi, J - 1), cid(0, bj), cid(I - 1, bj)]).astype(np.int32)
    bound = np.concatenate([np.ones(2 * I, np.int32), np.full(2 * J, 2, np.int32)])
    mid = 0.5 * (x[ba] + x[bb])
    ba, bb = _orient(x, ba, bb, cen[bc], mid)
    bedge = np.stack([ba, bb], axis=1)

    mesh = Mesh(x=x, cell=cell, edge=edge, ecell=ecell, bedge=bedge, becell=bc,
                bound=bound, meta=dict(I=I, J=J, seed=seed, bump=bump,
                                       perturb=perturb, permuted=bool(permute)))
    if permute:
        mesh = permute_mesh(mesh, rng)
    return mesh


def permute_mesh(mesh: Mesh, rng: np.random.Generator) -> Mesh:
    """Shuffle node, cell, edge and boundary-edge numbering with one generator."""
    pn = rng.permutation(mesh.nnode)   # new node k is old node pn[k]
    pc = rng.permutation(mesh.ncell)
    pe = rng.permutation(mesh.nedge)
    pb = rng.permutation(mesh.nbedge)
    return renumber_mesh(mesh, pn, pc, pe, pb)


def renumber_mesh(mesh: Mesh, pn, pc, pe, pb) -> Mesh:
    """Apply new->old orderings ``pn, pc, pe, pb`` to every array and map of the mesh."""
    inv_n = np.empty_like(pn)
    inv_n[pn] = np.arange(pn.size)
    inv_c = np.empty_like(pc)
    inv_c[pc] = np.arange(pc.size)
    return Mesh(
        x=np.ascontiguousarray(mesh.x[pn]),
        cell=inv_n[mesh.cell[pc]].astype(np.int32),
        edge=inv_n[mesh.edge[pe]].astype(np.int32),
        ecell=inv_c[mesh.ecell[pe]].astype(np.int32),
        bedge=inv_n[mesh.bedge[pb]].astype(np.int32),
        becell=inv_c[mesh.becell[pb]].astype(np.int32),
        bound=np.ascontiguousarray(mesh.bound[pb]).astype(np.int32),
        meta=dict(mesh.meta),
    )


def airfoil_constants(mach: float | None = None, alpha_deg: float | None = None):
    """Flow constants as the reference driver sets them.

    apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:149-164 stores float literals in
    doubles (``gam = 1.4f`` ...) and sets ``qinf[2] = 0`` so the angle of attack
    never enters the flow.  With ``mach=None, alpha_deg=None`` this returns those
    exact double values.  Passing ``mach`` replaces the 0.4f Mach number, and
    passing ``alpha_deg`` tilts the freestream velocity to
    ``(cos a, sin a)`` -- an extension used by the batched and learned forms,
    which vary the flow condition per instance.
    """
    f32 = lambda v: float(np.float32(v))
    gam = f32(1.4)
    gm1 = gam - 1.0
    cfl = f32(0.9)
    eps = f32(0.05)
    m = f32(0.4) if mach is None else float(mach)
    p = 1.0
    r = 1.0
    u = math.sqrt(gam * p / r) * m
    e = p / (r * gm1) + 0.5 * u * u
    if alpha_deg is None:
        qinf = [r, r * u, 0.0, r * e]
    else:
        a = math.radians(alpha_deg)
        qinf = [r, r * u * math.cos(a), r * u * math.sin(a), r * e]
    return dict(gam=gam, gm1=gm1, cfl=cfl, eps=eps, mach=m,
                alpha=0.0 if alpha_deg is None else math.radians(alpha_deg),
                qinf=np.array(qinf, np.float64))


def write_grid_dat(mesh: Mesh, path: str) -> None:
    """Write the mesh in the reference's new_grid.dat text layout (exact doubles)."""
    with open(path, "w") as f:
        f.write(f"{mesh.nnode} {mesh.ncell} {mesh.nedge} {mesh.nbedge} \n")
        np.savetxt(f, mesh.x, fmt="%.17g %.17g")
        np.savetxt(f, mesh.cell, fmt="%d %d %d %d")
        np.savetxt(f, np.concatenate([mesh.edge, mesh.ecell], axis=1), fmt="%d %d %d %d")
        np.savetxt(f, np.concatenate([mesh.bedge, mesh.becell[:, None], mesh.bound[:, None]],
                                     axis=1), fmt="%d %d %d %d")


def write_fe_grid_dat(mesh: Mesh, path: str) -> None:
    """Write the mesh as the reference's aero application reads it from
    FE_grid.dat (apps/c/aero/aero_plain/aero.cpp:79-117): a header
    ``nnode ncell nbnodes``, ``x y`` per node, four node ids per cell in the
    bilinear element's tensor order -- (0,0), (1,0), (0,1), (1,1), the order
    its shape-function derivatives Ng2_xi assume -- and one id per boundary
    node, ascending.  The boundary nodes (aero's Dirichlet set, where the
    potential stays at its free-stream value) are the far-field ones (bound
    2); the walls keep the natural no-flux condition, so the flow has to go
    round the bump."""
    bnode = np.unique(mesh.bedge[mesh.bound == 2].reshape(-1))
    with open(path, "w") as f:
        f.write(f"{mesh.nnode} {mesh.ncell} {bnode.size} \n")
        np.savetxt(f, mesh.x, fmt="%.17g %.17g")
        np.savetxt(f, mesh.cell[:, [0, 1, 3, 2]], fmt="%d %d %d %d")
        np.savetxt(f, bnode, fmt="%d")


def read_grid_dat(path: str) -> Mesh:
    with open(path) as f:
        nnode, ncell, nedge, nbedge = (int(v) for v in f.readline().split())
        data = np.loadtxt(f, max_rows=nnode)
        x = data.reshape(nnode, 2)
        f_rest = np.loadtxt(f, dtype=np.int64).reshape(-1, 4)
    cell = f_rest[:ncell].astype(np.int32)
    e = f_rest[ncell:ncell + nedge].astype(np.int32)
    b = f_rest[ncell + nedge:ncell + nedge + nbedge].astype(np.int32)
    return Mesh(x=x, cell=cell, edge=e[:, :2].copy(), ecell=e[:, 2:].copy(),
                bedge=b[:, :2].copy(), becell=b[:, 2].copy(), bound=b[:, 3].copy())


def write_grid_bin(mesh: Mesh, path: str) -> None:
    """Binary layout: int32 magic,nnode,ncell,nedge,nbedge then x,cell,edge,ecell,bedge,becell,bound."""
    with open(path, "wb") as f:
        f.write(struct.pack("<5i", _BIN_MAGIC, *mesh.sizes()))
        for a, t in ((mesh.x, np.float64), (mesh.cell, np.int32), (mesh.edge, np.int32),
                     (mesh.ecell, np.int32), (mesh.bedge, np.int32), (mesh.becell, np.int32),
                     (mesh.bound, np.int32)):
            f.write(np.ascontiguousarray(a, dtype=t).tobytes())


def read_grid_bin(path: str) -> Mesh:
    with open(path, "rb") as f:
        magic, nn, nc, ne, nb = struct.unpack("<5i", f.read(20))
        if magic != _BIN_MAGIC:
            raise ValueError(f"{path}: not an op2b binary mesh")
        rd = lambda t, n: np.frombuffer(f.read(n * np.dtype(t).itemsize), dtype=t).copy()
        x = rd(np.float64, 2 * nn).reshape(nn, 2)
        cell = rd(np.int32, 4 * nc).reshape(nc, 4)
        edge = rd(np.int32, 2 * ne).reshape(ne, 2)
        ecell = rd(np.int32, 2 * ne).reshape(ne, 2)
        bedge = rd(np.int32, 2 * nb).reshape(nb, 2)
        becell = rd(np.int32, nb)
        bound = rd(np.int32, nb)
    return Mesh(x=x, cell=cell, edge=edge, ecell=ecell, bedge=bedge, becell=becell, bound=bound)


def check_mesh(mesh: Mesh) -> None:
    """Validate map ranges the way op_decl_map's check_map does (op_lib_core.cpp:146-164)."""
    for name, arr, hi in (("pcell", mesh.cell, mesh.nnode), ("pedge", mesh.edge, mesh.nnode),
                          ("pecell", mesh.ecell, mesh.ncell), ("pbedge", mesh.bedge, mesh.nnode),
                          ("pbecell", mesh.becell, mesh.ncell)):
        if arr.size and (arr.min() < 0 or arr.max() >= hi):
            raise ValueError(f"map {name} has entries outside [0, {hi})")
