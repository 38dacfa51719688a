"""Learned warm start for Airfoil: a message-passing graph network on the
solver's own mesh, trained and run by the kernels of include/op2b_gnn.h.

The graph is the mesh's cell graph: one node per cell, two directed edges per
interior edge (pecell; edge 2i runs c1 -> c2, edge 2i+1 the reverse).  Node
inputs: the cell centroid, the flow condition (Mach, angle of attack), the
bump height, the wall shape under the cell and the cell's boundary flags; edge
inputs: the unit face normal, the unit centroid-to-centroid direction and
their length ratio -- all independent of the mesh resolution, so a network
trained at 200x100 runs at 480x240 or 2400x1200.  The network predicts
(q - qinf), normalised per component; the solver then iterates from
qinf + prediction.

Encode - process - decode (the CPU restatement in the oracle pins the same
definition):
    h0 = MLP(node_in), e0 = MLP(edge_in)
    L steps: e' = e + MLP([e, h_src, h_dst]); agg = sum of e' into each node;
             h' = h + MLP([h, agg])
    out = MLP(h_L)
Every MLP is Linear-SiLU-Linear-SiLU-Linear, width 128, bf16 weights and
activations on the tensor cores with FP32 accumulation (op2b_gemm_bf16), FP32
master weights and AdamW moments.  PyTorch only allocates device memory and
provides the stream; every kernel is the library's.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import lib as L
from .mesh import Mesh

EPI_STORE_F32, EPI_ATOMIC_F32, EPI_STORE_BF16, EPI_BIAS_BF16, EPI_BIAS_SILU_BF16, \
    EPI_SILU_GRAD_BF16 = range(6)
WIDTH = 128
NODE_IN = 16
EDGE_IN = 8
OUT = 8        # 4 predicted components, padded to the tensor-core N granularity

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_long
_F = ctypes.c_float
_GNN_SIGS = {
    "op2b_gemm_bf16": (_I, [_I, _I, _I, _P, _L, _L, _P, _L, _L, _P, _L, _I, _P, _P, _P, _L, _I,
                            _I, _P]),
    "op2b_gemm_error": (_I, [_I]),
    "op2b_gnn_gather_pair": (_I, [_I, _I, _P, _P, _P, _L, _P, _L, _I, _P]),
    "op2b_gnn_aggregate": (_I, [_I, _I, _P, _P, _P, _L, _P, _L, _P]),
    "op2b_gnn_to_bf16": (_I, [_I, _I, _P, _L, _P, _L, _P]),
    "op2b_gnn_add_f32": (_I, [_I, _I, _P, _P, _L, _P]),
    "op2b_gnn_edge_grad": (_I, [_I, _I, _P, _P, _P, _L, _P, _P]),
    "op2b_gnn_cat_grad": (_I, [_I, _I, _I, _P, _L, _P, _P, _P, _P, _P, _P]),
    "op2b_gnn_colsum": (_I, [_I, _I, _P, _L, _P, _P]),
    "op2b_gnn_mse": (_I, [_I, _I, _P, _L, _P, _P, _P, _F, _P]),
    "op2b_gnn_adam": (_I, [_L, _P, _P, _P, _P, _P, _F, _F, _F, _F, _F, _P]),
    "op2b_gnn_memset": (_I, [_P, _I, _L, _P]),
    "op2b_gnn_decode_q": (_I, [_I, _P, _L, _P, _P, _P, _P]),
}


def _lib():
    lib = L.load()
    if not getattr(lib, "_gnn_sigs", False):
        for name, (res, args) in _GNN_SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        lib._gnn_sigs = True
    return lib


def _call(name, *args):
    if getattr(_lib(), name)(*args) != 0:
        raise L.Op2Error(L.last_error())


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise L.Op2Error("the learned warm start needs a CUDA device (no CPU path)")
    return torch


# ---------------------------------------------------------------- parameters
def layout(node_in=NODE_IN, edge_in=EDGE_IN, width=WIDTH, steps=8, out=OUT):
    """[(mlp name, [(k_in, n_out) per layer])] in parameter order."""
    w = width
    mlps = [("enc_node", [(node_in, w), (w, w), (w, w)]),
            ("enc_edge", [(edge_in, w), (w, w), (w, w)])]
    for l in range(steps):
        mlps.append((f"edge{l}", [(3 * w, w), (w, w), (w, w)]))
        mlps.append((f"node{l}", [(2 * w, w), (w, w), (w, w)]))
    mlps.append(("dec", [(w, w), (w, w), (w, out)]))
    return mlps


def offsets(lay):
    """Flat offsets {(mlp, layer): (w_off, b_off, k_in, n_out)} and the total size.
    W is stored [n_out][k_in] (rows k-contiguous: the B operand of X W^T)."""
    off, o = {}, 0
    for name, layers in lay:
        for i, (kin, nout) in enumerate(layers):
            off[(name, i)] = (o, o + kin * nout, kin, nout)
            o += kin * nout + nout
    return off, o


def init_params(lay, seed=0, resid_scale=0.1):
    """LeCun-normal weights, zero biases; the last layer of every residual
    branch scaled by resid_scale; decoder rows >= 4 zero (padding)."""
    off, n = offsets(lay)
    rng = np.random.default_rng(seed)
    p = np.zeros(n, np.float32)
    for (name, i), (w0, b0, kin, nout) in off.items():
        W = rng.standard_normal((nout, kin)) / math.sqrt(kin)
        if i == 2 and (name.startswith("edge") or name.startswith("node")):
            W *= resid_scale
        if name == "dec" and i == 2:
            W[4:] = 0.0
        p[w0:w0 + kin * nout] = W.ravel()
    return p


# ---------------------------------------------------------------- graph + features
def cell_graph(mesh: Mesh):
    """Directed cell graph: src, dst (2 per interior edge), rev, and the CSR
    (off, idx) of incoming edges per cell in increasing edge order."""
    c = mesh.ecell.astype(np.int64)
    E = 2 * c.shape[0]
    src = np.empty(E, np.int32)
    dst = np.empty(E, np.int32)
    src[0::2], dst[0::2] = c[:, 0], c[:, 1]
    src[1::2], dst[1::2] = c[:, 1], c[:, 0]
    rev = (np.arange(E) ^ 1).astype(np.int32)
    idx = np.argsort(dst, kind="stable").astype(np.int32)
    off = np.zeros(mesh.ncell + 1, np.int32)
    np.cumsum(np.bincount(dst, minlength=mesh.ncell), out=off[1:])
    return dict(src=src, dst=dst, rev=rev, off=off, idx=idx, N=mesh.ncell, E=E)


def replicate_graph(g, copies):
    """Disjoint union of `copies` copies of graph g (a batch of samples)."""
    N, E = g["N"], g["E"]
    out = dict(N=N * copies, E=E * copies)
    for k in ("src", "dst", "rev", "idx"):
        base = N if k in ("src", "dst") else E
        out[k] = np.concatenate([g[k] + i * base for i in range(copies)]).astype(np.int32)
    offs = [g["off"][:-1] + i * E for i in range(copies)] + [np.array([copies * E])]
    out["off"] = np.concatenate(offs).astype(np.int32)
    return out


def _wall(xc, bump, length=2.0, height=1.0):
    lo, hi = 0.25 * length, 0.75 * length
    inside = (xc >= lo) & (xc <= hi)
    return np.where(inside, bump * height * np.sin(math.pi * (xc - lo) / (hi - lo)) ** 2, 0.0)


def node_features(mesh: Mesh, mach, alpha_deg, bump):
    """(ncell, 16) float32: centroid x, y (scaled to [-1, 1]), Mach, angle of
    attack, bump height, height above the lower wall (fraction of the local
    channel height), wall shape under the cell, wall / far-field flags."""
    cen = mesh.x[mesh.cell].mean(axis=1)
    ylow = _wall(cen[:, 0], bump)
    eta = (cen[:, 1] - ylow) / (1.0 - ylow)
    f = np.zeros((mesh.ncell, NODE_IN), np.float32)
    f[:, 0] = cen[:, 0] - 1.0
    f[:, 1] = 2.0 * cen[:, 1] - 1.0
    f[:, 2] = (mach - 0.5) / 0.2
    f[:, 3] = alpha_deg / 5.0
    f[:, 4] = (bump - 0.05) / 0.05
    f[:, 5] = 2.0 * eta - 1.0
    f[:, 6] = ylow / 0.05
    wall = np.zeros(mesh.ncell)
    far = np.zeros(mesh.ncell)
    np.add.at(wall, mesh.becell[mesh.bound == 1], 1.0)
    np.add.at(far, mesh.becell[mesh.bound == 2], 1.0)
    f[:, 7] = wall
    f[:, 8] = far
    return f


def edge_features(mesh: Mesh, g=None):
    """(2 * nedge, 8) float32 per directed edge: unit face normal (pointing
    from source to destination cell), unit centroid direction, face length /
    centroid distance."""
    g = g or cell_graph(mesh)
    cen = mesh.x[mesh.cell].mean(axis=1)
    d = mesh.x[mesh.edge[:, 0]] - mesh.x[mesh.edge[:, 1]]
    nrm = np.stack([d[:, 1], -d[:, 0]], axis=1)          # from c1 into c2 (res_calc.h)
    nd = np.empty((g["E"], 2))
    nd[0::2], nd[1::2] = nrm, -nrm
    cd = cen[g["dst"]] - cen[g["src"]]
    ln = np.linalg.norm(nd, axis=1)
    lc = np.linalg.norm(cd, axis=1)
    f = np.zeros((g["E"], EDGE_IN), np.float32)
    f[:, 0:2] = nd / ln[:, None]
    f[:, 2:4] = cd / lc[:, None]
    f[:, 4] = ln / lc
    return f


# ---------------------------------------------------------------- the network
# products with k-contiguous operands (the forward MLP layers) run on the
# TMA-fed tensor-core kernel; False keeps the register-staged one everywhere
GEMM_TMA = True


class GraphNet:
    """Device-resident network: FP32 master parameters, bf16 copies, AdamW
    moments, gradient; forward / backward / step through the C ABI."""

    def __init__(self, steps=8, seed=0, params=None, norm=None):
        torch = _torch()
        self.torch = torch
        self.steps = steps
        self.lay = layout(steps=steps)
        self.off, self.n = offsets(self.lay)
        p = init_params(self.lay, seed) if params is None else np.asarray(params, np.float32)
        if p.size != self.n:
            raise L.Op2Error(f"parameter vector of {p.size}, layout needs {self.n}")
        dev = torch.device("cuda")
        self.p = torch.from_numpy(p.copy()).to(dev)
        self.pb = self.p.to(torch.bfloat16)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.t = 0
        # normalisation of the target (q - qinf): mean[4], std[4]
        self.norm = np.array([0, 0, 0, 0, 1, 1, 1, 1], np.float64) if norm is None else \
            np.asarray(norm, np.float64)
        self._ws = {}
        self.launches = 0
        self.gemm_tma = GEMM_TMA

    # -- helpers ------------------------------------------------------------
    @property
    def stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    def _w(self, name, i):
        w0, b0, kin, nout = self.off[(name, i)]
        return self.pb.data_ptr() + 2 * w0, self.p.data_ptr() + 4 * b0, self.g.data_ptr() + \
            4 * w0, self.g.data_ptr() + 4 * b0, kin, nout

    def _gemm(self, M, N, K, A, a_m, a_k, B, b_n, b_k, C, ldc, epi, bias=None, Z=None, R=None,
              ldr=0, split=1):
        # every product goes to the TMA-fed persistent kernel (engine 2: k-
        # contiguous operands as K-major tiles, the others as MN-major tiles)
        # unless gemm_tma is off (engine 0, operands staged through registers)
        engine = 2 if self.gemm_tma else 0
        _call("op2b_gemm_bf16", M, N, K, A, a_m, a_k, B, b_n, b_k, C, ldc, epi, bias, Z, R, ldr,
              split, engine, self.stream)
        self.launches += 1

    def _split_for(self, rows, ntiles):
        ctas = 2 * 148
        s = max(1, min(ctas // max(1, ntiles), rows // 256))
        return s

    def workspace(self, N, E, train):
        key = (N, E, train)
        if key in self._ws:
            return self._ws[key]
        torch = self.torch
        bf, f32 = torch.bfloat16, torch.float32
        w, S = WIDTH, self.steps
        z = lambda *shape, dt=bf: torch.zeros(*shape, dtype=dt, device="cuda")
        nb = S + 1 if train else 1
        ws = dict(N=N, E=E, train=train)
        ws["node_in"] = z(N, NODE_IN)
        ws["edge_in"] = z(E, EDGE_IN)
        ws["CE"] = [z(E, 3 * w) for _ in range(S if train else 1)]
        ws["E_last"] = z(E, w) if train else None
        ws["CN"] = [z(N, 2 * w) for _ in range(nb)]
        R = max(N, E)
        if train:
            # per MLP: Z0, A0, Z1, A1 (enc_node, enc_edge, each step's two, dec)
            ws["act"] = {}
            for name, _layers in self.lay:
                rows = E if name.startswith("edge") or name == "enc_edge" else N
                ws["act"][name] = [z(rows, w) for _ in range(4)]
            ws["out"] = z(N, OUT, dt=f32)
            ws["dOut"] = z(N, OUT)
            ws["dH"] = z(N, w, dt=f32)
            ws["dE"] = z(E, w, dt=f32)
            ws["dyN"] = z(N, w)
            ws["dyE"] = z(E, w)
            ws["dZa"] = z(R, w)
            ws["dZb"] = z(R, w)
            ws["dCat"] = z(max(E * 3 * w, N * 2 * w), dt=f32)
            ws["loss"] = z(1, dt=f32)
        else:
            shared = [z(R, w), z(R, w)]
            ws["act"] = {name: [None, shared[0], None, shared[1]] for name, _ in self.lay}
            ws["out"] = z(N, OUT, dt=f32)
        self._ws[key] = ws
        return ws

    def release(self):
        """Drop every cached workspace (device memory returns to torch's pool)."""
        self._ws = {}

    # -- forward --------------------------------------------------------------
    def _mlp_fwd(self, name, M, X, ldx, out, ldo, resid=None, ldr=0, last=EPI_BIAS_BF16,
                 ws=None):
        Z0, A0, Z1, A1 = ws["act"][name]
        ptr = lambda t: None if t is None else t.data_ptr()
        w = WIDTH
        Wp, bp, _, _, kin, nout = self._w(name, 0)
        self._gemm(M, nout, kin, X, ldx, 1, Wp, kin, 1, A0.data_ptr(), w, EPI_BIAS_SILU_BF16,
                   bias=bp, Z=ptr(Z0))
        Wp, bp, _, _, kin, nout = self._w(name, 1)
        self._gemm(M, nout, kin, A0.data_ptr(), w, 1, Wp, kin, 1, A1.data_ptr(), w,
                   EPI_BIAS_SILU_BF16, bias=bp, Z=ptr(Z1))
        Wp, bp, _, _, kin, nout = self._w(name, 2)
        self._gemm(M, nout, kin, A1.data_ptr(), w, 1, Wp, kin, 1, out, ldo, last, bias=bp,
                   R=resid, ldr=ldr)

    def upload_graph(self, g):
        t = self.torch
        dev = lambda a: t.from_numpy(np.ascontiguousarray(a, np.int32)).to("cuda")
        return dict(N=g["N"], E=g["E"], **{k: dev(g[k]) for k in ("src", "dst", "rev", "off",
                                                                  "idx")})

    def forward(self, dg, node_in, edge_in, train=True, ws=None):
        """node_in (N x 16), edge_in (E x 8): bf16 device tensors (or float,
        converted).  Returns the FP32 output (N x 8) device tensor."""
        torch = self.torch
        N, E = dg["N"], dg["E"]
        ws = ws or self.workspace(N, E, train)
        w, S, st = WIDTH, self.steps, self.stream
        ni = node_in if node_in.dtype == torch.bfloat16 else node_in.to(torch.bfloat16)
        ei = edge_in if edge_in.dtype == torch.bfloat16 else edge_in.to(torch.bfloat16)
        ws["_node_in"], ws["_edge_in"] = ni, ei
        CN0 = ws["CN"][0]
        CE0 = ws["CE"][0]
        self._mlp_fwd("enc_node", N, ni.data_ptr(), NODE_IN, CN0.data_ptr(), 2 * w, ws=ws)
        self._mlp_fwd("enc_edge", E, ei.data_ptr(), EDGE_IN, CE0.data_ptr(), 3 * w, ws=ws)
        src, dst, off, idx = (dg[k].data_ptr() for k in ("src", "dst", "off", "idx"))
        for l in range(S):
            CE = ws["CE"][l if train else 0]
            CN = ws["CN"][l if train else 0]
            _call("op2b_gnn_gather_pair", E, w, src, dst, CN.data_ptr(), 2 * w, CE.data_ptr(),
                  3 * w, w, st)
            if train:
                if l + 1 < S:
                    eo, lde = ws["CE"][l + 1].data_ptr(), 3 * w
                else:
                    eo, lde = ws["E_last"].data_ptr(), w
            else:
                eo, lde = CE.data_ptr(), 3 * w              # in place: same thread reads R
            self._mlp_fwd(f"edge{l}", E, CE.data_ptr(), 3 * w, eo, lde, resid=CE.data_ptr(),
                          ldr=3 * w, ws=ws)
            _call("op2b_gnn_aggregate", N, w, off, idx, eo, lde, CN.data_ptr() + 2 * w, 2 * w,
                  st)
            CNn = ws["CN"][l + 1] if train else CN
            self._mlp_fwd(f"node{l}", N, CN.data_ptr(), 2 * w, CNn.data_ptr(), 2 * w,
                          resid=CN.data_ptr(), ldr=2 * w, ws=ws)
            self.launches += 2
        CNl = ws["CN"][S if train else 0]
        self._mlp_fwd("dec", N, CNl.data_ptr(), 2 * w, ws["out"].data_ptr(), OUT,
                      last=EPI_STORE_F32, ws=ws)
        return ws["out"]

    # -- backward -------------------------------------------------------------
    def _mlp_bwd(self, name, M, dy, ldy, X, ldx, dx=None, lddx=0, ws=None):
        """dy: bf16 gradient of the MLP output (M x n_out, leading dim ldy).
        Accumulates dW, db; writes dX (FP32) when dx is given."""
        Z0, A0, Z1, A1 = ws["act"][name]
        inputs = {0: (X, ldx), 1: (A0.data_ptr(), WIDTH), 2: (A1.data_ptr(), WIDTH)}
        dz = {1: ws["dZa"], 0: ws["dZb"]}
        Zs = {1: Z1, 0: Z0}
        d, ld = dy, ldy
        for i in (2, 1, 0):
            Wp, _bp, gW, gb, kin, nout = self._w(name, i)
            xin, ldxin = inputs[i]
            ntiles = (kin + 127) // 128
            split = self._split_for(M, ntiles)
            # dW[nout][kin] += sum_m d(m, nout) x(m, kin): both operands transposed
            self._gemm(nout, kin, M, d, 1, ld, xin, 1, ldxin, gW, kin, EPI_ATOMIC_F32,
                       split=split)
            _call("op2b_gnn_colsum", M, nout, d, ld, gb, self.stream)
            self.launches += 1
            if i > 0:
                nxt = dz[i - 1].data_ptr()
                self._gemm(M, kin, nout, d, ld, 1, Wp, 1, kin, nxt, WIDTH, EPI_SILU_GRAD_BF16,
                           R=Zs[i - 1].data_ptr(), ldr=WIDTH)
                d, ld = nxt, WIDTH
            elif dx is not None:
                self._gemm(M, kin, nout, d, ld, 1, Wp, 1, kin, dx, lddx, EPI_STORE_F32)

    def backward(self, dg, ws, dOut=None):
        """Backpropagate the gradient in ws['dOut'] (bf16, N x 8) through the
        network of the last forward(train=True); accumulates into self.g."""
        N, E = dg["N"], dg["E"]
        w, S, st = WIDTH, self.steps, self.stream
        dH, dE, dCat = ws["dH"], ws["dE"], ws["dCat"]
        dyN, dyE = ws["dyN"].data_ptr(), ws["dyE"].data_ptr()
        dst, off, idx, rev = (dg[k].data_ptr() for k in ("dst", "off", "idx", "rev"))
        dO = ws["dOut"].data_ptr() if dOut is None else dOut
        self._mlp_bwd("dec", N, dO, OUT, ws["CN"][S].data_ptr(), 2 * w, dx=dH.data_ptr(),
                      lddx=w, ws=ws)
        _call("op2b_gnn_memset", dE.data_ptr(), 0, dE.numel() * 4, st)
        for l in reversed(range(S)):
            _call("op2b_gnn_to_bf16", N, w, dH.data_ptr(), w, dyN, w, st)
            CN = ws["CN"][l]
            self._mlp_bwd(f"node{l}", N, dyN, w, CN.data_ptr(), 2 * w, dx=dCat.data_ptr(),
                          lddx=2 * w, ws=ws)
            _call("op2b_gnn_add_f32", N, w, dH.data_ptr(), dCat.data_ptr(), 2 * w, st)
            _call("op2b_gnn_edge_grad", E, w, dst, dE.data_ptr(), dCat.data_ptr() + 4 * w, 2 * w,
                  dyE, st)
            CE = ws["CE"][l]
            self._mlp_bwd(f"edge{l}", E, dyE, w, CE.data_ptr(), 3 * w, dx=dCat.data_ptr(),
                          lddx=3 * w, ws=ws)
            _call("op2b_gnn_cat_grad", E, N, w, dCat.data_ptr(), 3 * w, dE.data_ptr(), off, idx,
                  rev, dH.data_ptr(), st)
            self.launches += 5
        _call("op2b_gnn_to_bf16", N, w, dH.data_ptr(), w, dyN, w, st)
        self._mlp_bwd("enc_node", N, dyN, w, ws["_node_in"].data_ptr(), NODE_IN, ws=ws)
        _call("op2b_gnn_to_bf16", E, w, dE.data_ptr(), w, dyE, w, st)
        self._mlp_bwd("enc_edge", E, dyE, w, ws["_edge_in"].data_ptr(), EDGE_IN, ws=ws)
        self.launches += 2

    def loss_grad(self, dg, node_in, edge_in, target, ws=None, zero_loss=True):
        """Forward, MSE against target (N x 4 float device tensor, normalised
        units), backward.  Returns the device loss accumulator (1 float): this
        step's loss, or the running sum when zero_loss is False."""
        N = dg["N"]
        ws = ws or self.workspace(N, dg["E"], True)
        out = self.forward(dg, node_in, edge_in, train=True, ws=ws)
        if zero_loss:
            _call("op2b_gnn_memset", ws["loss"].data_ptr(), 0, 4, self.stream)
        _call("op2b_gnn_mse", N, 4, out.data_ptr(), OUT, target.data_ptr(), ws["dOut"].data_ptr(),
              ws["loss"].data_ptr(), 1.0 / (4.0 * N), self.stream)
        self.launches += 1
        self.backward(dg, ws)
        return ws["loss"]

    def step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.t += 1
        lr_t = lr * math.sqrt(1 - beta2 ** self.t) / (1 - beta1 ** self.t)
        _call("op2b_gnn_adam", self.n, self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
              self.v.data_ptr(), self.pb.data_ptr(), lr_t, beta1, beta2, eps, lr * weight_decay,
              self.stream)
        self.launches += 1

    def average_grad(self, group=None):
        """Data-parallel training: the gradient of this rank's minibatch
        replaced by the mean over the ranks of a torch.distributed group --
        an all-reduce on the device with NCCL, through host memory with gloo
        (ranks sharing a GPU).  Each rank's loss is a mean over its own
        minibatch, so the result is the gradient of the mean over all ranks'
        samples."""
        import torch.distributed as dist
        w = dist.get_world_size(group)
        if w == 1:
            return
        if dist.get_backend(group) == "nccl":
            dist.all_reduce(self.g, group=group)
            self.g.div_(w)
        else:
            t = self.g.cpu()
            dist.all_reduce(t, group=group)
            self.g.copy_(t.div_(w))

    def zero_grad(self):
        _call("op2b_gnn_memset", self.g.data_ptr(), 0, self.n * 4, self.stream)

    def grad(self):
        return self.g.cpu().numpy().astype(np.float64)

    def params(self):
        return self.p.cpu().numpy()

    def save(self, path):
        np.savez(path, params=self.params(), norm=self.norm, steps=self.steps)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(steps=int(z["steps"]), params=z["params"], norm=z["norm"])
