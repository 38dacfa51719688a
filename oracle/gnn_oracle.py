"""CPU oracle of the learned warm start's graph network -- test infrastructure.

Only tests, the smoke check and the benchmark's baseline leg use this module,
as the checker of the GPU kernels (include/op2b_gnn.h, op2b/gnn.py); the
product never imports it.  The reference has no learned component (its
Airfoil always starts from freestream, apps/c/airfoil/airfoil_plain/dp/
airfoil.cpp:204-210), so this restatement pins the network's own definition:

  encoder   h0 = MLP_n(node_in), e0 = MLP_e(edge_in)
  step l    cat_e = [e_l, h_l[src], h_l[dst]]
            e_{l+1} = e_l + MLP_edge_l(cat_e)
            agg[n] = sum over edges k with dst[k] = n of e_{l+1}[k]
            h_{l+1} = h_l + MLP_node_l([h_l, agg])
  decoder   out = MLP_d(h_L)   (no activation on the last layer)

Each MLP is Linear - SiLU - Linear - SiLU - Linear.  Arithmetic is float64.
With ``rnd=True`` every value the GPU path stores in bf16 (weights, inputs,
pre-activations, activations, layer outputs, aggregates, the bf16 copies of
gradients fed to the tensor cores) is rounded to bf16 at the same point, so
the oracle and the GPU differ only by FP32-vs-FP64 accumulation.
Gradients are checked here against central finite differences.
"""
from __future__ import annotations

import numpy as np

WIDTH = 128


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64).reshape(a.shape)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def layout(node_in=16, edge_in=8, width=WIDTH, steps=8, out=8):
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
    """Flat offsets: {(mlp, layer): (w_off, b_off, k_in, n_out)}, total size."""
    off, o = {}, 0
    for name, layers in lay:
        for i, (kin, nout) in enumerate(layers):
            off[(name, i)] = (o, o + kin * nout, kin, nout)
            o += kin * nout + nout
    return off, o


class Net:
    def __init__(self, params, lay, rnd=True):
        self.lay = lay
        self.off, n = offsets(lay)
        assert params.size == n
        self.p = np.asarray(params, np.float64)
        self.rnd = rnd

    def r(self, x):
        return bf16(x) if self.rnd else x

    def W(self, name, i):
        w0, b0, kin, nout = self.off[(name, i)]
        return self.r(self.p[w0:w0 + kin * nout].reshape(nout, kin)), self.p[b0:b0 + nout]

    # -- MLP pieces -------------------------------------------------------
    def mlp_fwd(self, name, x, resid=None, last="bf16"):
        c = {"x": x}
        h = x
        for i in range(2):
            W, b = self.W(name, i)
            z = h @ W.T + b
            c[f"z{i}"] = self.r(z)
            h = self.r(silu(z))
            c[f"a{i}"] = h
        W, b = self.W(name, 2)
        y = h @ W.T + b
        if resid is not None:
            y = y + resid
        return (self.r(y) if last == "bf16" else y), c

    def mlp_bwd(self, name, dy, c, g, need_dx=True):
        """dy: bf16-valued gradient of the MLP output; accumulates into g."""
        inp = {2: c["a1"], 1: c["a0"], 0: c["x"]}
        d = dy
        dx = None
        for i in (2, 1, 0):
            W, _ = self.W(name, i)
            w0, b0, kin, nout = self.off[(name, i)]
            g[w0:w0 + kin * nout] += (d.T @ inp[i]).ravel()
            g[b0:b0 + nout] += d.sum(axis=0)
            if i > 0:
                d = self.r((d @ W) * silu_grad(c[f"z{i - 1}"]))
            elif need_dx:
                dx = d @ W
        return dx

    # -- the network ------------------------------------------------------
    def forward(self, graph, node_in, edge_in, steps):
        src, dst, off, idx = graph["src"], graph["dst"], graph["off"], graph["idx"]
        N = node_in.shape[0]
        w = WIDTH
        caches = {}
        h, caches["enc_node"] = self.mlp_fwd("enc_node", self.r(node_in))
        e, caches["enc_edge"] = self.mlp_fwd("enc_edge", self.r(edge_in))
        for l in range(steps):
            cat = np.concatenate([e, h[src], h[dst]], axis=1)
            e_new, caches[f"edge{l}"] = self.mlp_fwd(f"edge{l}", cat, resid=e)
            agg = np.zeros((N, w))
            for n in range(N):
                ks = idx[off[n]:off[n + 1]]
                if ks.size:
                    agg[n] = e_new[ks].sum(axis=0)
            agg = self.r(agg)
            h_new, caches[f"node{l}"] = self.mlp_fwd(f"node{l}", np.concatenate([h, agg], 1),
                                                     resid=h)
            e, h = e_new, h_new
        out, caches["dec"] = self.mlp_fwd("dec", h, last="f32")
        return out, caches

    def backward(self, graph, caches, dy_out, steps):
        src, dst, off, idx, rev = (graph[k] for k in ("src", "dst", "off", "idx", "rev"))
        N = caches["dec"]["x"].shape[0]
        w = WIDTH
        g = np.zeros_like(self.p)
        dH = self.mlp_bwd("dec", dy_out, caches["dec"], g)
        dE = np.zeros((src.size, w))
        for l in reversed(range(steps)):
            dCN = self.mlp_bwd(f"node{l}", self.r(dH), caches[f"node{l}"], g)
            dH = dH + dCN[:, :w]
            dE = dE + dCN[dst, w:]
            dCE = self.mlp_bwd(f"edge{l}", self.r(dE), caches[f"edge{l}"], g)
            dE = dE + dCE[:, :w]
            add = np.zeros((N, w))
            for n in range(N):
                ks = idx[off[n]:off[n + 1]]
                if ks.size:
                    add[n] = dCE[ks, 2 * w:].sum(axis=0) + dCE[rev[ks], w:2 * w].sum(axis=0)
            dH = dH + add
        self.mlp_bwd("enc_node", self.r(dH), caches["enc_node"], g, need_dx=False)
        self.mlp_bwd("enc_edge", self.r(dE), caches["enc_edge"], g, need_dx=False)
        return g


def mse_grad(out, target, scale, rnd=True):
    """Loss scale * sum (out[:, :4] - target)^2 and its bf16 gradient (width of out)."""
    d = out[:, :target.shape[1]] - target
    dy = np.zeros_like(out)
    dy[:, :target.shape[1]] = 2.0 * scale * d
    return scale * float((d * d).sum()), (bf16(dy) if rnd else dy)


def loss_and_grad(params, lay, graph, node_in, edge_in, target, steps, rnd=True):
    net = Net(params, lay, rnd)
    out, caches = net.forward(graph, node_in, edge_in, steps)
    scale = 1.0 / target.size
    loss, dy = mse_grad(out, target, scale, rnd)
    return loss, net.backward(graph, caches, dy, steps), out


def finite_difference(params, lay, graph, node_in, edge_in, target, steps, which, h=1e-6):
    """Central differences of the (unrounded) loss at parameter indices `which`."""
    fd = []
    for i in which:
        p = params.copy()
        p[i] += h
        lp = loss_and_grad(p, lay, graph, node_in, edge_in, target, steps, rnd=False)[0]
        p[i] -= 2 * h
        lm = loss_and_grad(p, lay, graph, node_in, edge_in, target, steps, rnd=False)[0]
        fd.append((lp - lm) / (2 * h))
    return np.array(fd)
