"""GPU parity of the learned warm start's kernels (include/op2b_gnn.h).

* op2b_gemm_bf16 on the tensor cores against float64 products of the same
  bf16 operands: relative error <= 2e-5 of the output's scale (FP32
  accumulation over K <= 512), for every epilogue, transposed operands,
  split-K, ragged M/N/K; the CUDA-core engine agrees too.
* The graph kernels (gather, aggregate, gradient combines, column sums, MSE,
  AdamW) against numpy: bit-exact where the arithmetic is a copy, 1e-6
  relative where FP32 sums are reordered.
* The whole network, forward and backward, against the CPU oracle with bf16
  rounding emulated at the same points: output within 2e-2 of its scale and
  every parameter tensor's gradient within 5e-2 relative (L2) -- the gap
  left by FP32-vs-FP64 accumulation flipping bf16 roundings.
"""
import numpy as np
import pytest

from op2b import gnn as G
from op2b import lib as L
from op2b import mesh as M
from oracle import gnn_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _bf(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16)


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _gemm(M_, N, K, A, a_m, a_k, B, b_n, b_k, C, ldc, epi, bias=None, Z=None, R=None, ldr=0,
          split=1, engine=0):
    ptr = lambda t: None if t is None else t.data_ptr()
    rc = G._lib().op2b_gemm_bf16(M_, N, K, A.data_ptr(), a_m, a_k, B.data_ptr(), b_n, b_k,
                                 C.data_ptr(), ldc, epi, ptr(bias), ptr(Z), ptr(R), ldr, split,
                                 engine, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, L.last_error()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


SHAPES = [(128, 128, 64), (300, 128, 384), (1000, 256, 136), (77, 8, 128), (515, 16, 8),
          (4099, 384, 256)]


@pytest.mark.parametrize("shape", SHAPES)
def test_gemm_store_f32_matches_float64(op2, shape):
    M_, N, K = shape
    rng = np.random.default_rng(M_ + N + K)
    a = _bf(rng.standard_normal((M_, K)))
    b = _bf(rng.standard_normal((N, K)))
    ref = _np(a) @ _np(b).T
    A, B = a.cuda(), b.cuda()
    C = torch.zeros(M_, N, device="cuda")
    _gemm(M_, N, K, A, K, 1, B, K, 1, C, N, G.EPI_STORE_F32)
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0
    assert _rel(_np(C), ref) < 2e-5
    C2 = torch.zeros(M_, N, device="cuda")
    _gemm(M_, N, K, A, K, 1, B, K, 1, C2, N, G.EPI_STORE_F32, engine=1)
    assert _rel(_np(C2), ref) < 2e-5


@pytest.mark.parametrize("split", [1, 3, 37])
def test_gemm_transposed_operands_split_k(op2, split):
    # dW[n_out][k_in] = sum_m dY[m][n_out] X[m][k_in]: both operands transposed
    rng = np.random.default_rng(split)
    Mr, nout, kin = 5003, 128, 384
    dy = _bf(rng.standard_normal((Mr, nout)))
    x = _bf(rng.standard_normal((Mr, kin)))
    ref = _np(dy).T @ _np(x)
    C = torch.zeros(nout, kin, device="cuda")
    _gemm(nout, kin, Mr, dy.cuda(), 1, nout, x.cuda(), 1, kin, C, kin, G.EPI_ATOMIC_F32,
          split=split)
    assert _rel(_np(C), ref) < 2e-5
    # dX = dY W with W [n_out][k_in]: B transposed
    w = _bf(rng.standard_normal((nout, kin)))
    C = torch.zeros(Mr, kin, device="cuda")
    _gemm(Mr, kin, nout, dy.cuda(), nout, 1, w.cuda(), 1, kin, C, kin, G.EPI_STORE_F32)
    assert _rel(_np(C), _np(dy) @ _np(w)) < 2e-5
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0


def test_gemm_epilogues(op2):
    rng = np.random.default_rng(7)
    Mr, N, K = 700, 128, 256
    a = _bf(rng.standard_normal((Mr, K)) * 0.2)
    b = _bf(rng.standard_normal((N, K)) * 0.2)
    bias = torch.from_numpy(rng.standard_normal(N).astype(np.float32))
    acc = _np(a) @ _np(b).T
    A, B, bc = a.cuda(), b.cuda(), bias.cuda()
    z = acc + bias.numpy()
    # bias + SiLU, with the pre-activation
    C = torch.zeros(Mr, N, dtype=torch.bfloat16, device="cuda")
    Z = torch.zeros_like(C)
    _gemm(Mr, N, K, A, K, 1, B, K, 1, C, N, G.EPI_BIAS_SILU_BF16, bias=bc, Z=Z)
    assert np.abs(_np(Z) - z).max() <= 2 ** -7 * np.abs(z).max()
    assert np.abs(_np(C) - O.silu(z)).max() <= 2 ** -7 * np.abs(O.silu(z)).max()
    # bias + residual into a strided destination
    R = _bf(rng.standard_normal((Mr, 3 * N))).cuda()
    C = R.clone()
    _gemm(Mr, N, K, A, K, 1, B, K, 1, C, 3 * N, G.EPI_BIAS_BF16, bias=bc, R=R, ldr=3 * N)
    want = z + _np(R)[:, :N]
    got = _np(C)
    assert np.abs(got[:, :N] - want).max() <= 2 ** -7 * np.abs(want).max()
    assert np.array_equal(got[:, N:], _np(R)[:, N:])            # untouched columns
    # product times silu'(R)
    zz = _bf(rng.standard_normal((Mr, N)))
    C = torch.zeros(Mr, N, dtype=torch.bfloat16, device="cuda")
    _gemm(Mr, N, K, A, K, 1, B, K, 1, C, N, G.EPI_SILU_GRAD_BF16, R=zz.cuda(), ldr=N)
    want = acc * O.silu_grad(_np(zz))
    assert np.abs(_np(C) - want).max() <= 2 ** -7 * np.abs(want).max()
    # bias into FP32 (the decoder's last layer)
    C = torch.zeros(Mr, N, device="cuda")
    _gemm(Mr, N, K, A, K, 1, B, K, 1, C, N, G.EPI_STORE_F32, bias=bc)
    assert _rel(_np(C), z) < 2e-5
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0


TMA_SHAPES = [(128, 128, 64), (300, 128, 384), (1000, 256, 136), (77, 8, 128), (515, 16, 8),
              (4099, 384, 256), (20000, 128, 384)]


@pytest.mark.parametrize("shape", TMA_SHAPES)
def test_gemm_tma_engine_matches_float64(op2, shape):
    """engine 2: the operand tiles arrive by TMA (tensor maps, 128-byte
    swizzle, zero fill past the matrix) into a three-stage mbarrier ring.
    Against float64 products (2e-5 of the scale) and bit for bit against the
    register-staged engine 0 (the same MMAs in the same K order)."""
    M_, N, K = shape
    rng = np.random.default_rng(M_ * 3 + N + K)
    a = _bf(rng.standard_normal((M_, K)))
    b = _bf(rng.standard_normal((N, K)))
    ref = _np(a) @ _np(b).T
    A, B = a.cuda(), b.cuda()
    C = torch.zeros(M_, N, device="cuda")
    _gemm(M_, N, K, A, K, 1, B, K, 1, C, N, G.EPI_STORE_F32, engine=2)
    C0 = torch.zeros(M_, N, device="cuda")
    _gemm(M_, N, K, A, K, 1, B, K, 1, C0, N, G.EPI_STORE_F32, engine=0)
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0
    assert _rel(_np(C), ref) < 2e-5
    assert torch.equal(C, C0)


def test_gemm_tma_engine_epilogues_and_split_k(op2):
    rng = np.random.default_rng(11)
    Mr, N, K = 2000, 128, 384
    a = _bf(rng.standard_normal((Mr, K)) * 0.2)
    b = _bf(rng.standard_normal((N, K)) * 0.2)
    bias = torch.from_numpy(rng.standard_normal(N).astype(np.float32)).cuda()
    A, B = a.cuda(), b.cuda()
    outs = []
    for engine in (0, 2):
        C = torch.zeros(Mr, N, dtype=torch.bfloat16, device="cuda")
        Z = torch.zeros_like(C)
        _gemm(Mr, N, K, A, K, 1, B, K, 1, C, N, G.EPI_BIAS_SILU_BF16, bias=bias, Z=Z,
              engine=engine)
        S = torch.zeros(Mr, N, device="cuda")
        _gemm(Mr, N, K, A, K, 1, B, K, 1, S, N, G.EPI_ATOMIC_F32, split=3, engine=engine)
        outs.append((C, Z, S))
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0
    (c0, z0, s0), (c2, z2, s2) = outs
    assert torch.equal(c0, c2) and torch.equal(z0, z2)
    ref = _np(a) @ _np(b).T
    assert _rel(_np(s2), ref) < 2e-5


@pytest.mark.parametrize("shape", [(300, 128, 384), (20000, 128, 8), (40000, 256, 136),
                                   (300000, 128, 384), (1000, 136, 64), (5000, 8, 128),
                                   (777, 40, 72)])
def test_gemm_persistent_kernel_matches_per_tile_kernel(op2, shape):
    """engine 2's persistent warp-specialised kernel (one CTA per SM walking
    the tiles, TMEM accumulator double-buffered so a tile's epilogue overlaps
    the next tile's loads and MMAs; 8 or 16 epilogue warps, rows stored
    through shared memory or by each lane) against the one-tile-per-CTA TMA
    kernel (option gemm_persistent 0): bit for bit, FP32 store and bias+SiLU
    with the pre-activation, and split-K to rounding; N not a multiple of the
    tile or of a warp's columns included."""
    M_, N, K = shape
    rng = np.random.default_rng(M_ + 7 * N + K)
    a = _bf(rng.standard_normal((M_, K)) * 0.2)
    b = _bf(rng.standard_normal((N, K)) * 0.2)
    bias = torch.from_numpy(rng.standard_normal(N).astype(np.float32)).cuda()
    A, B = a.cuda(), b.cuda()
    outs = []
    for persistent, rows in ((1, 0), (2, 1), (2, 0), (0, 0)):
        op2.set_option("gemm_persistent", persistent)
        op2.set_option("gemm_rows", rows)
        C = torch.zeros(M_, N, device="cuda")
        _gemm(M_, N, K, A, K, 1, B, K, 1, C, N, G.EPI_STORE_F32, engine=2)
        H = torch.zeros(M_, N, dtype=torch.bfloat16, device="cuda")
        Z = torch.zeros_like(H)
        _gemm(M_, N, K, A, K, 1, B, K, 1, H, N, G.EPI_BIAS_SILU_BF16, bias=bias, Z=Z, engine=2)
        S = torch.zeros(M_, N, device="cuda")
        _gemm(M_, N, K, A, K, 1, B, K, 1, S, N, G.EPI_ATOMIC_F32, split=2, engine=2)
        outs.append((C, H, Z, S))
    op2.set_option("gemm_persistent", 2)
    op2.set_option("gemm_rows", 1)
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0
    (c0, h0, z0, s0) = outs[-1]
    for c1, h1, z1, s1 in outs[:-1]:
        assert torch.equal(c1, c0) and torch.equal(h1, h0) and torch.equal(z1, z0)
        assert _rel(_np(s1), _np(c1)) < 1e-6
    if M_ <= 40000:
        assert _rel(_np(c1), _np(a) @ _np(b).T) < 2e-5


def test_gemm_tma_engine_refuses_transposed_operands_one_tile_per_cta(op2):
    op2.set_option("gemm_persistent", 0)
    A = torch.zeros(64, 128, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(128, 128, device="cuda")
    rc = G._lib().op2b_gemm_bf16(128, 128, 64, A.data_ptr(), 1, 128, A.data_ptr(), 1, 128,
                                 C.data_ptr(), 128, G.EPI_STORE_F32, None, None, None, 0, 1, 2,
                                 torch.cuda.current_stream().cuda_stream)
    op2.set_option("gemm_persistent", 2)
    assert rc == -1 and "k-contiguous" in L.last_error()


@pytest.mark.parametrize("layout", ["a_mn", "b_mn", "both_mn"])
@pytest.mark.parametrize("shape", [(128, 128, 64), (304, 136, 520), (128, 384, 40000),
                                   (8, 128, 20000), (20000, 256, 128)])
def test_gemm_persistent_mn_major_operands(op2, shape, layout):
    """Transposed operands on engine 2: the persistent kernel loads them by
    TMA as MN-major tiles (two 64 x 64 boxes, 128-byte swizzle) and the MMAs
    read them through MN-major descriptors.  Against engine 0 (which
    transposes them in registers into K-major tiles) and float64."""
    M_, N, K = shape
    rng = np.random.default_rng(M_ + 3 * N + 5 * K)
    a = _bf(rng.standard_normal((M_, K)) * 0.2)
    b = _bf(rng.standard_normal((N, K)) * 0.2)
    ref = _np(a) @ _np(b).T
    if layout in ("a_mn", "both_mn"):
        A, a_m, a_k = a.t().contiguous().cuda(), 1, M_   # stored K x M
    else:
        A, a_m, a_k = a.cuda(), K, 1
    if layout in ("b_mn", "both_mn"):
        B, b_n, b_k = b.t().contiguous().cuda(), 1, N    # stored K x N
    else:
        B, b_n, b_k = b.cuda(), K, 1
    outs = []
    for engine in (2, 0):
        C = torch.zeros(M_, N, device="cuda")
        _gemm(M_, N, K, A, a_m, a_k, B, b_n, b_k, C, N, G.EPI_STORE_F32, engine=engine)
        S = torch.zeros(M_, N, device="cuda")
        _gemm(M_, N, K, A, a_m, a_k, B, b_n, b_k, S, N, G.EPI_ATOMIC_F32, split=3, engine=engine)
        outs.append((C, S))
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0
    (c2, s2), (c0, s0) = outs
    tol = 2e-5 if K <= 1024 else 2e-4     # FP32 accumulation over K terms
    assert _rel(_np(c2), ref) < tol
    assert _rel(_np(s2), ref) < tol
    assert _rel(_np(c2), _np(c0)) < 1e-6


def test_gemm_rejects_bad_shapes(op2):
    A = torch.zeros(64, 12, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(64, 8, device="cuda")
    rc = G._lib().op2b_gemm_bf16(64, 8, 12, A.data_ptr(), 12, 1, A.data_ptr(), 12, 1,
                                 C.data_ptr(), 8, 0, None, None, None, 0, 1, 0, None)
    assert rc == -1 and "multiples of 8" in L.last_error()
    rc = G._lib().op2b_gemm_bf16(64, 8, 8, A.data_ptr(), 12, 1, A.data_ptr(), 12, 1,
                                 C.data_ptr(), 8, 2, None, None, None, 0, 4, 0, None)
    assert rc == -1


def _graph(I=10, J=5, seed=3):
    m = M.channel_bump(I, J, seed=seed, bump=0.07)
    g = G.cell_graph(m)
    return m, g


def test_graph_kernels_match_numpy(op2):
    m, g = _graph(24, 12)
    net = G.GraphNet(steps=1)
    dg = net.upload_graph(g)
    N, E, D = g["N"], g["E"], 128
    rng = np.random.default_rng(1)
    st = torch.cuda.current_stream().cuda_stream
    h = _bf(rng.standard_normal((N, 2 * D)))
    cat = torch.zeros(E, 3 * D, dtype=torch.bfloat16, device="cuda")
    G._call("op2b_gnn_gather_pair", E, D, dg["src"].data_ptr(), dg["dst"].data_ptr(),
            h.cuda().data_ptr(), 2 * D, cat.data_ptr(), 3 * D, D, st)
    hn = _np(h)
    assert np.array_equal(_np(cat)[:, D:2 * D], hn[g["src"], :D])
    assert np.array_equal(_np(cat)[:, 2 * D:], hn[g["dst"], :D])
    e = _bf(rng.standard_normal((E, 3 * D)))
    out = torch.zeros(N, 2 * D, dtype=torch.bfloat16, device="cuda")
    G._call("op2b_gnn_aggregate", N, D, dg["off"].data_ptr(), dg["idx"].data_ptr(),
            e.cuda().data_ptr(), 3 * D, out.data_ptr() + 2 * D, 2 * D, st)
    want = np.zeros((N, D))
    np.add.at(want, g["dst"], _np(e)[:, :D])
    assert np.abs(_np(out)[:, D:] - want).max() <= 2 ** -7 * np.abs(want).max()
    # cat backward
    dcat = torch.from_numpy(rng.standard_normal((E, 3 * D)).astype(np.float32)).cuda()
    dE = torch.from_numpy(rng.standard_normal((E, D)).astype(np.float32)).cuda()
    dH = torch.from_numpy(rng.standard_normal((N, D)).astype(np.float32)).cuda()
    dE0, dH0, dc = dE.cpu().numpy().astype(np.float64), dH.cpu().numpy().astype(np.float64), \
        dcat.cpu().numpy().astype(np.float64)
    G._call("op2b_gnn_cat_grad", E, N, D, dcat.data_ptr(), 3 * D, dE.data_ptr(),
            dg["off"].data_ptr(), dg["idx"].data_ptr(), dg["rev"].data_ptr(), dH.data_ptr(), st)
    wantE = dE0 + dc[:, :D]
    wantH = dH0.copy()
    np.add.at(wantH, g["dst"], dc[:, 2 * D:])
    np.add.at(wantH, g["src"], dc[:, D:2 * D])
    assert _rel(dE.cpu().numpy(), wantE) < 1e-6
    assert _rel(dH.cpu().numpy(), wantH) < 1e-6
    # column sums
    dz = _bf(rng.standard_normal((E, D)))
    db = torch.zeros(D, device="cuda")
    G._call("op2b_gnn_colsum", E, D, dz.cuda().data_ptr(), D, db.data_ptr(), st)
    assert _rel(db.cpu().numpy(), _np(dz).sum(0)) < 1e-5


def test_adam_step_matches_formula(op2):
    net = G.GraphNet(steps=1, seed=2)
    rng = np.random.default_rng(0)
    g = rng.standard_normal(net.n).astype(np.float32)
    p0 = net.params().astype(np.float64)
    net.g.copy_(torch.from_numpy(g))
    net.step(1e-3, weight_decay=0.01)
    m = 0.1 * g
    v = 0.001 * g.astype(np.float64) ** 2
    lr_t = 1e-3 * np.sqrt(1 - 0.999) / (1 - 0.9)
    want = p0 * (1 - 1e-5) - lr_t * m / (np.sqrt(v) + 1e-8)
    assert np.abs(net.params() - want).max() < 1e-6
    assert float(net.g.abs().max()) == 0.0
    assert torch.equal(net.pb, net.p.to(torch.bfloat16))


@pytest.mark.parametrize("steps", [2, 8])
def test_forward_backward_match_cpu_oracle(op2, steps):
    m, g = _graph(10, 5)
    ni = G.node_features(m, 0.55, 3.0, 0.07)
    ei = G.edge_features(m, g)
    net = G.GraphNet(steps=steps, seed=5)
    net.p.copy_(torch.from_numpy(G.init_params(net.lay, 5, resid_scale=0.5)))
    net.pb.copy_(net.p.to(torch.bfloat16))
    rng = np.random.default_rng(2)
    target = rng.standard_normal((m.ncell, 4)).astype(np.float32)
    dg = net.upload_graph(g)
    loss = net.loss_grad(dg, torch.from_numpy(ni).cuda(), torch.from_numpy(ei).cuda(),
                         torch.from_numpy(target).cuda())
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0
    ws = net.workspace(g["N"], g["E"], True)
    out_gpu = ws["out"].cpu().numpy().astype(np.float64)
    p = net.params().astype(np.float64)
    lref, gref, out_ref = O.loss_and_grad(p, O.layout(steps=steps), g, ni.astype(np.float64),
                                          ei.astype(np.float64), target.astype(np.float64),
                                          steps, rnd=True)
    assert np.abs(out_gpu[:, :4] - out_ref[:, :4]).max() <= 2e-2 * np.abs(out_ref[:, :4]).max()
    assert abs(float(loss.item()) / lref - 1) < 2e-2
    ggpu = net.grad()
    off, _ = O.offsets(O.layout(steps=steps))
    worst = 0.0
    for (name, i), (w0, b0, kin, nout) in off.items():
        for lo, hi in ((w0, w0 + kin * nout), (b0, b0 + nout)):
            ref = gref[lo:hi]
            if np.linalg.norm(ref) == 0:
                assert np.linalg.norm(ggpu[lo:hi]) == 0
                continue
            err = np.linalg.norm(ggpu[lo:hi] - ref) / np.linalg.norm(ref)
            worst = max(worst, err)
            assert err < 5e-2, (name, i, lo == b0, err)
    print("worst relative gradient error", worst)
