"""The partitioned single mesh (op2b/partition.py) on the host: partition
invariants, and a world-size-2 gloo run in which each rank iterates its
partition with the oracle's restated loops (the CPU stand-in for its GPU)
and exchanges halo q with the other rank after every update, as the GPU path
does.  Owned q must equal the unpartitioned oracle run bit for bit: every
owned cell adds its edges' fluxes in the global edge order."""
import os
import socket

import numpy as np
import pytest

from op2b import mesh as M
from op2b import partition as P


@pytest.mark.parametrize("nparts", [1, 2, 3, 4, 7])
def test_partition_invariants(nparts):
    m = M.channel_bump(60, 30, seed=4)
    parts = P.partition(m, nparts)
    owned = np.concatenate([p.cells[:p.nowned] for p in parts])
    assert np.array_equal(np.sort(owned), np.arange(m.ncell))      # each cell owned once
    edge_count = np.zeros(m.nedge, int)
    for p in parts:
        edge_count[p.edges] += 1
        lm = p.mesh
        # local maps point at the same cells, nodes and edges as the global ones
        assert np.array_equal(p.cells[lm.ecell], m.ecell[p.edges])
        assert np.array_equal(p.nodes[lm.edge], m.edge[p.edges])
        assert np.array_equal(p.nodes[lm.cell], m.cell[p.cells])
        assert np.array_equal(p.cells[lm.becell], m.becell[p.bedges])
        assert np.all(lm.becell < p.nowned)                    # boundary edges of owned cells
        assert np.all((lm.ecell < p.nowned).any(axis=1))        # every edge touches an owned cell
        assert np.all(np.diff(p.edges) > 0) and np.all(np.diff(p.cells[:p.nowned]) > 0)
        # the halo is grouped by owner, one contiguous import slice each
        nh = sum(n for _, n in p.imports.values())
        assert nh == p.nhalo
        for r, (first, n) in p.imports.items():
            g = p.cells[first:first + n]
            src = parts[r]
            assert np.array_equal(src.cells[src.exports[p.rank]], g)
            assert np.all(src.exports[p.rank] < src.nowned)
    cross = (parts[0].nparts > 1) and np.any(edge_count == 2)
    assert np.all((edge_count >= 1) & (edge_count <= 2)) and (cross or nparts == 1)
    bcount = np.zeros(m.nbedge, int)
    for p in parts:
        bcount[p.bedges] += 1
    assert np.all(bcount == 1)


def test_rcb_is_balanced():
    rng = np.random.default_rng(1)
    pts = rng.random((10007, 2))
    for k in (2, 3, 5, 8):
        part = P.rcb_partition(pts, k)
        sizes = np.bincount(part, minlength=k)
        assert sizes.max() - sizes.min() <= k


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, niter, q):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = M.channel_bump(48, 24, seed=9)
        c = M.airfoil_constants()
        part = P.partition(m, world)[rank]
        lm = part.mesh
        st = O.State(lm.ncell, c["qinf"])
        for _ in range(niter):
            O.loop("save_soln", lm, c, st)
            for _k in range(2):
                for name in ("adt_calc", "res_calc", "bres_calc", "update"):
                    O.loop(name, lm, c, st)
                # halo exchange of q (the halo rows' own update is overwritten)
                ops = [dist.P2POp(dist.isend, torch.from_numpy(
                    np.ascontiguousarray(st.q[rows])), r) for r, rows in part.exports.items()]
                bufs = {r: torch.empty((n, 4), dtype=torch.float64)
                        for r, (_, n) in part.imports.items()}
                ops += [dist.P2POp(dist.irecv, bufs[r], r) for r in part.imports]
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
                for r, (first, n) in part.imports.items():
                    st.q[first:first + n] = bufs[r].numpy()
        q.put((rank, part.cells[:part.nowned], st.q[:part.nowned].copy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_partitioned_run_is_bit_exact():
    import torch.multiprocessing as mp
    from oracle import oracle as O
    niter = 15
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, niter, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m = M.channel_bump(48, 24, seed=9)
    st, *_ = O.airfoil_run(m, M.airfoil_constants(), niter)
    seen = np.zeros(m.ncell, bool)
    for rank, cells, qo in got:
        assert np.array_equal(qo, st.q[cells]), f"rank {rank}: owned q differs"
        seen[cells] = True
    assert seen.all()
