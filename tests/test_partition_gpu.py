"""The partitioned single mesh on the GPU (op2b/partition.py): several
partitions in one process on one GPU, each through the OP2 API on libop2b,
halo q moved between them by op2b_dat_pack / op2b_dat_unpack after every
update (no kernel of one partition waits for another's).  Owned q must equal
the single-mesh run's bit for bit (each owned cell adds its edges' fluxes in
the global edge order, the partition-boundary edges being computed by both
sides), maxerr and its global cell exactly, rms to 1e-13 (the rms sums of
the partitions add in another order)."""
import numpy as np
import pytest

from op2b import lib as L
from op2b import mesh as M
from op2b import partition as P
from op2b.airfoil import Airfoil

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("I,J,nparts", [(120, 60, 2), (120, 60, 3), (400, 200, 4)])
def test_partitioned_run_matches_single_mesh(op2, I, J, nparts):
    m = M.channel_bump(I, J, seed=3)
    niter = 20
    ref = Airfoil(m)
    hist_ref = ref.iterate(niter)
    q_ref = ref.fetch()["q"]
    parts = [P.PartAirfoil(p) for p in P.partition(m, nparts)]
    hist = P.run_partitioned(parts, niter, m.ncell)
    q = np.empty_like(q_ref)
    for p in parts:
        q[p.part.cells[:p.part.nowned]] = p.fetch_owned()
    assert np.array_equal(q, q_ref)
    rms, rms_ref = np.array([h[0] for h in hist]), np.array([h[0] for h in hist_ref])
    assert np.max(np.abs(rms / rms_ref - 1)) < 1e-13
    assert [h[1] for h in hist] == [h[1] for h in hist_ref]
    assert [h[2] for h in hist] == [h[2] for h in hist_ref]


def test_pack_and_unpack_rows(op2):
    import torch
    s = L.op_decl_set(1000, "s")
    a = np.arange(4000, dtype=np.float64).reshape(1000, 4)
    d = L.op_decl_dat(s, 4, "double", a, "d")
    rows = np.array([5, 999, 0, 17, 5], np.int32)
    rd = torch.from_numpy(rows).cuda()
    buf = torch.zeros((5, 4), dtype=torch.float64, device="cuda")
    assert L.load().op2b_dat_pack(d, rd.data_ptr(), 5, buf.data_ptr()) == 0
    L.synchronize()
    assert np.array_equal(buf.cpu().numpy(), a[rows])
    assert L.load().op2b_dat_unpack(d, None, 990, 5, buf.data_ptr()) == 0
    back = L.op_fetch_data(d)
    want = a.copy()
    want[990:995] = a[rows]
    assert np.array_equal(back, want)
    # a slice beyond the set is refused before any launch
    assert L.load().op2b_dat_unpack(d, None, 998, 5, buf.data_ptr()) == -1
    assert "outside the set" in L.last_error()
