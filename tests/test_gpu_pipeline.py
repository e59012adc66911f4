"""Host records copied back while later rows are answered: one plain kNN
group on a tile of at least 4M points writing pinned host records runs in
chunks of the point-id range (2 below 8M points, 4 from 8M), each chunk's
records copied back on a copy stream while the next chunk's queries run.
The records, row exceptions and row counts equal those of the same stages
written to device records and to pageable host records (one copy at the
end) bit for bit."""
import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from gpupdal_b200.native import record_columns

pytestmark = pytest.mark.gpu


def _stage_sets():
    return [
        [abi.make_opts(abi.STAGE_EIGENVALUES, knn=16), abi.make_opts(abi.STAGE_NORMAL, knn=16)],
        [abi.make_opts(abi.STAGE_NORMAL, knn=10, always_up=False),
         abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10,
                       feature_mask=abi.FEAT_ALL & ~abi.FEAT_DENSITY)],
    ]


def _sorted_ex(ex):
    return np.sort(ex, order=["stage", "point_id", "code"])


@pytest.mark.parametrize("points,seed,chunks", [(4_500_000, 3, 2), (9_000_000, 4, 4)])
def test_pipelined_host_records_equal_device_records(nbg, points, seed, chunks):
    import torch
    x, y, z = syn.stress(points, seed)
    n = len(x)
    tile = nbg.tile(x, y, z)
    for sts in _stage_sets():
        nd = sum(len(abi.stage_dims(s)) for s in sts)
        rec = 8 * nd
        # device records keep the caller's values on skipped rows; fresh host
        # records read 0 there
        drec = torch.zeros((n, nd), dtype=torch.float64, device="cuda")
        cap = n  # every row's exception fits: no run keeps an order-dependent subset
        ex_d, st_d = nbg.run_columns(tile, sts, record_columns(drec.data_ptr(), sts, rec, 1),
                                     exception_capacity=cap)
        assert len(ex_d) < cap
        hpin = torch.empty((n, nd), dtype=torch.float64).pin_memory()
        ex_p, st_p = nbg.run_columns(tile, sts, record_columns(hpin.data_ptr(), sts, rec, 2),
                                     exception_capacity=cap)
        hpage = np.empty((n, nd), dtype=np.float64)
        ex_h, st_h = nbg.run_columns(tile, sts, record_columns(hpage.ctypes.data, sts, rec, 2),
                                     exception_capacity=cap)
        assert st_p.output_chunks == chunks
        assert st_h.output_chunks == 0 and st_d.output_chunks == 0
        want = drec.cpu().numpy()
        assert np.array_equal(hpin.numpy(), want, equal_nan=True)
        assert np.array_equal(hpage, want, equal_nan=True)
        assert np.array_equal(_sorted_ex(ex_p), _sorted_ex(ex_d))
        assert np.array_equal(_sorted_ex(ex_h), _sorted_ex(ex_d))
        for f in ("tie_rows", "deferred_rows", "replay_rows", "resolved_rows"):
            assert getattr(st_p, f) == getattr(st_d, f), f
        assert st_p.tie_rows > 0
