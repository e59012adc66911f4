"""The no-allocation entry point (nbg_stage_noalloc), through the C ABI.

Callers that cannot allocate device memory (inside another framework's
allocator, real-time loops, restricted plug-in callbacks) use this entry
point: its working memory is a fixed device array inside the library.  This
file runs last so that a failure here leaves every other test already run.

Checked on two calls in a row: every row the entry point answers equals the
regular nbg_run output (within the 1e-5 bar of the parity tests; in fact
identical, the same kernels run), the rows it hands back are exactly the ones
the regular path sends to its exact KD fallback, their outputs are untouched,
and a tile above the size limit is refused with a message.
"""
import ctypes

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _call(lib, dx, dy, dz, n, opts, out, unresolved, exc, cap):
    import torch
    cols = abi.Columns()
    cols.base = out.data_ptr()
    cols.point_stride = 8
    cols.ndims = out.shape[0]
    cols.on_device = 1
    for d in range(out.shape[0]):
        cols.offset[d] = d * n * 8
    sc = (ctypes.c_double * 3)(0.01, 0.01, 0.01)
    of = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    nu = ctypes.c_uint32(0)
    ne = ctypes.c_uint32(0)
    msg = ctypes.create_string_buffer(256)
    rc = lib.nbg_stage_noalloc(dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), n, sc, of,
                               ctypes.byref(opts), ctypes.byref(cols), None, None,
                               unresolved.data_ptr(), ctypes.byref(nu), exc.data_ptr(), cap,
                               ctypes.byref(ne), None, msg, 256)
    torch.cuda.synchronize()
    return rc, nu.value, ne.value, msg.value.decode()


def test_noalloc_matches_nbg_run_on_two_calls(lib_path):
    import torch
    from gpupdal_b200.native import Context
    lib = abi.load_library()
    x, y, z = syn.terrain(250_000, 0)
    n = len(x)
    assert n <= abi.NOALLOC_MAX_POINTS
    dx, dy, dz = (torch.from_numpy(v).cuda() for v in (x, y, z))
    opts = abi.make_opts(abi.STAGE_NORMAL, knn=8, always_up=True)
    ctx = Context(0)
    tile = ctx.tile(dx, dy, dz)
    want, ex, stats = ctx.run(tile, [opts], device_out=True)
    want = want[0].cpu().numpy()
    exact_rows = int(stats.tie_rows + stats.deferred_rows)
    cap = 4096
    for call in range(2):
        out = torch.full((4, n), float("nan"), dtype=torch.float64, device="cuda")
        unresolved = torch.zeros(n, dtype=torch.int32, device="cuda")
        exc = torch.zeros(cap * 2, dtype=torch.int32, device="cuda")
        rc, nu, ne, msg = _call(lib, dx, dy, dz, n, opts, out, unresolved, exc, cap)
        assert rc == abi.NBG_OK, msg
        assert nu == exact_rows, f"call {call}: {nu} unresolved rows, nbg_run sent {exact_rows}"
        assert ne == len(ex)
        got = out.cpu().numpy()
        ids = unresolved[:nu].cpu().numpy().astype(np.int64)
        keep = np.ones(n, bool)
        keep[ids] = False
        keep[ex["point_id"].astype(np.int64)] = False
        assert np.all(np.abs(got[:, keep] - want[:, keep]) <= 1e-5), f"call {call}: outputs differ"
        assert np.isnan(got[:, ids]).all(), f"call {call}: unresolved rows were written"


def test_noalloc_refuses_tiles_above_the_limit(lib_path):
    import torch
    lib = abi.load_library()
    n = abi.NOALLOC_MAX_POINTS + 1
    dx = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros((4, 8), dtype=torch.float64, device="cuda")
    unresolved = torch.zeros(8, dtype=torch.int32, device="cuda")
    exc = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc, nu, ne, msg = _call(lib, dx, dx, dx, n, abi.make_opts(abi.STAGE_NORMAL, knn=8), out,
                            unresolved, exc, 8)
    assert rc == abi.NBG_ERR_UNSUPPORTED
    assert "NBG_NOALLOC_MAX_POINTS" in msg
