"""The no-allocation entry point (nbg_stage_noalloc), through the C ABI.

Callers that cannot allocate device memory when they need results (code
running inside another framework's allocator or memory pool, real-time loops
that must not call cudaMalloc/cudaFree, plug-in hosts that forbid allocation
in their processing callbacks) use this entry point: its working memory is a
fixed device array inside the library.  This file runs last so that a failure
here leaves every other test already run.

Checked for normal (always_up and the sign-exact always_up=false form),
eigenvalues (normalize) and covariancefeatures (feature_set=all, Density from
device OptimalKNN / OptimalRadius columns), each on two calls in a row:

* the rows it hands back are exactly the tie rows the oracle's integer
  distances show (plus the rows nbg_run defers), and their outputs are left
  untouched;
* every other row equals nbg_run's output and meets the parity bars of
  tests/_util.py against the FP64 oracle, with the same row statuses;
* refusals: a tile above the size limit, a tile extent of 2^24 raw units, a
  null exception array with a capacity, and a row-exception list smaller
  than the exceptions found (NBG_ERR_EXCEPTIONS, the count still reported).
"""
import ctypes

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from tests import _util as U

pytestmark = pytest.mark.gpu

CASES = {
    "normal_up": lambda: abi.make_opts(abi.STAGE_NORMAL, knn=8, always_up=True),
    "normal_sign": lambda: abi.make_opts(abi.STAGE_NORMAL, knn=8, always_up=False),
    "eigen_normalize": lambda: abi.make_opts(abi.STAGE_EIGENVALUES, knn=8, normalize=True),
    "covfeat_all": lambda: abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10,
                                         feature_mask=abi.FEAT_ALL),
}


def _columns(out, n):
    cols = abi.Columns()
    cols.base = out.data_ptr() if out is not None else 0
    cols.point_stride = 8
    cols.ndims = out.shape[0] if out is not None else 0
    cols.on_device = 1
    for d in range(cols.ndims):
        cols.offset[d] = d * n * 8
    return cols


def _call(lib, dx, dy, dz, n, opts, out, unresolved, exc, cap, kopt=None, ropt=None,
          exc_ptr=None):
    import torch
    cols = _columns(out, n)
    sc = (ctypes.c_double * 3)(0.01, 0.01, 0.01)
    of = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    nu = ctypes.c_uint32(0)
    ne = ctypes.c_uint32(0)
    msg = ctypes.create_string_buffer(256)
    rc = lib.nbg_stage_noalloc(
        dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), n, sc, of, ctypes.byref(opts),
        ctypes.byref(cols), kopt.data_ptr() if kopt is not None else None,
        ropt.data_ptr() if ropt is not None else None, unresolved.data_ptr(), ctypes.byref(nu),
        exc.data_ptr() if exc_ptr is None else exc_ptr, cap, ctypes.byref(ne), None, msg, 256)
    torch.cuda.synchronize()
    return rc, nu.value, ne.value, msg.value.decode()


def _exceptions(exc, count):
    from gpupdal_b200.native import EXC_DTYPE
    raw = exc.cpu().numpy().view(np.uint8)[: count * 8]
    return raw.view(np.dtype(EXC_DTYPE)).copy()


def _oracle_tie_rows(tree, x, y, z, K):
    """Rows whose K-th and (K+1)-th smallest integer squared distances are
    equal: the rows whose neighbour set depends on the reference's tie order."""
    nb = tree.all_neighbors(K + 1).astype(np.int64)
    P = np.stack([np.asarray(v, np.int64) for v in (x, y, z)], 1)
    d2 = np.sort(((P[nb] - P[:, None, :]) ** 2).sum(2), axis=1)
    return np.flatnonzero(d2[:, K - 1] == d2[:, K])


@pytest.fixture(scope="module")
def terrain():
    x, y, z = syn.terrain(250_000, 0)
    return x, y, z


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_two_calls_match_oracle_and_nbg_run(lib_path, port, terrain, case):
    import torch
    from gpupdal_b200.native import Context
    lib = abi.load_library()
    x, y, z = terrain
    n = len(x)
    assert n <= abi.NOALLOC_MAX_POINTS
    opts = CASES[case]()
    K = opts.knn + 1
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    dx, dy, dz = (torch.from_numpy(v).cuda() for v in (x, y, z))
    kopt = ropt = dk = dr = None
    if opts.kind == abi.STAGE_COVARIANCEFEATURES:
        kopt, ropt = syn.optimal_columns(n, 1, knn=opts.knn)
        dk, dr = torch.from_numpy(kopt).cuda(), torch.from_numpy(ropt).cuda()
    ctx = Context(0)
    tile = ctx.tile(dx, dy, dz)
    want_run, ex_run, stats = ctx.run(tile, [opts], optimal_knn=kopt, optimal_radius=ropt)
    want_run = want_run[0]
    tree = port.tree(X, Y, Z)
    ties = _oracle_tie_rows(tree, x, y, z, K)
    want64, st64 = tree.run_stage(opts, mode=1, optimal_knn=kopt, optimal_radius=ropt)
    lam, _ = tree.run_stage(abi.make_opts(abi.STAGE_EIGENVALUES, knn=opts.knn), mode=1)
    nd = len(abi.stage_dims(opts))
    cap = 4096
    for call in range(2):
        out = torch.full((nd, n), float("nan"), dtype=torch.float64, device="cuda")
        unresolved = torch.zeros(n, dtype=torch.int32, device="cuda")
        exc = torch.zeros(cap * 2, dtype=torch.int32, device="cuda")
        rc, nu, ne, msg = _call(lib, dx, dy, dz, n, opts, out, unresolved, exc, cap, dk, dr)
        assert rc == abi.NBG_OK, msg
        ids = np.sort(unresolved[:nu].cpu().numpy().astype(np.int64))
        # the handed-back rows: the tie rows the oracle sees, plus what nbg_run defers
        assert nu == int(stats.tie_rows + stats.deferred_rows), (
            f"{case} call {call}: {nu} rows handed back, nbg_run sent "
            f"{stats.tie_rows + stats.deferred_rows} to its exact path")
        assert np.isin(ties, ids).all(), f"{case} call {call}: a tie row was answered"
        assert len(ids) - len(ties) == int(stats.deferred_rows)
        got = out.cpu().numpy()
        assert np.isnan(got[:, ids]).all(), f"{case} call {call}: handed-back rows were written"
        keep = np.ones(n, bool)
        keep[ids] = False
        # same statuses as the oracle on the rows answered here
        got_ex = _exceptions(exc, ne)
        assert ne == int(np.count_nonzero(st64[keep]))
        got_st = U.status_from_exceptions(n, got_ex)
        assert np.array_equal(got_st[keep], st64[keep])
        ok = keep & (st64 == 0)
        # the regular entry point's outputs (the same kernels run)
        assert np.all(np.abs(got[:, ok] - want_run[:, ok]) <= 1e-5 *
                      np.maximum(1.0, np.abs(want_run[:, ok]))), f"{case} call {call}: vs nbg_run"
        # the FP64 oracle, within the parity bars
        sub = np.flatnonzero(keep)
        sign_free = True if (opts.kind == abi.STAGE_NORMAL and not opts.always_up) else None
        U.compare_stage(opts, got[:, sub], want64[:, sub], st64[sub], got_st[sub],
                        lam=lam[:, sub], label=f"{case} call {call} vs f64", sign_free=sign_free)


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


def test_noalloc_refuses_wide_tiles_and_null_exceptions(lib_path):
    import torch
    lib = abi.load_library()
    x = np.array([0, 1 << 24, 5, 9], np.int32)
    y = np.array([0, 0, 3, 7], np.int32)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    out = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    unresolved = torch.zeros(4, dtype=torch.int32, device="cuda")
    exc = torch.zeros(16, dtype=torch.int32, device="cuda")
    opts = abi.make_opts(abi.STAGE_NORMAL, knn=2)
    rc, _, _, msg = _call(lib, dx, dy, dy, 4, opts, out, unresolved, exc, 8)
    assert rc == abi.NBG_ERR_UNSUPPORTED and "2^24" in msg
    rc, _, _, msg = _call(lib, dy, dy, dy, 4, opts, out, unresolved, exc, 8, exc_ptr=0)
    assert rc == abi.NBG_ERR_INVALID and "exception" in msg


def test_noalloc_reports_exception_overflow(lib_path):
    # normal knn=1: two points per neighbourhood, so every row is the
    # reference's "fewer than 3 neighbours" skip (one exception per row)
    import torch
    lib = abi.load_library()
    rng = np.random.default_rng(5)
    n = 3000
    x, y, z = (rng.integers(0, 2000, n).astype(np.int32) for _ in range(3))
    dx, dy, dz = (torch.from_numpy(v).cuda() for v in (x, y, z))
    opts = abi.make_opts(abi.STAGE_NORMAL, knn=1)
    out = torch.full((4, n), float("nan"), dtype=torch.float64, device="cuda")
    unresolved = torch.zeros(n, dtype=torch.int32, device="cuda")
    cap = 100
    exc = torch.zeros(cap * 2, dtype=torch.int32, device="cuda")
    rc, nu, ne, msg = _call(lib, dx, dy, dz, n, opts, out, unresolved, exc, cap)
    assert rc == abi.NBG_ERR_EXCEPTIONS, msg
    assert ne == n - nu and ne > cap
    got = _exceptions(exc, cap)
    assert (got["code"] == abi.ROW_TOO_FEW).all()
