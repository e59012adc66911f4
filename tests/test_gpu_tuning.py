"""The autotuner's tuning file: choices (cell factor and select kernel) made in
one context, saved and loaded into a fresh context, are applied there without
measuring (use_cache), and the cache refuses malformed entries."""
import pytest

from gpupdal_b200 import synthetic as syn
from gpupdal_b200.native import Context, NbgError

pytestmark = pytest.mark.gpu


def test_tuning_file_round_trip(nbg, tmp_path):
    x, y, z = syn.mixture(1_000_000, 7)
    tile = nbg.tile(x, y, z)
    chosen = tile.autotune(16, candidates=[2.0, 4.0])
    assert chosen in (2.0, 4.0)
    cache = nbg.tuning_cache()
    assert len(cache) >= 1
    # 1M points: class floor(log2 n) = 19
    assert any(e["size_class"] == 19 and e["cell_factor"] == chosen for e in cache)
    # the select kernel is chosen with the cell factor
    assert all(e["select_kernel"] in (0, 1, 2, 32) for e in cache)
    path = tmp_path / "tuning.json"
    nbg.save_tuning(path)
    fresh = Context(0)
    try:
        assert fresh.tuning_cache() == []
        assert fresh.load_tuning(path) == len(cache)
        assert fresh.tuning_cache() == cache
        # a cached class is applied without measuring: the factor comes back
        # even when it is not among the candidates offered
        t2 = fresh.tile(x, y, z)
        assert t2.autotune(16, candidates=[1.0], use_cache=True) == chosen
        with pytest.raises(NbgError):
            fresh.set_tuning_cache([{"size_class": 19, "slots": 18, "cell_factor": -1.0}])
        with pytest.raises(NbgError):
            fresh.set_tuning_cache([{"size_class": 99, "slots": 18, "cell_factor": 2.0}])
        with pytest.raises(NbgError):
            fresh.set_tuning_cache([{"size_class": 19, "slots": 18, "cell_factor": 2.0,
                                     "select_kernel": 7}])
        assert fresh.tuning_cache() == cache
    finally:
        fresh.close()


def test_cached_tuning_reaches_untuned_tiles():
    """nbg_run applies the context's cached choice of a tile's class (here
    loaded, as from a tuning file) to tiles the caller did not tune, and leaves
    a tile whose select kernel the caller set alone; results are the same."""
    from gpupdal_b200 import abi
    import numpy as np

    x, y, z = syn.mixture(1_000_000, 7)
    st = [abi.make_opts(abi.STAGE_NORMAL, knn=16)]
    ctx = Context(0)
    try:
        # 1M points: class 19; knn 16 -> 17 neighbours -> 18 select slots.
        # Kernel 2 (single pass) hands some rows to the two-pass search,
        # kernel 0 never does: the retry count shows which one ran.
        ctx.set_tuning_cache([{"size_class": 19, "slots": 18, "cell_factor": 3.0,
                               "select_kernel": 2}])
        untuned = ctx.tile(x, y, z)
        out_a, ex_a, st_a = ctx.run(untuned, st)
        untuned.free()
        assert st_a.retry_rows > 0
        chosen = ctx.tile(x, y, z)
        chosen.set_select(0)
        out_b, ex_b, st_b = ctx.run(chosen, st)
        chosen.free()
        assert st_b.retry_rows == 0
        assert np.array_equal(out_a[0], out_b[0], equal_nan=True)
        assert np.array_equal(np.sort(ex_a, order=["point_id", "stage"]),
                              np.sort(ex_b, order=["point_id", "stage"]))
    finally:
        ctx.close()
