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
