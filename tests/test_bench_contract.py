"""The bench's reference arm and CPU baseline on CPU (small samples): the
JSON line carries the keys of the bench contract, and the CPU baseline
reports the all-threads and one-thread timings with the host's model."""
import contextlib
import io
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle_ready():
    from oracle import oracle
    return oracle.available("port") or oracle.available("reference")


@pytest.fixture(scope="module")
def bench():
    if not _oracle_ready():
        pytest.skip("oracle library not built")
    sys.path.insert(0, ROOT)
    import bench as b
    return b


def test_reference_line_keys(bench):
    class A:
        points, knn, cpu_sample, warmup, steps, gpus = 30_000, 8, 6_000, 0, 2, 1
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(A, 1, 0)
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["higher_is_better"] is True and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("reference", "port")
    assert cb["cores"] >= 1 and cb["nproc"] >= 1 and "cpu_model" in cb
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_cpu_baseline_single_thread(bench):
    x, y, z = bench.workload(40_000, 2)
    r = bench.cpu_reference(x, y, z, 8, 8_000, single_thread=True)
    st = r["single_thread"]
    assert st["cores"] == 1 and st["value"] > 0 and st["seconds"] > 0
    assert r["cores"] == (os.cpu_count() or 1) and r["value"] > 0


def test_cpu_baseline_runs_in_a_fresh_process(bench):
    # the main line's CPU baselines come from a child interpreter that has
    # touched no GPU; it prints one JSON object the main process reads
    class A:
        points, knn, cpu_sample, no_extras = 40_000, 8, 8_000, True
    out = bench.run_cpu_child(A)
    assert "error" not in out, out
    main = out["main"]
    assert main["value"] > 0 and main["cores"] == (os.cpu_count() or 1)
    assert main["single_thread"]["cores"] == 1
    assert "extras" not in out
