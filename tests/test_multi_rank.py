"""Host logic of the N > 1 bench path on CPU: two gloo ranks (replicas, no
data-path collective) agree on the max-over-ranks time, get different tiles,
and only rank 0 runs and prints the reference arm."""
import io
import os
import socket
import sys
import contextlib

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update(WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup()
    res = {"ws": w, "rank": r, "max": bench.rank_max(10.0 + r, w)}
    x, y, z = bench.workload(20_000, 2 + r)
    res["tile0"] = int(x[0])

    class A:
        points, knn, cpu_sample, warmup, steps, gpus = 20_000, 8, 5_000, 0, 1, ws
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(A, w, r)
    res["printed"] = buf.getvalue().strip() != ""
    dist.barrier()
    dist.destroy_process_group()
    out.put(res)


def test_two_gloo_ranks():
    from oracle import oracle
    if not oracle.available("port") and not oracle.available("reference"):
        pytest.skip("oracle library not built")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda d: d["rank"])
    assert all(d["ws"] == 2 for d in res)
    assert all(d["max"] == 11.0 for d in res)
    assert res[0]["tile0"] != res[1]["tile0"]
    assert res[0]["printed"] and not res[1]["printed"]
