"""One context shared by several host threads: uploads, runs and frees from
different threads serialise on the context, and every thread's results equal
the single-threaded ones (ctypes releases the GIL inside each call, so the
calls do interleave)."""
import threading

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def test_shared_context_across_threads(nbg):
    clouds = []
    for s in range(4):
        x, y, z = syn.tile(300_000 + 50_000 * s, 40 + s)
        clouds.append((x, y, z))
    stages = [abi.make_opts(abi.STAGE_NORMAL, knn=12),
              abi.make_opts(abi.STAGE_EIGENVALUES, knn=12)]
    want = []
    for x, y, z in clouds:
        t = nbg.tile(x, y, z)
        outs, _, _ = nbg.run(t, stages)
        t.free()
        want.append(outs)
    errors = []

    def worker(i):
        try:
            x, y, z = clouds[i]
            for _ in range(3):
                t = nbg.tile(x, y, z)
                outs, _, _ = nbg.run(t, stages)
                t.free()
                for g, w in zip(outs, want[i]):
                    assert np.array_equal(g, w, equal_nan=True)
        except Exception as e:  # reported to the main thread
            errors.append(repr(e))

    ths = [threading.Thread(target=worker, args=(i,)) for i in range(4)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    assert not errors, errors
