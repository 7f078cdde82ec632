"""The pipelined kernels never spin forever: every mbarrier wait gives up
after a time limit, records a timeout status and returns.  The self-test
entry point runs that bounded wait on a barrier nothing completes (no fault,
no trap, no hang) and the device must stay usable afterwards."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KNNB200_ETIMEOUT = 5


def test_bounded_wait_times_out_and_context_survives(knncuda, oracle, gpu):
    t0 = time.perf_counter()
    rc = knncuda.selftest_wait_timeout(50_000_000)   # 50 ms
    dt = time.perf_counter() - t0
    assert rc == KNNB200_ETIMEOUT, knncuda.status_string(rc)
    assert 0.04 < dt < 5.0
    # the context is intact: an ordinary call right after gives exact results
    rng = np.random.default_rng(41)
    ref = rng.random((24, 3000), dtype=np.float32)
    query = rng.random((24, 50), dtype=np.float32)
    d, i = knncuda.knn(ref, query, 10)
    d64, i64 = oracle.knn_f64(ref, query, 10)
    assert np.array_equal(i, i64) or np.allclose(d, d64, rtol=1e-5)
    assert knncuda.sync_status() == 0


def test_bounded_wait_rejects_bad_limits(knncuda, gpu):
    assert knncuda.selftest_wait_timeout(0) == 1          # KNNB200_EINVAL
    assert knncuda.selftest_wait_timeout(2_000_000_000) == 1
