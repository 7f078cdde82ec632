"""GPU tests of the resident reference set and the continuous-batching server.

* RefSet.knn equals the per-call device entry point bit for bit (exact and
  tensor-core methods).
* Server: requests of mixed sizes and k, submitted from several threads so
  that they arrive while others are on the GPU, each get exactly the answer
  they get alone; a tight memory budget (admission holds batches back) still
  completes.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(seed, dim, n, q):
    rng = np.random.default_rng(seed)
    return rng.random((dim, n), dtype=np.float32), rng.random((dim, q), dtype=np.float32)


@pytest.mark.parametrize("method", ["global", "cublas"])
def test_refset_equals_device_entry(knncuda, gpu, method):
    import torch

    ref, query = _data(1, 96, 70000, 300)
    rs = knncuda.RefSet(ref)
    assert rs.device_bytes() >= ref.nbytes
    r = torch.from_numpy(ref).to(gpu)
    q = torch.from_numpy(query).to(gpu)
    for k in (1, 17, 100):
        d0, i0 = knncuda.knn_device(r, q, k, method)
        d1, i1 = rs.knn(q, k, method)
        assert torch.equal(d0, d1) and torch.equal(i0, i1)
    rs.close()


def test_refset_from_device_memory(knncuda, gpu):
    import torch

    ref, query = _data(2, 40, 5000, 64)
    r = torch.from_numpy(ref).to(gpu)
    rs = knncuda.RefSet(r)
    d, i = rs.knn(torch.from_numpy(query).to(gpu), 12)
    hd, hi = knncuda.knn(ref, query, 12)
    assert np.array_equal(d.cpu().numpy(), hd) and np.array_equal(i.cpu().numpy(), hi)
    rs.close()


def _alone(knncuda, rs, query, k, method, gpu):
    import torch

    dim, qn = query.shape
    buf = torch.zeros((dim, (qn + 3) // 4 * 4), dtype=torch.float32, device=gpu)
    buf[:, :qn] = torch.from_numpy(query)
    d, i = rs.knn(buf[:, :qn], k, method)
    return d.cpu().numpy(), i.cpu().numpy()


@pytest.mark.parametrize("method,budget", [("cublas", 8 << 30), ("global", 8 << 30),
                                           ("cublas", 48 << 20)])   # tight: few batches in flight
def test_server_results_same_alone_and_in_the_mix(knncuda, gpu, method, budget):
    ref, _ = _data(3, 128, 131072, 1)
    rs = knncuda.RefSet(ref)
    srv = knncuda.Server(rs, slots=3, memory_budget=budget, max_batch_queries=700,
                         method=method)
    rng = np.random.default_rng(4)
    reqs = []
    for _ in range(24):
        qn = int(np.exp(rng.uniform(0, np.log(400))))
        k = int(rng.choice([1, 10, 50, 100, 129]))
        reqs.append((rng.random((128, qn), dtype=np.float32), k))
    tickets = [None] * len(reqs)

    def submit(lo, hi):
        for j in range(lo, hi):
            tickets[j] = srv.submit(*reqs[j])

    threads = [threading.Thread(target=submit, args=(a, a + 8)) for a in (0, 8, 16)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert st["queries"] == sum(q.shape[1] for q, _ in reqs)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()
    for (query, k), (d, i, lat) in zip(reqs, results):
        ad, ai = _alone(knncuda, rs, query, k, method, gpu)
        assert lat > 0
        assert np.array_equal(d.view(np.uint32), ad.view(np.uint32))
        assert np.array_equal(i, ai)
    rs.close()


def test_server_rejects_request_beyond_budget(knncuda, gpu):
    ref, _ = _data(5, 32, 40000, 1)
    rs = knncuda.RefSet(ref)
    srv = knncuda.Server(rs, slots=1, memory_budget=1 << 20, max_batch_queries=100000,
                         method="global")
    with pytest.raises(RuntimeError):
        srv.submit(np.zeros((32, 60000), np.float32), 50)   # its working set alone > 1 MiB
    srv.close()
    rs.close()
