"""Parity at the full sizes of the benchmark configurations.

Each configuration runs at its stated size through the C ABI; results are
checked by size-independent properties on every query (ascending distances,
distinct indices, the exact and tensor paths bit-identical) and exactly
against an FP64 brute force on sampled queries (distances within 1e-3
relative, index sets equal except boundary ties), plus the reference
harness's criterion against knn_c (code/test.cpp:216-217) where the CPU
oracle finishes in seconds.

  2a  262,144 x 16,384, d = 128, k = 32, mixture of 256 clusters, sigma 0.05
  2b  1,048,576 x 65,536, d = 3, k = 8, U[0,1)^3 point cloud
  3   1,048,576 x 16,384, d = 256, k = 100, mixture of 1024 unit-norm centres
  4   512 uneven problems from one seed, one persistent launch
  5   2,097,152 x 128 resident set, a mixed-size, mixed-k request stream
"""
import os
import threading

import numpy as np
import pytest

from knn_check import check_exact, check_exact_sampled_torch

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 4


def _props(d, i):
    assert np.all(np.isfinite(d))
    assert np.all(np.diff(d, axis=0) >= 0), "not ascending"
    s = np.sort(i, axis=0)
    assert np.all(np.diff(s, axis=0) != 0), "repeated index"


def _sampled_vs_oracle(oracle, ref, query, d, i, k, sample):
    qs = np.ascontiguousarray(query[:, sample])
    gt_d, gt_i = oracle.knn_c(ref, qs, k, threads=THREADS)
    ok, dacc, iacc = oracle.reference_criterion(d[:, sample], i[:, sample], gt_d, gt_i)
    assert ok, (dacc, iacc)
    d64, i64 = oracle.knn_f64(ref, qs, k, threads=THREADS)
    check_exact(d[:, sample], i[:, sample], ref, qs, d64, i64)


def test_config_2a_mixture128_full(knncuda, oracle, gpu):
    import workloads

    w = workloads.WORKLOADS["mixture128"]
    ref, query = workloads.generate(w)
    assert ref.shape == (128, 262144) and query.shape == (128, 16384)
    dg, ig = knncuda.knn(ref, query, w.k, "global")
    dc, ic = knncuda.knn(ref, query, w.k, "cublas")
    _props(dg, ig)
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)
    _sampled_vs_oracle(oracle, ref, query, dg, ig, w.k, np.arange(0, 16384, 256))


def test_config_2b_cloud3_full(knncuda, oracle, gpu):
    import workloads

    w = workloads.WORKLOADS["cloud3"]
    ref, query = workloads.generate(w)
    assert ref.shape == (3, 1 << 20) and query.shape == (3, 65536)
    d, i = knncuda.knn(ref, query, w.k, "global")
    _props(d, i)
    dc, ic = knncuda.knn(ref, query, w.k, "cublas")   # d < 16: the same exact kernels
    assert np.array_equal(dc.view(np.uint32), d.view(np.uint32)) and np.array_equal(ic, i)
    _sampled_vs_oracle(oracle, ref, query, d, i, w.k, np.arange(0, 65536, 1024))


def test_config_3_mixture256_full(knncuda, gpu):
    import torch
    import workloads

    w = workloads.WORKLOADS["mixture256"]
    ref, query = workloads.generate(w)
    r, q = torch.from_numpy(ref).to(gpu), torch.from_numpy(query).to(gpu)
    dg, ig = knncuda.knn_device(r, q, w.k, "global")
    dc, ic = knncuda.knn_device(r, q, w.k, "cublas")
    assert knncuda.sync_status() == 0
    assert torch.equal(dg, dc) and torch.equal(ig, ic)
    _props(dg.cpu().numpy(), ig.cpu().numpy())
    recall, err = check_exact_sampled_torch(torch, r, q, dc, ic, range(0, 16384, 256))
    assert recall > 0.999 and err <= 1e-3, (recall, err)


def test_config_4_batched512_full(knncuda, gpu):
    import torch
    import workloads

    shapes = workloads.batched_problems()
    assert len(shapes) == 512
    probs, outs, exp = [], [], []
    for n, qn, d, k, seed in shapes:
        g = torch.Generator(device=gpu).manual_seed(seed)
        ldr, ldq = (n + 3) // 4 * 4, (qn + 3) // 4 * 4
        ref = torch.rand((d, ldr), generator=g, device=gpu)[:, :n]
        qry = torch.rand((d, ldq), generator=g, device=gpu)[:, :qn]
        probs.append((ref, qry, k))
        outs.append((torch.full((k, qn), -1.0, device=gpu),
                     torch.full((k, qn), -1, dtype=torch.int32, device=gpu)))
        exp.append(knncuda.knn_device(ref, qry, k, "global"))
    torch.cuda.synchronize()
    arr = knncuda.problems_from([(r, q, k, d, i) for (r, q, k), (d, i) in zip(probs, outs)])
    plan = knncuda.BatchedPlan(arr)
    plan.run()
    assert plan.status() == 0
    for (d, i), (ed, ei) in zip(outs, exp):
        assert torch.equal(d, ed) and torch.equal(i, ei)
    plan.close()
    # every problem exact against FP64 on its first and last query
    for (ref, qry, k), (d, i) in zip(probs, outs):
        qn = qry.shape[1]
        check_exact_sampled_torch(torch, ref, qry, d, i, sorted({0, qn - 1}))


def test_config_5_serving_2m_full(knncuda, gpu):
    import torch
    import workloads

    w = workloads.WORKLOADS["serving128"]
    ref, _ = workloads.generate(w, query_nb=1)
    assert ref.shape == (128, 2097152)
    rs = knncuda.RefSet(ref)
    reqs = workloads.serving_requests(w, 40)
    srv = knncuda.Server(rs, slots=3, memory_budget=8 << 30, max_batch_queries=4096,
                         method="cublas")
    tickets = [None] * len(reqs)

    def submit(lo, hi):
        for j in range(lo, hi):
            tickets[j] = srv.submit(*reqs[j])

    threads = [threading.Thread(target=submit, args=(a, a + 20)) for a in (0, 20)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["queries"] == sum(q.shape[1] for q, _ in reqs)
    ref_d = torch.from_numpy(ref).to(gpu)
    for j, ((query, k), (d, i, lat)) in enumerate(zip(reqs, results)):
        qn = query.shape[1]
        qbuf = torch.zeros((128, (qn + 3) // 4 * 4), dtype=torch.float32, device=gpu)
        qbuf[:, :qn] = torch.from_numpy(query)
        ad, ai = rs.knn(qbuf[:, :qn], k, "global")
        assert np.array_equal(d.view(np.uint32), ad.cpu().numpy().view(np.uint32)), j
        assert np.array_equal(i, ai.cpu().numpy()), j
        if j % 8 == 0:
            check_exact_sampled_torch(torch, ref_d, qbuf[:, :qn], d, i, [0, qn - 1])
    rs.close()
