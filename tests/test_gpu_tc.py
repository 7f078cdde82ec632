"""GPU parity tests of the tensor-core expansion path (knn_cublas).

The BF16 tcgen05 candidate scan is followed by an exact FP32 re-rank in the
fused exact kernel's arithmetic and a certification against the derived BF16
error bound; uncertified queries are recomputed by the exact kernel.  So the
strongest property holds: knn_cublas returns exactly what knn_cuda_global
returns, bit for bit, on every shape -- certified or not.
"""
import os

import numpy as np
import pytest

from knn_check import check_exact, recall_at_k

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 4


def _uniform(seed, dim, n, q):
    rng = np.random.default_rng(seed)
    return rng.random((dim, n), dtype=np.float32), rng.random((dim, q), dtype=np.float32)


CASES = [
    # (seed, ref_nb, query_nb, dim, k)
    (1, 65536, 300, 64, 16),
    (2, 65536, 513, 128, 100),
    (3, 40000, 257, 256, 128),       # ragged N, k at the tensor-path maximum
    (4, 32768, 1, 32, 1),            # Q = 1, k = 1
    (5, 70001, 1000, 200, 50),       # d not a multiple of 64
    (6, 131072, 96, 16, 10),         # smallest tensor-path dim
    (7, 33000, 300, 96, 20),         # last 256-point tile: second half partly valid
]


@pytest.mark.parametrize("case", CASES, ids=[f"n{c[1]}q{c[2]}d{c[3]}k{c[4]}" for c in CASES])
def test_cublas_equals_global_bitwise(knncuda, gpu, case):
    seed, n, q, dim, k = case
    ref, query = _uniform(seed, dim, n, q)
    dg, ig = knncuda.knn(ref, query, k, "global")
    dc, ic = knncuda.knn(ref, query, k, "cublas")
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)


def test_cublas_exact_vs_fp64_and_reference(knncuda, oracle, gpu):
    ref, query = _uniform(11, 96, 50000, 64)
    d, i = knncuda.knn(ref, query, 32, "cublas")
    gt_d, gt_i = oracle.knn_c(ref, query, 32, threads=THREADS)
    ok, dacc, iacc = oracle.reference_criterion(d, i, gt_d, gt_i)
    assert ok, (dacc, iacc)
    d64, i64 = oracle.knn_f64(ref, query, 32, threads=THREADS)
    check_exact(d, i, ref, query, d64, i64)
    assert recall_at_k(i, i64) > 0.999


def test_mixture_near_ties(knncuda, oracle, gpu):
    """Clustered data (sigma 0.05 around 256 centres): dense near-ties."""
    import workloads

    w = workloads.WORKLOADS["mixture128"]
    ref, query = workloads.generate(w, ref_nb=131072, query_nb=700)
    dg, ig = knncuda.knn(ref, query, w.k, "global")
    dc, ic = knncuda.knn(ref, query, w.k, "cublas")
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)
    sample = np.arange(0, 700, 70)
    qs = np.ascontiguousarray(query[:, sample])
    d64, i64 = oracle.knn_f64(ref, qs, w.k, threads=THREADS)
    check_exact(dc[:, sample], ic[:, sample], ref, qs, d64, i64)


def test_headline_workload_mostly_certified(knncuda, gpu):
    """1M x 256 mixture, k = 100: the BF16 scan certifies almost every query,
    and the answer is the exact kernel's."""
    import workloads

    w = workloads.WORKLOADS["mixture256"]
    ref, query = workloads.generate(w, query_nb=1024)
    dg, ig = knncuda.knn(ref, query, w.k, "global")
    dc, ic = knncuda.knn(ref, query, w.k, "cublas")
    second, exact = knncuda.last_fallback_counts()
    assert second <= 1024 // 50 and exact <= second, (second, exact)
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)


def test_second_scan_certifies_threshold_failures(knncuda, gpu):
    """Clustered 256-d data where the sampled threshold is sometimes too low:
    those queries are certified by the second scan, not by the exact kernel."""
    import workloads

    w = workloads.WORKLOADS["mixture256"]
    ref, query = workloads.generate(w, ref_nb=262144, query_nb=4096)
    dg, ig = knncuda.knn(ref, query, w.k, "global")
    dc, ic = knncuda.knn(ref, query, w.k, "cublas")
    second, exact = knncuda.last_fallback_counts()
    assert exact == 0, (second, exact)
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)


def test_exact_fallback_takes_only_the_still_uncertified(knncuda, gpu):
    """Three queries sit on 10000 copies of one point (more equal distances
    than the longest second-chance list holds): only they go to the exact
    kernel.  Three more sit on 2000 copies of another point: their pass-2
    lists overflow and the second scan's longer lists certify them.  The
    answer equals the exact kernel's, ties to the lower index."""
    import torch

    ref, query = _uniform(31, 64, 65536, 300)
    ref[:, 1000:11000] = ref[:, [5]]
    ref[:, 30000:32000] = ref[:, [7]]
    rng = np.random.default_rng(32)
    for j, col in enumerate((5, 5, 5, 7, 7, 7)):
        query[:, 10 + 40 * j] = ref[:, col] + 1e-3 * rng.standard_normal(64).astype(np.float32)
    r, x = torch.from_numpy(ref).to(gpu), _pitched(torch, gpu, query)
    dg, ig = knncuda.knn_device(r, x, 16, "global")
    dc, ic = knncuda.knn_device(r, x, 16, "cublas")
    second, exact = knncuda.last_fallback_counts()
    assert knncuda.sync_status() == 0
    assert exact >= 3 and second > exact, (second, exact)
    assert torch.equal(dc, dg) and torch.equal(ic, ig)


def test_device_entry_cublas(knncuda, gpu):
    import torch

    ref, query = _uniform(21, 128, 65536, 200)
    hd, hi = knncuda.knn(ref, query, 20, "global")
    r = torch.from_numpy(ref).to(gpu)
    q = torch.from_numpy(query).to(gpu)
    d, i = knncuda.knn_device(r, q, 20, "cublas")
    assert knncuda.sync_status() == 0
    assert np.array_equal(d.cpu().numpy(), hd)
    assert np.array_equal(i.cpu().numpy(), hi)


def _unit_clusters(seed, dim, n, q, centres, sigma, sort):
    """Unit-norm centres plus N(0, sigma^2) noise; with sort, the reference
    points are stored cluster by cluster (each cluster's points contiguous)."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((dim, centres)).astype(np.float32)
    c /= np.linalg.norm(c, axis=0, keepdims=True)
    pick = rng.integers(0, centres, size=n)
    if sort:
        pick = np.sort(pick)
    ref = c[:, pick] + np.float32(sigma) * rng.standard_normal((dim, n), dtype=np.float32)
    qry = c[:, rng.integers(0, centres, size=q)] + np.float32(sigma) * rng.standard_normal(
        (dim, q), dtype=np.float32)
    return np.ascontiguousarray(ref, dtype=np.float32), np.ascontiguousarray(qry, dtype=np.float32)


def test_threshold_sample_spans_a_cluster_sorted_set(knncuda, gpu):
    """A reference set stored cluster by cluster gets thresholds as good as
    the same kind of set in random order: the threshold sample of a set
    prepared as a whole is every 16th point, spread over all clusters, not
    runs of consecutive tiles (which would see a few clusters only and make
    every list of the other clusters' queries overflow).  The answers are
    knn_cuda_global's, bit for bit."""
    import torch

    n, q, dim, k = 131072, 512, 64, 32
    stats = {}
    for sort in (False, True):
        ref, query = _unit_clusters(31, dim, n, q, 128, 0.1, sort)
        r = torch.from_numpy(ref).to(gpu)
        qq = torch.from_numpy(query).to(gpu)
        dg, ig = knncuda.knn_device(r, qq, k, "global")
        dc, ic = knncuda.knn_device(r, qq, k, "cublas")
        st = knncuda.last_tc_stats()
        assert torch.equal(dc, dg) and torch.equal(ic, ig)
        stats[sort] = st
    assert stats[True]["exact"] == 0, stats
    assert stats[True]["second_scan"] <= stats[False]["second_scan"] + q // 50, stats
    assert stats[True]["candidates"] <= 1.5 * stats[False]["candidates"], stats


def test_streamed_cluster_sorted_set_needs_no_exact_fallback(knncuda, gpu):
    """knn_cublas from page-locked host buffers samples runs of tiles (pass 1
    starts before the set has arrived), so on a set stored cluster by
    cluster most queries' lists overflow.  The k-th exact distance of the
    entries an overflowing list kept bounds the true k-th from above, so the
    second scan gets thresholds that certify: no query goes to the exact
    kernel, and the answers are knn_cuda_global's bit for bit."""
    import torch

    n, q, dim, k = 262144, 512, 64, 32
    ref, query = _unit_clusters(7, dim, n, q, 256, 0.1, True)
    ref_p = torch.from_numpy(ref).pin_memory().numpy()
    qry_p = torch.from_numpy(query).pin_memory().numpy()
    d = torch.empty((k, q), dtype=torch.float32).pin_memory().numpy()
    i = torch.empty((k, q), dtype=torch.int32).pin_memory().numpy()
    assert knncuda.knn_cublas(ref_p, n, qry_p, q, dim, k, d, i)
    second, exact = knncuda.last_fallback_counts()
    dg, ig = np.empty((k, q), np.float32), np.empty((k, q), np.int32)
    assert knncuda.knn_cuda_global(ref, n, query, q, dim, k, dg, ig)
    assert np.array_equal(d.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(i, ig)
    assert second > 0 and exact == 0, (second, exact)


def _far_clusters(seed, dim, n, centres, radius, sigma):
    """Tight clusters around centres in random directions at distance radius
    from the origin: the set's mean is near 0, so translating it does not
    shrink the norms, while in-cluster distances are tiny against them."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((dim, centres))
    c *= radius / np.linalg.norm(c, axis=0, keepdims=True)
    pick = rng.integers(0, centres, size=n)
    x = c[:, pick] + sigma * rng.standard_normal((dim, n))
    return np.ascontiguousarray(x, dtype=np.float32)


def test_fallback_path_exercised(knncuda, gpu):
    """16 tight clusters at radius 6 in 256-d: the BF16 error bound exceeds
    the in-cluster spread, every point of the query's cluster becomes a
    candidate and the lists overflow, so queries take the second scan (and
    the exact kernel); results must still equal knn_cuda_global."""
    ref = _far_clusters(31, 256, 32768, 16, 6.0, 0.05)
    query = _far_clusters(31, 256, 32768 + 400, 16, 6.0, 0.05)[:, 32768:].copy()
    dg, ig = knncuda.knn(ref, query, 100, "global")
    dc, ic = knncuda.knn(ref, query, 100, "cublas")
    second, exact = knncuda.last_fallback_counts()
    assert second > 0 and exact <= second
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)


def test_offset_data_is_translated_before_the_bf16_scan(knncuda, gpu):
    """All coordinates in [50, 51): norms are ~100x the distances, so the BF16
    expansion's error bound would swallow every distance gap.  The scan works
    on both sets translated by a sample mean (distances unchanged), so the
    queries certify without the exact kernel, and results equal
    knn_cuda_global bit for bit."""
    rng = np.random.default_rng(37)
    ref = (rng.random((64, 65536), dtype=np.float32) + np.float32(50)).astype(np.float32)
    query = (rng.random((64, 300), dtype=np.float32) + np.float32(50)).astype(np.float32)
    dg, ig = knncuda.knn(ref, query, 20, "global")
    dc, ic = knncuda.knn(ref, query, 20, "cublas")
    second, exact = knncuda.last_fallback_counts()
    assert exact == 0, (second, exact)
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)


def test_overflowing_lists_rescanned_with_longer_lists(knncuda, gpu):
    """Clusters whose in-cluster distance spread is below the BF16 error
    slack, through the host entry from page-locked buffers (the streamed
    path, whose pass 2 starts before the set has arrived and so cannot
    switch kinds): most BF16 candidate lists overflow on the first scan, and
    the second scan runs in split BF16 with longer lists instead of sending
    those queries to the exact kernel.  Results equal knn_cuda_global bit
    for bit."""
    import torch
    import workloads

    w = workloads.WORKLOADS["mixture128"]
    ref0, query0 = workloads.generate(w, ref_nb=262144, query_nb=1000)
    ref = torch.from_numpy(ref0).pin_memory().numpy()
    query = torch.from_numpy(query0).pin_memory().numpy()
    dg, ig = knncuda.knn(ref0, query0, w.k, "global")
    d = torch.empty((w.k, 1000), dtype=torch.float32).pin_memory().numpy()
    i = torch.empty((w.k, 1000), dtype=torch.int32).pin_memory().numpy()
    assert knncuda.knn_cublas(ref, 262144, query, 1000, 128, w.k, d, i)
    second, exact = knncuda.last_fallback_counts()
    first_kind, second_kind = knncuda.last_tc_kinds()
    assert first_kind == "bf16" and second > 0, (first_kind, second)
    assert second_kind == "bf16x3" and exact < second, (second_kind, second, exact)
    assert np.array_equal(d.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(i, ig)


@pytest.mark.parametrize("n,dim,k", [(262144, 64, 20),     # tile-aligned, 8 whole chunks
                                     (299108, 96, 100),    # ragged last sample tile and chunk
                                     (262244, 48, 20),     # last sample run: one ragged tile
                                     (1 << 20, 256, 100)])  # the headline shape
def test_cublas_host_streamed_from_pinned_memory(knncuda, gpu, n, dim, k):
    """knn_cublas from page-locked host buffers on a large set streams the
    reference set in (the threshold sample's runs of tiles first, then
    chunks without them, each scanned once it has landed); the answer equals
    knn_cuda_global's bit for bit."""
    import torch

    rng = np.random.default_rng(n + dim)
    q = 300
    ref = torch.from_numpy(rng.random((dim, n), dtype=np.float32)).pin_memory().numpy()
    query = torch.from_numpy(rng.random((dim, q), dtype=np.float32)).pin_memory().numpy()
    d0, i0 = np.empty((k, q), np.float32), np.empty((k, q), np.int32)
    d1 = torch.empty((k, q), dtype=torch.float32).pin_memory().numpy()
    i1 = torch.empty((k, q), dtype=torch.int32).pin_memory().numpy()
    assert knncuda.knn_cuda_global(ref, n, query, q, dim, k, d0, i0)
    for _ in range(2):   # the second call reuses the workspace's buffers
        d1[:] = -1
        i1[:] = -1
        assert knncuda.knn_cublas(ref, n, query, q, dim, k, d1, i1)
        assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
        assert np.array_equal(i0, i1)


HIGH_DIM = [
    # (seed, ref_nb, query_nb, dim, k): d > 256 (A streamed beside B above
    # d = 512) and k in (128, 256]
    (61, 40000, 300, 384, 200),
    (62, 36000, 260, 512, 200),
    (63, 33000, 200, 1024, 200),
    (64, 50000, 300, 130, 256),
    (65, 40000, 513, 640, 64),
]


@pytest.mark.parametrize("case", HIGH_DIM, ids=[f"n{c[1]}q{c[2]}d{c[3]}k{c[4]}" for c in HIGH_DIM])
def test_tensor_path_high_dim_and_large_k(knncuda, gpu, case):
    """knn_cublas on d up to 1024 and k up to 256 runs the tcgen05 scan and
    returns exactly knn_cuda_global's answer (the reference's knn_cublas
    has no d limit, code/knncuda.cu:612-832)."""
    seed, n, q, dim, k = case
    ref, query = _uniform(seed, dim, n, q)
    dg, ig = knncuda.knn(ref, query, k, "global")
    dc, ic = knncuda.knn(ref, query, k, "cublas")
    first, _ = knncuda.last_tc_kinds()
    assert first in ("bf16", "bf16x3"), first
    assert knncuda.last_tc_stats()["candidates"] > 0
    assert np.array_equal(dc.view(np.uint32), dg.view(np.uint32))
    assert np.array_equal(ic, ig)


FP8_CASES = [
    # (seed, ref_nb, query_nb, dim, k)
    (71, 65536, 300, 16, 16),
    (72, 65536, 513, 32, 32),
    (73, 65536, 513, 128, 100),
    (74, 40000, 257, 256, 128),
    (75, 50000, 200, 200, 50),       # d not a multiple of 128: zero-padded K block
    (76, 33000, 150, 1024, 32),
]


def _pitched(torch, gpu, x):
    """(dim, n) device copy in a buffer whose row pitch is a multiple of 4."""
    dim, n = x.shape
    buf = torch.zeros((dim, (n + 3) // 4 * 4), dtype=torch.float32, device=gpu)
    buf[:, :n] = torch.from_numpy(x)
    return buf[:, :n]


def test_fp8_scan_equals_global_bitwise(knncuda, gpu):
    """The FP8 (e4m3, power-of-two scaled) candidate scan, certified against
    its own error bound and re-ranked exactly, returns the exact kernel's
    answer bit for bit.  Pass 2 is forced to FP8 (the sample pass would
    predict overflowing FP8 lists on uniform data and run BF16): queries
    whose FP8 lists overflow take the second scan, the rest certify."""
    import torch

    knncuda.set_tc_kind_override("fp8")
    try:
        for seed, n, q, dim, k in FP8_CASES:
            ref, query = _uniform(seed, dim, n, q)
            r, x = _pitched(torch, gpu, ref), _pitched(torch, gpu, query)
            dg, ig = knncuda.knn_device(r, x, k, "global")
            df, i8 = knncuda.knn_device(r, x, k, "fp8")
            assert knncuda.sync_status() == 0
            assert knncuda.last_tc_kinds()[0] == "fp8", (dim, knncuda.last_tc_kinds())
            assert torch.equal(df, dg) and torch.equal(i8, ig), dim
    finally:
        knncuda.set_tc_kind_override(None)


def _clusters(seed, dim, n, centres, sigma, q):
    """Tight clusters (about n / centres points each) around unit-norm
    centres: distance gaps between clusters far above the FP8 bound."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((dim, centres))
    c /= np.linalg.norm(c, axis=0, keepdims=True)
    pick = rng.integers(0, centres, size=n + q)
    x = (c[:, pick] + sigma * rng.standard_normal((dim, n + q))).astype(np.float32)
    return np.ascontiguousarray(x[:, :n]), np.ascontiguousarray(x[:, n:])


def test_fp8_scan_certifies_on_tight_clusters(knncuda, gpu):
    """256 clusters of about 512 points, far apart: the sample (one tile in
    16) holds about 32 points of the query's cluster, so the threshold lies
    inside it, and forced FP8 lists (the whole cluster, under 1024 entries)
    certify without a second scan for most queries; exact answers."""
    import torch

    ref, query = _clusters(81, 128, 131072, 256, 0.01, 500)
    r, x = torch.from_numpy(ref).to(gpu), _pitched(torch, gpu, query)
    dg, ig = knncuda.knn_device(r, x, 16, "global")
    knncuda.set_tc_kind_override("fp8")
    try:
        df, i8 = knncuda.knn_device(r, x, 16, "fp8")
        kinds = knncuda.last_tc_kinds()
        second, _ = knncuda.last_fallback_counts()
    finally:
        knncuda.set_tc_kind_override(None)
    assert kinds[0] == "fp8"
    assert second <= 50, second
    assert torch.equal(df, dg) and torch.equal(i8, ig)


def test_fp8_request_on_headline_mixture(knncuda, gpu):
    """On the headline mixture the FP8 bound (about 1.1 in squared distance)
    exceeds the in-cluster spread (about 0.45): the sample pass predicts
    overflowing lists and the call runs BF16, with the exact answer."""
    import torch
    import workloads

    w = workloads.WORKLOADS["mixture256"]
    ref, query = workloads.generate(w, query_nb=1024)
    r, x = torch.from_numpy(ref).to(gpu), torch.from_numpy(query).to(gpu)
    dg, ig = knncuda.knn_device(r, x, w.k, "global")
    df, i8 = knncuda.knn_device(r, x, w.k, "fp8")
    assert knncuda.sync_status() == 0
    assert knncuda.last_tc_kinds()[0] in ("bf16", "bf16x3")
    assert torch.equal(df, dg) and torch.equal(i8, ig)


def test_split_bf16_when_bf16_would_overflow(knncuda, gpu):
    """mixture128's BF16 error slack exceeds its in-cluster spread: the
    threshold pass predicts overflowing lists and pass 2 runs in split BF16
    (hi + lo parts), so the exact kernel is not needed."""
    import workloads

    import torch

    w = workloads.WORKLOADS["mixture128"]
    ref, query = workloads.generate(w, ref_nb=262144, query_nb=2000)
    r, x = torch.from_numpy(ref).to(gpu), torch.from_numpy(query).to(gpu)
    dg, ig = knncuda.knn_device(r, x, w.k, "global")
    dc, ic = knncuda.knn_device(r, x, w.k, "cublas")
    assert knncuda.sync_status() == 0
    first, second = knncuda.last_tc_kinds()
    _, exact = knncuda.last_fallback_counts()
    assert first == "bf16x3", (first, second)
    assert exact == 0
    assert torch.equal(dc, dg) and torch.equal(ic, ig)


@pytest.mark.parametrize("n,dim,k", [(299108, 96, 100), (1 << 20, 256, 100)])
def test_cublas_host_streamed_from_pageable_memory(knncuda, gpu, n, dim, k):
    """knn_cublas from ordinary (pageable) host buffers, as the reference's
    harness passes them (code/test.cpp:314-317): the reference set is
    gathered piece by piece into pinned staging buffers and streamed in
    under the scans; the answer equals knn_cuda_global's bit for bit, on two
    calls in a row (the staging buffers are reused)."""
    rng = np.random.default_rng(n + 7 * dim)
    q = 257
    ref = rng.random((dim, n), dtype=np.float32)
    query = rng.random((dim, q), dtype=np.float32)
    d0, i0 = knncuda.knn(ref, query, k, "global")
    for _ in range(2):
        d1, i1 = knncuda.knn(ref, query, k, "cublas")
        assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
        assert np.array_equal(i0, i1)
