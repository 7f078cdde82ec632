"""CPU tests of the oracle: pinned against the reference's own knn_c.

* oracle restatement == golden fixtures (outputs of the reference knn_c), bit for bit;
* oracle restatement == reference knn_c (oracle/_ref) on fresh seeded inputs, bit for bit;
* the FP64 oracle and the checkers behave on hand-made cases.
"""
import glob
import os

import numpy as np
import pytest

from knn_check import check_exact, recall_at_k

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 8


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden_bitwise(oracle, path):
    g = np.load(path)
    dist, idx = oracle.knn_c(g["ref"], g["query"], int(g["k"]), threads=2)
    assert np.array_equal(dist.view(np.uint32), g["dist"].view(np.uint32))
    assert np.array_equal(idx, g["index"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden_is_exact_vs_fp64(oracle, path):
    g = np.load(path)
    k = int(g["k"])
    d64, i64 = oracle.knn_f64(g["ref"], g["query"], k)
    check_exact(g["dist"], g["index"], g["ref"], g["query"], d64, i64)


@pytest.mark.parametrize("seed,dim,n,q,k", [(1, 128, 2048, 64, 16), (2, 3, 5000, 100, 8),
                                           (3, 33, 777, 31, 40), (4, 1, 300, 20, 7)])
def test_oracle_matches_reference_knn_c(oracle, seed, dim, n, q, k):
    if not oracle.ref_available():
        pytest.skip("reference knn_c not built (oracle/_ref)")
    rng = np.random.default_rng(seed)
    ref = rng.random((dim, n), dtype=np.float32)
    query = rng.random((dim, q), dtype=np.float32)
    d0, i0 = oracle.ref_knn_c(ref, query, k)
    d1, i1 = oracle.knn_c(ref, query, k, threads=3)
    assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
    assert np.array_equal(i0, i1)
    # the threaded driver around the reference gives the same answer
    d2, i2 = oracle.ref_knn_c(ref, query, k, threads=4)
    assert np.array_equal(d0, d2) and np.array_equal(i0, i2)


def test_tie_order_lower_index_first(oracle):
    # all reference points equidistant from the query: indices must come out 0..k-1
    ref = np.array([[1.0, -1.0, 1.0, -1.0, 1.0, -1.0]], np.float32)
    query = np.zeros((1, 1), np.float32)
    d, i = oracle.knn_c(ref, query, 4)
    assert i[:, 0].tolist() == [0, 1, 2, 3]
    assert np.all(d == 1.0)
    d64, i64 = oracle.knn_f64(ref, query, 4)
    assert i64[:, 0].tolist() == [0, 1, 2, 3]


def test_fp64_oracle_on_line(oracle):
    ref = np.arange(10, dtype=np.float32)[None, :]
    query = np.array([[3.2, 7.9]], np.float32)
    d, i = oracle.knn_f64(ref, query, 3)
    assert i[:, 0].tolist() == [3, 4, 2]
    assert i[:, 1].tolist() == [8, 7, 9]
    assert np.allclose(d[:, 0], [0.2, 0.8, 1.2], atol=1e-6)


def test_checker_rejects_wrong_results(oracle):
    rng = np.random.default_rng(5)
    ref = rng.random((8, 200), dtype=np.float32)
    query = rng.random((8, 10), dtype=np.float32)
    d64, i64 = oracle.knn_f64(ref, query, 6)
    d, i = oracle.knn_c(ref, query, 6)
    check_exact(d, i, ref, query, d64, i64)
    assert recall_at_k(i, i64) == 1.0
    bad_i = i.copy()
    bad_i[-1, 0] = (i64[:, 0].max() + 1) % 200
    while bad_i[-1, 0] in i[:, 0]:
        bad_i[-1, 0] = (bad_i[-1, 0] + 1) % 200
    with pytest.raises(AssertionError):
        check_exact(d, bad_i, ref, query, d64, i64)
    bad_d = d.copy()
    bad_d[0, 3] *= 1.01
    with pytest.raises(AssertionError):
        check_exact(bad_d, i, ref, query, d64, i64)


def test_reference_criterion(oracle):
    rng = np.random.default_rng(6)
    ref = rng.random((4, 100), dtype=np.float32)
    query = rng.random((4, 30), dtype=np.float32)
    d, i = oracle.knn_c(ref, query, 5)
    ok, dacc, iacc = oracle.reference_criterion(d, i, d, i)
    assert ok and dacc == 1.0 and iacc == 1.0
    i2 = i.copy()
    i2[0, :] = -1
    ok, _, iacc = oracle.reference_criterion(d, i2, d, i)
    assert not ok and iacc == pytest.approx(1 - 30 / 150)
