"""GPU tests of memory admission: when the buffers for all queries of a call
do not fit in the memory the library may use, the host and device entry
points run the queries in chunks (as the reference's legacy code split its
queries by free memory, legacy/KNN.CUDA.with.indexes/
knn_cuda_with_indexes.cu:348-349, :406-444), with bit-identical results.
The usable memory is lowered with the library's host-side cap, so no test
needs a full GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [
    # (ref_nb, query_nb, dim, k, method)
    (50000, 3000, 64, 16, "global"),
    (50000, 3000, 64, 16, "cublas"),     # tensor path: reference prepared once
    (40000, 2000, 24, 300, "texture"),   # k > 256 passes in every chunk
]


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{s[4]}_k{s[3]}" for s in SHAPES])
def test_host_entry_chunks_by_memory(knncuda, gpu, shape):
    n, q, d, k, method = shape
    rng = np.random.default_rng(n + k)
    ref = rng.random((d, n), dtype=np.float32)
    query = rng.random((d, q), dtype=np.float32)
    want_d, want_i = knncuda.knn(ref, query, k, method)
    assert knncuda.last_query_chunks() == 1
    cap = knncuda.call_bytes(n, q // 4, d, k, method, host=True)
    knncuda.set_memory_cap(cap)
    try:
        got_d, got_i = knncuda.knn(ref, query, k, method)
        chunks = knncuda.last_query_chunks()
    finally:
        knncuda.set_memory_cap(0)
    assert chunks >= 3, chunks
    assert np.array_equal(got_d.view(np.uint32), want_d.view(np.uint32))
    assert np.array_equal(got_i, want_i)


@pytest.mark.parametrize("method", ["global", "cublas"])
def test_device_entry_chunks_by_memory(knncuda, gpu, method):
    import torch

    n, q, d, k = 60000, 2500, 96, 20
    rng = np.random.default_rng(91)
    r = torch.from_numpy(rng.random((d, n), dtype=np.float32)).to(gpu)
    x = torch.from_numpy(rng.random((d, q), dtype=np.float32)).to(gpu)
    want_d, want_i = knncuda.knn_device(r, x, k, method)
    torch.cuda.synchronize()
    cap = knncuda.call_bytes(n, q // 4, d, k, method, host=False)
    knncuda.set_memory_cap(cap)
    try:
        got_d, got_i = knncuda.knn_device(r, x, k, method)
        assert knncuda.sync_status() == 0
        chunks = knncuda.last_query_chunks()
    finally:
        knncuda.set_memory_cap(0)
    assert chunks >= 3, chunks
    assert torch.equal(got_d, want_d) and torch.equal(got_i, want_i)


def test_cap_too_small_for_one_query_fails_cleanly(knncuda, gpu, capfd):
    rng = np.random.default_rng(92)
    ref = rng.random((32, 5000), dtype=np.float32)
    query = rng.random((32, 100), dtype=np.float32)
    knncuda.set_memory_cap(1 << 10)
    try:
        d = np.empty((8, 100), np.float32)
        i = np.empty((8, 100), np.int32)
        assert knncuda.knn_cuda_global(ref, 5000, query, 100, 32, 8, d, i) is False
    finally:
        knncuda.set_memory_cap(0)
    assert "ERROR: Memory allocation error" in capfd.readouterr().out
    # and the next call works
    d0, i0 = knncuda.knn(ref, query, 8)
    assert np.all(np.diff(d0, axis=0) >= 0)
