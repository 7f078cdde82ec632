"""GPU test of knnb200_knn_device_noalloc, the entry point for callers that
cannot allocate device memory (their memory belongs to their own pool, or
cudaMalloc / cudaFree -- which can stall the whole device -- are not allowed
where they call from).

The call is made through the C ABI with caller-owned inputs and outputs; its
result must match the ordinary device entry point (knnb200_knn_device,
which uses the library's allocated workspace) on two calls in a row: the
second call runs on the static scratch area exactly as the first one left
it.  Both run the same kernel with the same arithmetic, so the distances are
required to agree bit for bit, which also keeps them inside the 1e-3
relative tolerance the other parity tests use.  This file is collected last
so that a run stopping at the first failure has run every other test first;
it needs nothing from the other tests and passes in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-3          # the distance tolerance of the other parity tests
STATIC_SCRATCH = 64 << 20


def _noalloc(knncuda, r, q, k, dist, index, stream):
    return knncuda.lib().knnb200_knn_device_noalloc(
        r.data_ptr(), r.shape[1], r.stride(0), q.data_ptr(), q.shape[1], q.stride(0),
        r.shape[0], k, dist.data_ptr(), index.data_ptr(), dist.stride(0),
        ctypes.c_void_p(stream.cuda_stream))


def test_noalloc_matches_device_entry_twice(knncuda, gpu):
    import torch

    dim, n, qn, k = 48, 20000, 150, 32
    # the planner splits the reference set, so the static scratch is in use
    assert knncuda.plan_splits(n, qn, dim, k) > 1
    assert 0 < knncuda.scratch_bytes(n, qn, dim, k) <= STATIC_SCRATCH
    rng = np.random.default_rng(77)
    r = torch.from_numpy(rng.random((dim, n), dtype=np.float32)).to(gpu)
    stream = torch.cuda.current_stream(gpu)
    for call in range(2):
        # ragged query count in a row-pitched buffer (pitch a multiple of 4)
        qbuf = torch.zeros((dim, qn + 2), dtype=torch.float32, device=gpu)
        qbuf[:, :qn] = torch.from_numpy(rng.random((dim, qn), dtype=np.float32))
        q = qbuf[:, :qn]
        want_d, want_i = knncuda.knn_device(r, q, k, "global")
        torch.cuda.synchronize(gpu)
        d = torch.full((k, qn), -1.0, dtype=torch.float32, device=gpu)
        i = torch.full((k, qn), -1, dtype=torch.int32, device=gpu)
        assert _noalloc(knncuda, r, q, k, d, i, stream) == 0, f"call {call}"
        got_d, got_i = d.cpu().numpy(), i.cpu().numpy()
        want_d, want_i = want_d.cpu().numpy(), want_i.cpu().numpy()
        np.testing.assert_allclose(got_d, want_d, rtol=REL_TOL, atol=1e-6)
        assert np.array_equal(got_d.view(np.uint32), want_d.view(np.uint32)), f"call {call}"
        assert np.array_equal(got_i, want_i), f"call {call}"


def test_noalloc_rejects_shapes_beyond_static_scratch(knncuda, gpu, capfd):
    import torch

    # the duplicated query copy alone (dim * round_up(qn, 32) * 8 bytes) is
    # 72 MiB here, whatever the split planner chooses
    dim, n, qn, k = 256, 4096, 36864, 8
    need = knncuda.scratch_bytes(n, qn, dim, k)
    assert need > STATIC_SCRATCH, need
    r = torch.zeros((dim, n), dtype=torch.float32, device=gpu)
    q = torch.zeros((dim, qn), dtype=torch.float32, device=gpu)
    d = torch.zeros((k, qn), dtype=torch.float32, device=gpu)
    i = torch.zeros((k, qn), dtype=torch.int32, device=gpu)
    rc = _noalloc(knncuda, r, q, k, d, i, torch.cuda.current_stream(gpu))
    assert rc == 8   # KNNB200_ESCRATCH
    assert "static maximum" in capfd.readouterr().out
