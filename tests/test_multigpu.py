"""Multi-process tests of the sharding logic (gloo, world_size 2, CPU).

The compute step is the CPU oracle (the C restatement of the reference's
knn_c), so the sharded answers must equal the single-process answer bit for
bit: per-pair distances do not depend on how the sets are split, and both
merges order by (distance, global index)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG, ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, result_path):
    for p in (PKG, ROOT):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist

    import multigpu
    from oracle import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        ref = rng.random((12, 701), dtype=np.float32)
        query = rng.random((12, 97), dtype=np.float32)
        compute = lambda r, q, k: oracle.knn_c(r, q, k)
        fn = multigpu.query_sharded_knn if mode == "query" else multigpu.ref_sharded_knn
        out = fn(ref, query, 9, compute)
        if rank == 0:
            np.savez(result_path, dist=out[0], index=out[1])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["query", "ref"])
def test_sharded_equals_single(tmp_path, oracle, mode):
    path = str(tmp_path / "out.npz")
    mp.start_processes(_worker, args=(2, _free_port(), mode, path), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(path)
    rng = np.random.default_rng(5)
    ref = rng.random((12, 701), dtype=np.float32)
    query = rng.random((12, 97), dtype=np.float32)
    d, i = oracle.knn_c(ref, query, 9)
    assert np.array_equal(got["dist"], d)
    assert np.array_equal(got["index"], i)


def test_shard_ranges_cover_exactly():
    import multigpu

    for n in (0, 1, 7, 16384):
        for world in (1, 2, 3, 8):
            spans = [multigpu.shard_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))


def test_merge_keeps_lower_index_on_ties():
    import multigpu

    # two shards with identical distances: the lower global index wins
    d0 = np.array([[1.0], [2.0]], np.float32)
    i0 = np.array([[0], [1]], np.int32)
    d1 = np.array([[1.0], [2.0]], np.float32)
    i1 = np.array([[0], [1]], np.int32)
    d, i = multigpu.merge_ref_shards([(d1, i1, 10), (d0, i0, 0)], 3)
    assert d[:, 0].tolist() == [1.0, 1.0, 2.0]
    assert i[:, 0].tolist() == [0, 10, 1]
