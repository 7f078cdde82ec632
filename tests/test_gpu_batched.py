"""GPU tests of the batched persistent launch: many uneven problems in one
launch from a device work queue give exactly the per-problem answers, also
when replayed from a captured CUDA graph and with autotuned work items."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(torch, gpu, seed, count, kmax=64, dims=(3, 32, 64, 128, 256)):
    """Uneven problems in the spirit of the batched workload: ref_nb
    log-uniform 1k-24k, query_nb log-uniform 16-600, dim from `dims`, k 1..kmax."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(24000))))
        q = int(np.exp(rng.uniform(np.log(16), np.log(600))))
        d = int(rng.choice(dims))
        k = int(rng.integers(1, kmax + 1))
        ldr = (n + 3) // 4 * 4
        ref = torch.zeros((d, ldr), dtype=torch.float32, device=gpu)
        ref[:, :n] = torch.rand((d, n), generator=torch.Generator().manual_seed(int(rng.integers(1 << 30)))).to(gpu)
        query = torch.rand((d, q), generator=torch.Generator().manual_seed(int(rng.integers(1 << 30)))).to(gpu)
        out.append((ref[:, :n], query, k))
    return out


def _outputs(torch, gpu, probs):
    return [(torch.full((k, q.shape[1]), -1.0, device=gpu),
             torch.full((k, q.shape[1]), -1, dtype=torch.int32, device=gpu)) for _, q, k in probs]


def _expected(knncuda, torch, probs):
    exp = []
    for ref, q, k in probs:
        qp = torch.zeros((q.shape[0], (q.shape[1] + 3) // 4 * 4), device=q.device)
        qp[:, :q.shape[1]] = q
        d, i = knncuda.knn_device(ref, qp[:, :q.shape[1]], k)
        exp.append((d, i))
    torch.cuda.synchronize()
    return exp


@pytest.mark.parametrize("kmax", [64, 200])
def test_batched_equals_per_problem(knncuda, gpu, kmax):
    import torch

    probs = _problems(torch, gpu, 11 + kmax, 96, kmax=kmax)
    exp = _expected(knncuda, torch, probs)
    outs = _outputs(torch, gpu, probs)
    arr = knncuda.problems_from([(r, q, k, d, i) for (r, q, k), (d, i) in zip(probs, outs)])
    plan = knncuda.BatchedPlan(arr, item_stages=128)
    assert plan.items() >= len(probs)
    plan.run()
    assert plan.status() == 0
    for (d, i), (ed, ei) in zip(outs, exp):
        assert torch.equal(d, ed) and torch.equal(i, ei)
    plan.close()


def test_batched_graph_replay_and_autotune(knncuda, gpu):
    import torch

    probs = _problems(torch, gpu, 21, 64)
    exp = _expected(knncuda, torch, probs)
    outs = _outputs(torch, gpu, probs)
    arr = knncuda.problems_from([(r, q, k, d, i) for (r, q, k), (d, i) in zip(probs, outs)])
    best, ms = knncuda.batched_autotune(arr)
    assert best in (32, 64, 128, 256, 512, 1024, 2048) and ms > 0
    plan = knncuda.BatchedPlan(arr, item_stages=best)
    plan.capture_graph()
    for _ in range(2):
        for d, i in outs:
            d.fill_(-1.0)
            i.fill_(-1)
        plan.replay()
        assert plan.status() == 0
        for (d, i), (ed, ei) in zip(outs, exp):
            assert torch.equal(d, ed) and torch.equal(i, ei)
    plan.close()


@pytest.mark.parametrize("qpw,lowdim", [(2, 0), (2, 1), (4, 1)])
def test_batched_configurations_equal_per_problem(knncuda, gpu, qpw, lowdim):
    """Both tile shapes, with and without routing d <= 4 / k <= 16 problems
    to the low-dimension kernel, give exactly the per-problem answers, also
    replayed from a captured graph."""
    import torch

    probs = _problems(torch, gpu, 31 + qpw + lowdim, 80, kmax=40)
    exp = _expected(knncuda, torch, probs)
    outs = _outputs(torch, gpu, probs)
    arr = knncuda.problems_from([(r, q, k, d, i) for (r, q, k), (d, i) in zip(probs, outs)])
    cfg = knncuda.BatchedConfig(128, qpw, lowdim)
    plan = knncuda.BatchedPlan(arr, config=cfg)
    info = plan.config()
    assert info["queries_per_warp"] == qpw
    n_low = sum(1 for r, q, k in probs if r.shape[0] <= 4 and k <= 16)
    assert info["lowdim_problems"] == (n_low if lowdim else 0)
    plan.capture_graph()
    plan.replay()
    assert plan.status() == 0
    for (d, i), (ed, ei) in zip(outs, exp):
        assert torch.equal(d, ed) and torch.equal(i, ei)
    plan.close()


def test_batched_autotune_config(knncuda, gpu):
    import torch

    probs = _problems(torch, gpu, 41, 48)
    exp = _expected(knncuda, torch, probs)
    outs = _outputs(torch, gpu, probs)
    arr = knncuda.problems_from([(r, q, k, d, i) for (r, q, k), (d, i) in zip(probs, outs)])
    best, ms = knncuda.batched_autotune_config(arr)
    assert best.queries_per_warp in (2, 4) and best.lowdim_kernel in (0, 1) and ms > 0
    plan = knncuda.BatchedPlan(arr, config=best)
    plan.run()
    assert plan.status() == 0
    for (d, i), (ed, ei) in zip(outs, exp):
        assert torch.equal(d, ed) and torch.equal(i, ei)
    plan.close()
