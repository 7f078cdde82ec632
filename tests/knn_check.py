"""Result checkers shared by the parity tests.

Two criteria are applied to every k-NN result (dist, index: k x Q):

* the reference harness's rule (code/test.cpp:216-217, :256-272):
  |dist - gt| <= 1e-3 absolute and index == gt index position by position,
  each for >= 99.9% of entries -- ``oracle.reference_criterion``;
* the stricter exactness rule used for this engine, against an FP64 brute
  force: distances within REL_TOL relative of FP64, ascending per query,
  each returned (index, distance) pair consistent with the FP64 distance of
  that index, no repeated index, and index SETS identical to FP64's except
  for points whose FP64 distance ties with the k-th FP64 distance within
  tolerance -- ``check_exact``.
"""
from __future__ import annotations

import numpy as np

REL_TOL = 1e-3     # distances within 1e-3 relative of FP64
ABS_FLOOR = 1e-6   # absolute floor for (near-)zero distances


def fp64_dist(ref, query, idx):
    """FP64 distance of query i to reference idx[j, i], shape (k, Q)."""
    r = ref.astype(np.float64)
    q = query.astype(np.float64)
    k, Q = idx.shape
    out = np.empty((k, Q))
    for i in range(Q):
        diff = r[:, idx[:, i]] - q[:, i:i + 1]
        out[:, i] = np.sqrt(np.sum(diff * diff, axis=0))
    return out


def check_exact(dist, idx, ref, query, d64, i64, rel=REL_TOL):
    """Raise AssertionError with a description if the result is not exact."""
    dist = np.asarray(dist)
    idx = np.asarray(idx)
    k, Q = d64.shape
    assert dist.shape == (k, Q) and idx.shape == (k, Q), (dist.shape, idx.shape, (k, Q))
    assert np.all(np.isfinite(dist)), "non-finite distance"
    ref_nb = ref.shape[1]
    assert idx.min() >= 0 and idx.max() < ref_nb, "index out of range"
    # ascending per query
    assert np.all(np.diff(dist, axis=0) >= 0), "distances not ascending"
    tol = np.maximum(rel * np.abs(d64), ABS_FLOOR)
    err = np.abs(dist.astype(np.float64) - d64)
    bad = err > tol
    assert not bad.any(), (f"{bad.sum()} distances off FP64 by more than {rel} rel; "
                           f"max rel err {np.max(err / np.maximum(np.abs(d64), ABS_FLOOR)):.3g}")
    # (index, distance) consistency
    recomputed = fp64_dist(ref, query, idx)
    tol2 = np.maximum(rel * recomputed, ABS_FLOOR)
    assert np.all(np.abs(dist - recomputed) <= tol2), "distance does not match its index"
    # distinct indices per query
    s = np.sort(idx, axis=0)
    assert np.all(np.diff(s, axis=0) != 0), "repeated index within a query"
    # index sets equal except ties at the k-th boundary
    kth = d64[-1]
    for i in range(Q):
        a = set(idx[:, i].tolist())
        b = set(i64[:, i].tolist())
        if a == b:
            continue
        band = max(rel * kth[i], ABS_FLOOR)
        extra = a - b
        missing = b - a
        ex_d = recomputed[:, i][[j for j, v in enumerate(idx[:, i]) if v in extra]]
        mi_d = d64[:, i][[j for j, v in enumerate(i64[:, i]) if v in missing]]
        assert np.all(np.abs(ex_d - kth[i]) <= band) and np.all(np.abs(mi_d - kth[i]) <= band), (
            f"query {i}: index sets differ beyond boundary ties "
            f"(extra {sorted(extra)[:5]}, missing {sorted(missing)[:5]})")


def recall_at_k(idx, i64):
    k, Q = i64.shape
    hit = 0
    for i in range(Q):
        hit += len(set(idx[:, i].tolist()) & set(i64[:, i].tolist()))
    return hit / (k * Q)


def max_rel_err(dist, d64):
    return float(np.max(np.abs(dist.astype(np.float64) - d64) / np.maximum(np.abs(d64), ABS_FLOOR)))


def check_exact_sampled_torch(torch, ref_d, qry_d, dist, idx, sample, rel=REL_TOL):
    """check_exact on sampled queries of a large problem, with the FP64 brute
    force computed by torch on the device that holds ref_d (dim x n) and
    qry_d (dim x Q).  dist / idx: (k, Q) tensors or arrays.  Returns
    (recall@k, max relative distance error) over the sample."""
    dist = torch.as_tensor(dist, device=ref_d.device)
    idx = torch.as_tensor(idx, device=ref_d.device).long()
    k = idx.shape[0]
    r64 = ref_d.double()
    hits, worst = 0, 0.0
    for q in sample:
        d2 = ((r64 - qry_d[:, q].double()[:, None]) ** 2).sum(0)
        top = torch.topk(d2, k, largest=False)           # ascending (sorted=True)
        truth_d = torch.sqrt(top.values)
        mine_i = idx[:, q]
        mine_d = dist[:, q].double()
        exact_mine = torch.sqrt(d2[mine_i])
        tol = torch.clamp(rel * exact_mine, min=ABS_FLOOR)
        assert bool(((mine_d - exact_mine).abs() <= tol).all()), f"query {q}: distance/index mismatch"
        assert bool((mine_d[1:] >= mine_d[:-1]).all()), f"query {q}: not ascending"
        assert torch.unique(mine_i).numel() == k, f"query {q}: repeated index"
        tol2 = torch.clamp(rel * truth_d, min=ABS_FLOOR)
        assert bool(((mine_d - truth_d).abs() <= tol2).all()), f"query {q}: rank distances off FP64"
        a, b = set(mine_i.tolist()), set(top.indices.tolist())
        hits += len(a & b)
        if a != b:
            kth = float(truth_d[-1])
            band = max(rel * kth, ABS_FLOOR)
            for j in (a - b) | (b - a):
                assert abs(float(torch.sqrt(d2[j])) - kth) <= band, (
                    f"query {q}: index sets differ beyond boundary ties")
        worst = max(worst, float(((mine_d - exact_mine).abs() /
                                  torch.clamp(exact_mine, min=ABS_FLOOR)).max()))
    return hits / (k * len(sample)), worst
