"""Seeded synthetic point sets for the k-NN workloads.

No public dataset is used by the reference or named for this engine, so every
workload is a seeded synthetic stand-in with the stated shape and value
distribution.  Point sets use the reference's layout: a dim x n row-major
float32 array, point i's coordinate d at ``x[d, i]`` (README.md "Data storage
and representation"; code/test.cpp:63).

Workloads (name: ref_nb, query_nb, dim, k, distribution, seed):

* ``readme``   16384, 4096, 128, 16 -- i.i.d. U[0,1) (the reference's default
  problem, code/test.cpp:295-298; the reference draws 10*U[0,1)).
* ``mixture128`` 262144, 16384, 128, 32 -- mixture of 256 isotropic Gaussian
  clusters, centres U[-1,1]^d, sigma 0.05 (many near-ties).
* ``cloud3``   1048576, 65536, 3, 8 -- U[0,1)^3 point cloud.
* ``mixture256`` 1048576, 16384, 256, 100 -- mixture of 1024 unit-norm centres
  (normalised Gaussian), sigma 0.1.
* ``batched512`` 512 independent problems (seed 5): ref_nb log-uniform
  1k-64k, query_nb log-uniform 16-2048, dim in {3, 32, 64, 128, 256}, k
  uniform 1-64, i.i.d. U[0,1) -- ``batched_problems``.
* ``serving128`` 2097152 resident points, dim 128 -- mixture of 2048
  unit-norm centres, sigma 0.1; requests of 1..1024 queries (log-uniform)
  with k in {10, 50, 100}, Poisson arrivals (query_nb / k below are the
  request maxima).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Workload:
    name: str
    ref_nb: int
    query_nb: int
    dim: int
    k: int
    dist: str          # "uniform" | "mixture"
    seed: int
    centres: int = 0
    sigma: float = 0.0
    centre_kind: str = ""   # "uniform11" | "unitnorm"

    def describe(self) -> dict:
        d = {"workload": self.name, "ref_nb": self.ref_nb, "query_nb": self.query_nb,
             "dim": self.dim, "k": self.k, "distribution": self.dist, "seed": self.seed}
        if self.dist == "mixture":
            d.update(centres=self.centres, sigma=self.sigma, centre_kind=self.centre_kind)
        return d

    def data_text(self) -> str:
        """One line naming the synthetic distribution of this workload."""
        if self.dist == "mixture":
            kind = {"unitnorm": "unit-norm", "uniform11": "U[-1,1]^d"}.get(self.centre_kind,
                                                                          self.centre_kind)
            return (f"synthetic (seeded Gaussian mixture, {self.centres} {kind} centres, "
                    f"sigma {self.sigma})")
        return "synthetic (seeded i.i.d. U[0,1))"


WORKLOADS = {
    "readme": Workload("readme", 16384, 4096, 128, 16, "uniform", 1),
    "mixture128": Workload("mixture128", 262144, 16384, 128, 32, "mixture", 2,
                           centres=256, sigma=0.05, centre_kind="uniform11"),
    "cloud3": Workload("cloud3", 1048576, 65536, 3, 8, "uniform", 3),
    "mixture256": Workload("mixture256", 1048576, 16384, 256, 100, "mixture", 4,
                           centres=1024, sigma=0.1, centre_kind="unitnorm"),
    "serving128": Workload("serving128", 2097152, 1024, 128, 100, "mixture", 6,
                           centres=2048, sigma=0.1, centre_kind="unitnorm"),
}


def batched_problems(count: int = 512, seed: int = 5):
    """Shapes (ref_nb, query_nb, dim, k) and a data seed per problem of the
    batched workload."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(65536))))
        q = int(np.exp(rng.uniform(np.log(16), np.log(2048))))
        d = int(rng.choice([3, 32, 64, 128, 256]))
        k = int(rng.integers(1, 65))
        out.append((n, q, d, k, int(rng.integers(1 << 31))))
    return out


def serving_requests(w: Workload, count: int, seed: int = 66):
    """Request stream for the serving workload: (queries dim x q, k) with q
    log-uniform in [1, w.query_nb] and k drawn from {10, 50, 100}; the queries
    come from the same mixture as the reference set."""
    rng = np.random.default_rng(w.seed)
    centres = make_centres(rng, w.centres, w.dim, w.centre_kind)
    rq = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        q = int(np.exp(rq.uniform(0.0, np.log(w.query_nb + 1))))
        q = max(1, min(w.query_nb, q))
        k = int(rq.choice([10, 50, 100]))
        out.append((np.ascontiguousarray(mixture_points(rq, centres, q, w.sigma)), k))
    return out


def uniform_points(rng: np.random.Generator, dim: int, n: int) -> np.ndarray:
    return rng.random((dim, n), dtype=np.float32)


def mixture_points(rng: np.random.Generator, centres: np.ndarray, n: int,
                   sigma: float) -> np.ndarray:
    """n points, each a uniformly chosen centre plus N(0, sigma^2) per coordinate."""
    dim = centres.shape[1]
    assign = rng.integers(0, centres.shape[0], size=n)
    pts = rng.standard_normal((dim, n), dtype=np.float32)
    pts *= np.float32(sigma)
    pts += centres.T[:, assign]
    return pts


def make_centres(rng: np.random.Generator, count: int, dim: int, kind: str) -> np.ndarray:
    if kind == "uniform11":
        return (rng.random((count, dim), dtype=np.float32) * 2 - 1).astype(np.float32)
    if kind == "unitnorm":
        c = rng.standard_normal((count, dim), dtype=np.float32)
        c /= np.linalg.norm(c, axis=1, keepdims=True)
        return c.astype(np.float32)
    raise ValueError(kind)


def generate(w: Workload, ref_nb: int | None = None, query_nb: int | None = None):
    """(ref, query) for workload w; sizes may be overridden (same distribution)."""
    n_ref = w.ref_nb if ref_nb is None else ref_nb
    n_q = w.query_nb if query_nb is None else query_nb
    rng = np.random.default_rng(w.seed)
    if w.dist == "uniform":
        ref = uniform_points(rng, w.dim, n_ref)
        query = uniform_points(rng, w.dim, n_q)
    else:
        centres = make_centres(rng, w.centres, w.dim, w.centre_kind)
        ref = mixture_points(rng, centres, n_ref, w.sigma)
        query = mixture_points(rng, centres, n_q, w.sigma)
    return np.ascontiguousarray(ref), np.ascontiguousarray(query)


def random_problem(seed: int, ref_nb: int, query_nb: int, dim: int, scale: float = 1.0):
    """Small seeded U[0,scale) problem for parity tests."""
    rng = np.random.default_rng(seed)
    ref = (rng.random((dim, ref_nb), dtype=np.float32) * np.float32(scale)).astype(np.float32)
    query = (rng.random((dim, query_nb), dtype=np.float32) * np.float32(scale)).astype(np.float32)
    return ref, query
