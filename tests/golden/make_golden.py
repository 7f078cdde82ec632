"""Generate the golden k-NN fixtures from the reference's own knn_c.

Runs the reference's unmodified CPU ground truth, ``knn_c``
(code/test.cpp:129-175, compiled by oracle/Makefile into
oracle/_ref/libknnref_c.so), on small seeded inputs and stores inputs and
outputs in tests/golden/*.npz.  The fixtures pin the oracle restatement
(bit-identical outputs) and serve as parity targets for the CUDA path.

    make -C oracle ref && python tests/golden/make_golden.py [name ...]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402


def cases():
    """name -> (ref, query, k, note).  Values are seeded and small."""
    out = {}
    rng = np.random.default_rng(11)
    # the reference harness's own value range: 10 * U[0,1) (code/test.cpp:31-38)
    out["uniform10_d7"] = (10 * rng.random((7, 300), dtype=np.float32),
                           10 * rng.random((7, 40), dtype=np.float32), 5,
                           "10*U[0,1), ragged sizes")
    rng = np.random.default_rng(12)
    out["uniform_d32"] = (rng.random((32, 1000), dtype=np.float32),
                          rng.random((32, 64), dtype=np.float32), 16, "U[0,1)")
    # exact ties: integer 1-D points with many duplicates; ties must keep the lower index
    rng = np.random.default_rng(13)
    out["ties_d1"] = (rng.integers(0, 12, size=(1, 64)).astype(np.float32),
                      rng.integers(0, 12, size=(1, 16)).astype(np.float32), 8,
                      "integer grid, exact distance ties")
    # duplicated reference points in 2-D
    rng = np.random.default_rng(14)
    base = rng.integers(0, 5, size=(2, 40)).astype(np.float32)
    out["dups_d2"] = (np.concatenate([base, base, base], axis=1),
                      rng.integers(0, 5, size=(2, 24)).astype(np.float32), 10,
                      "every reference point appears three times")
    rng = np.random.default_rng(15)
    out["ragged_d3"] = (rng.random((3, 257), dtype=np.float32),
                        rng.random((3, 33), dtype=np.float32), 32, "d=3, N=257, Q=33")
    rng = np.random.default_rng(16)
    centres = rng.random((8, 16), dtype=np.float32)
    a = rng.integers(0, 8, size=2048)
    ref = (centres.T[:, a] + 0.01 * rng.standard_normal((16, 2048), dtype=np.float32))
    b = rng.integers(0, 8, size=50)
    qry = (centres.T[:, b] + 0.01 * rng.standard_normal((16, 50), dtype=np.float32))
    out["mixture_d16"] = (ref.astype(np.float32), qry.astype(np.float32), 20,
                          "tight clusters, near ties")
    rng = np.random.default_rng(17)
    out["k_eq_n"] = (rng.random((5, 48), dtype=np.float32),
                     rng.random((5, 7), dtype=np.float32), 48, "k == ref_nb")
    rng = np.random.default_rng(18)
    out["single_query"] = (rng.random((64, 700), dtype=np.float32),
                           rng.random((64, 1), dtype=np.float32), 1, "Q=1, k=1")
    # k well above 256: the reference's insertion sort has no limit on k
    rng = np.random.default_rng(19)
    out["large_k"] = (10 * rng.random((8, 2000), dtype=np.float32),
                      10 * rng.random((8, 24), dtype=np.float32), 1000,
                      "k=1000 of 2000 points, 10*U[0,1)")
    return out


def main(names=None):
    """Write every fixture, or only those named on the command line."""
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libknnref_c.so missing: run make -C oracle ref")
    for name, (ref, query, k, note) in cases().items():
        if names and name not in names:
            continue
        ref = np.ascontiguousarray(ref, dtype=np.float32)
        query = np.ascontiguousarray(query, dtype=np.float32)
        dist, idx = oracle.ref_knn_c(ref, query, k)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, ref=ref, query=query, k=np.int32(k), dist=dist, index=idx,
                            note=np.array(note))
        print(f"{name}: ref {ref.shape} query {query.shape} k={k} -> {path}")


if __name__ == "__main__":
    main(sys.argv[1:])
