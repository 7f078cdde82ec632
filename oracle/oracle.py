"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle.

Loaded by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference arm, as the checker and the CPU baseline -- never by the product
path (``knn-cuda_b200``), which fails loudly without its CUDA library.

Two CPU implementations of the reference's ground truth are exposed:

* ``knn_c`` -- oracle/knn_oracle.c, a C restatement of the reference's
  ``knn_c`` (code/test.cpp:129-175); bit-identical to it.
* ``ref_knn_c`` -- the reference's own ``knn_c`` compiled from its unmodified
  code/test.cpp into oracle/_ref/libknnref_c.so (present when it was built
  from the sources; see oracle/Makefile).

plus ``knn_f64``, an FP64 brute force ordered by (distance, index).

All take dim x n row-major float32 arrays (``x[d, i]``) and return
(dist, index) arrays of shape (k, query_nb), the reference's output layout
(code/test.cpp:164-165).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libknnoracle.so")
REF_C_SO = os.path.join(HERE, "_ref", "libknnref_c.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libknnref_gpu.so")

_FP = ctypes.POINTER(ctypes.c_float)
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)

_oracle = None
_ref_c = None


def _load_oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle)")
        lib = ctypes.CDLL(ORACLE_SO)
        for name, dp in (("oracle_knn_c", _FP), ("oracle_knn_f64", _DP)):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [_FP, ctypes.c_int, _FP, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                           dp, _IP, ctypes.c_int]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_C_SO)


def _load_ref():
    global _ref_c
    if _ref_c is None:
        if not ref_available():
            raise RuntimeError(f"reference knn_c library missing: {REF_C_SO}")
        lib = ctypes.CDLL(REF_C_SO)
        lib.ref_knn_c.restype = ctypes.c_int
        lib.ref_knn_c.argtypes = [_FP, ctypes.c_int, _FP, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, _FP, _IP]
        lib.ref_knn_c_mt.restype = ctypes.c_int
        lib.ref_knn_c_mt.argtypes = [_FP, ctypes.c_int, _FP, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, _FP, _IP, ctypes.c_int]
        _ref_c = lib
    return _ref_c


def _prep(ref, query, k):
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    query = np.ascontiguousarray(query, dtype=np.float32)
    if ref.ndim != 2 or query.ndim != 2 or ref.shape[0] != query.shape[0]:
        raise ValueError("ref and query must be dim x n arrays with the same dim")
    dim, ref_nb = ref.shape
    query_nb = query.shape[1]
    if not (1 <= k <= ref_nb):
        raise ValueError("k must be in [1, ref_nb]")
    return ref, query, dim, ref_nb, query_nb


def _fp(a):
    return a.ctypes.data_as(_FP)


def knn_c(ref, query, k, threads: int = 1):
    """C restatement of the reference knn_c; (dist float32, index int32), (k, Q)."""
    ref, query, dim, ref_nb, query_nb = _prep(ref, query, k)
    dist = np.empty((k, query_nb), np.float32)
    idx = np.empty((k, query_nb), np.int32)
    ok = _load_oracle().oracle_knn_c(_fp(ref), ref_nb, _fp(query), query_nb, dim, k,
                                     _fp(dist), idx.ctypes.data_as(_IP), threads)
    if not ok:
        raise RuntimeError("oracle_knn_c failed")
    return dist, idx


def knn_f64(ref, query, k, threads: int = 1):
    """FP64 brute force; (dist float64, index int32), (k, Q), (dist, index) order."""
    ref, query, dim, ref_nb, query_nb = _prep(ref, query, k)
    dist = np.empty((k, query_nb), np.float64)
    idx = np.empty((k, query_nb), np.int32)
    ok = _load_oracle().oracle_knn_f64(_fp(ref), ref_nb, _fp(query), query_nb, dim, k,
                                       dist.ctypes.data_as(_DP), idx.ctypes.data_as(_IP),
                                       threads)
    if not ok:
        raise RuntimeError("oracle_knn_f64 failed")
    return dist, idx


def ref_knn_c(ref, query, k, threads: int = 1):
    """The reference's own knn_c (code/test.cpp:129-175), optionally over query slices."""
    ref, query, dim, ref_nb, query_nb = _prep(ref, query, k)
    dist = np.empty((k, query_nb), np.float32)
    idx = np.empty((k, query_nb), np.int32)
    lib = _load_ref()
    if threads <= 1:
        ok = lib.ref_knn_c(_fp(ref), ref_nb, _fp(query), query_nb, dim, k, _fp(dist),
                           idx.ctypes.data_as(_IP))
    else:
        ok = lib.ref_knn_c_mt(_fp(ref), ref_nb, _fp(query), query_nb, dim, k, _fp(dist),
                              idx.ctypes.data_as(_IP), threads)
    if not ok:
        raise RuntimeError("reference knn_c failed")
    return dist, idx


def reference_criterion(dist, idx, gt_dist, gt_idx, precision=1e-3, min_accuracy=0.999):
    """The reference harness's pass rule (code/test.cpp:216-217, :256-272):
    |dist - gt| <= 1e-3 absolute and index == gt index, position by position,
    each for at least 99.9% of the k*Q entries.  Returns (passed, dist_acc, idx_acc)."""
    n = dist.size
    dacc = float(np.count_nonzero(np.abs(dist.astype(np.float64) - gt_dist) <= precision)) / n
    iacc = float(np.count_nonzero(idx == gt_idx)) / n
    return (dacc >= min_accuracy and iacc >= min_accuracy), dacc, iacc
