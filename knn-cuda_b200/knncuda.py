"""Python mirror of the reference interface (code/knncuda.h) over libknnb200.so.

The three functions keep the reference's names, argument order and meaning
and its error behaviour (a bool result; "ERROR: ..." printed by the library
on failure):

    knn_cuda_global(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) -> bool
    knn_cuda_texture(...) -> bool
    knn_cublas(...) -> bool

``ref`` / ``query`` are float32 arrays holding dim x n row-major points
(``x[d, i]``, README.md "Data storage"); ``knn_dist`` (float32) and
``knn_index`` (int32) are preallocated k x query_nb outputs, filled in place.

``knn_device`` is the device-resident path (torch CUDA tensors, no host
copies, asynchronous on the given stream).

There is no CPU fallback: if libknnb200.so is missing, importing the
library raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libknnb200.so")

METHOD_GLOBAL = 0
METHOD_TEXTURE = 1
METHOD_CUBLAS = 2
METHOD_FP8 = 3
METHODS = {"global": METHOD_GLOBAL, "texture": METHOD_TEXTURE, "cublas": METHOD_CUBLAS,
           "fp8": METHOD_FP8}
TC_KINDS = {-1: None, 0: "bf16", 1: "bf16x3", 2: "fp8"}

_FP = ctypes.POINTER(ctypes.c_float)
_IP = ctypes.POINTER(ctypes.c_int)
_lib = None

# Every extern "C" symbol of include/knn_b200.h and the three C++-linkage
# symbols of include/knncuda.h.
C_SYMBOLS = (
    "knnb200_cuda_global", "knnb200_cuda_texture", "knnb200_cublas", "knnb200_knn_device",
    "knnb200_sync_status", "knnb200_scratch_bytes", "knnb200_plan_splits",
    "knnb200_release_workspace", "knnb200_status_string", "knnb200_version",
    "knnb200_measure_fp32_peak", "knnb200_last_tc_stats", "knnb200_selftest_wait_timeout",
    "knnb200_knn_device_noalloc", "knnb200_set_phase_timing", "knnb200_last_phase_times",
    "knnb200_refset_create", "knnb200_refset_destroy", "knnb200_refset_device_bytes",
    "knnb200_refset_knn", "knnb200_server_create", "knnb200_server_submit",
    "knnb200_server_wait", "knnb200_server_stats", "knnb200_server_destroy",
    "knnb200_batched_plan_create", "knnb200_batched_run", "knnb200_batched_status",
    "knnb200_batched_items", "knnb200_batched_plan_destroy", "knnb200_batched_graph_create",
    "knnb200_graph_launch", "knnb200_graph_destroy", "knnb200_batched_autotune",
    "knnb200_set_bound_check", "knnb200_last_bound_check", "knnb200_set_memory_cap",
    "knnb200_last_query_chunks", "knnb200_call_bytes", "knnb200_last_tc_kinds",
    "knnb200_batched_plan_create_config", "knnb200_batched_plan_config",
    "knnb200_batched_autotune_config", "knnb200_set_tc_kind_override",
)


class BatchedConfig(ctypes.Structure):
    """Mirror of knnb200_batched_config (include/knn_b200.h)."""
    _fields_ = [("item_stages", ctypes.c_int), ("queries_per_warp", ctypes.c_int),
                ("lowdim_kernel", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {"item_stages": self.item_stages, "queries_per_warp": self.queries_per_warp,
                "lowdim_kernel": self.lowdim_kernel}


class Problem(ctypes.Structure):
    """Mirror of knnb200_problem (include/knn_b200.h)."""
    _fields_ = [("ref", ctypes.c_void_p), ("ref_nb", ctypes.c_int), ("ref_ld", ctypes.c_longlong),
                ("query", ctypes.c_void_p), ("query_nb", ctypes.c_int),
                ("query_ld", ctypes.c_longlong), ("dim", ctypes.c_int), ("k", ctypes.c_int),
                ("knn_dist", ctypes.c_void_p), ("knn_index", ctypes.c_void_p),
                ("out_ld", ctypes.c_longlong)]
PHASES = ("tc_prep_ref", "tc_prep_query", "tc_pass1", "tc_threshold", "tc_pass2", "tc_rerank",
          "tc_fallback", "exact_main", "exact_merge", "tc_retry_scan", "tc_retry_rerank")
CXX_SYMBOLS = (
    "_Z15knn_cuda_globalPKfiS0_iiiPfPi",
    "_Z16knn_cuda_texturePKfiS0_iiiPfPi",
    "_Z10knn_cublasPKfiS0_iiiPfPi",
)


def lib():
    """Load libknnb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libknnb200.so not built ({LIB_PATH}); run make -C knn-cuda_b200")
        L = ctypes.CDLL(LIB_PATH)
        host_args = [_FP, ctypes.c_int, _FP, ctypes.c_int, ctypes.c_int, ctypes.c_int, _FP, _IP]
        for name in ("knnb200_cuda_global", "knnb200_cuda_texture", "knnb200_cublas"):
            fn = getattr(L, name)
            fn.restype = ctypes.c_int
            fn.argtypes = host_args
        L.knnb200_knn_device.restype = ctypes.c_int
        L.knnb200_knn_device.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p]
        L.knnb200_sync_status.restype = ctypes.c_int
        L.knnb200_sync_status.argtypes = [ctypes.c_void_p]
        L.knnb200_scratch_bytes.restype = ctypes.c_size_t
        L.knnb200_scratch_bytes.argtypes = [ctypes.c_int] * 5
        L.knnb200_plan_splits.restype = ctypes.c_int
        L.knnb200_plan_splits.argtypes = [ctypes.c_int] * 4
        L.knnb200_release_workspace.restype = None
        L.knnb200_release_workspace.argtypes = []
        L.knnb200_status_string.restype = ctypes.c_char_p
        L.knnb200_status_string.argtypes = [ctypes.c_int]
        L.knnb200_measure_fp32_peak.restype = ctypes.c_double
        L.knnb200_measure_fp32_peak.argtypes = [ctypes.c_int, ctypes.c_void_p]
        L.knnb200_selftest_wait_timeout.restype = ctypes.c_int
        L.knnb200_selftest_wait_timeout.argtypes = [ctypes.c_longlong, ctypes.c_void_p]
        L.knnb200_knn_device_noalloc.restype = ctypes.c_int
        L.knnb200_knn_device_noalloc.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_longlong, ctypes.c_void_p]
        L.knnb200_set_phase_timing.restype = None
        L.knnb200_set_phase_timing.argtypes = [ctypes.c_int]
        L.knnb200_last_phase_times.restype = ctypes.c_int
        L.knnb200_last_phase_times.argtypes = [_FP, ctypes.c_int]
        L.knnb200_last_tc_stats.restype = None
        L.knnb200_last_tc_stats.argtypes = [ctypes.POINTER(ctypes.c_longlong), _IP, _IP]
        vp, ll, sz = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_size_t
        L.knnb200_refset_create.restype = ctypes.c_int
        L.knnb200_refset_create.argtypes = [vp, ctypes.c_int, ll, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(vp)]
        L.knnb200_refset_destroy.restype = None
        L.knnb200_refset_destroy.argtypes = [vp]
        L.knnb200_refset_device_bytes.restype = sz
        L.knnb200_refset_device_bytes.argtypes = [vp]
        L.knnb200_refset_knn.restype = ctypes.c_int
        L.knnb200_refset_knn.argtypes = [vp, vp, ctypes.c_int, ll, ctypes.c_int, ctypes.c_int,
                                         vp, vp, ll, vp]
        L.knnb200_server_create.restype = ctypes.c_int
        L.knnb200_server_create.argtypes = [vp, ctypes.c_int, sz, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(vp)]
        L.knnb200_server_submit.restype = ll
        L.knnb200_server_submit.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.knnb200_server_wait.restype = ctypes.c_int
        L.knnb200_server_wait.argtypes = [vp, ll, ctypes.POINTER(ctypes.c_double)]
        dp = ctypes.POINTER(ctypes.c_double)
        L.knnb200_server_stats.restype = ctypes.c_int
        L.knnb200_server_stats.argtypes = [vp, dp, dp, ctypes.POINTER(ll), ctypes.POINTER(ll), dp]
        L.knnb200_server_destroy.restype = None
        L.knnb200_server_destroy.argtypes = [vp]
        PP = ctypes.POINTER(Problem)
        L.knnb200_batched_plan_create.restype = ctypes.c_int
        L.knnb200_batched_plan_create.argtypes = [PP, ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(vp)]
        L.knnb200_batched_run.restype = ctypes.c_int
        L.knnb200_batched_run.argtypes = [vp, vp]
        L.knnb200_batched_status.restype = ctypes.c_int
        L.knnb200_batched_status.argtypes = [vp, vp]
        L.knnb200_batched_items.restype = ll
        L.knnb200_batched_items.argtypes = [vp]
        L.knnb200_batched_plan_destroy.restype = None
        L.knnb200_batched_plan_destroy.argtypes = [vp]
        L.knnb200_batched_graph_create.restype = ctypes.c_int
        L.knnb200_batched_graph_create.argtypes = [vp, ctypes.POINTER(vp)]
        L.knnb200_graph_launch.restype = ctypes.c_int
        L.knnb200_graph_launch.argtypes = [vp, vp]
        L.knnb200_graph_destroy.restype = None
        L.knnb200_graph_destroy.argtypes = [vp]
        L.knnb200_batched_autotune.restype = ctypes.c_int
        L.knnb200_batched_autotune.argtypes = [PP, ctypes.c_int, vp, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_float)]
        L.knnb200_set_bound_check.restype = ctypes.c_int
        L.knnb200_set_bound_check.argtypes = [ctypes.c_int]
        L.knnb200_last_bound_check.restype = ctypes.c_int
        L.knnb200_last_bound_check.argtypes = [ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_longlong)]
        L.knnb200_set_memory_cap.restype = None
        L.knnb200_set_memory_cap.argtypes = [ctypes.c_size_t]
        L.knnb200_last_query_chunks.restype = ctypes.c_int
        L.knnb200_last_query_chunks.argtypes = []
        L.knnb200_set_tc_kind_override.restype = None
        L.knnb200_set_tc_kind_override.argtypes = [ctypes.c_int]
        L.knnb200_last_tc_kinds.restype = None
        L.knnb200_last_tc_kinds.argtypes = [_IP, _IP]
        L.knnb200_call_bytes.restype = ctypes.c_size_t
        L.knnb200_call_bytes.argtypes = [ctypes.c_int] * 6
        CP = ctypes.POINTER(BatchedConfig)
        L.knnb200_batched_plan_create_config.restype = ctypes.c_int
        L.knnb200_batched_plan_create_config.argtypes = [PP, ctypes.c_int, CP,
                                                         ctypes.POINTER(vp)]
        L.knnb200_batched_plan_config.restype = ctypes.c_int
        L.knnb200_batched_plan_config.argtypes = [vp, CP, _IP]
        L.knnb200_batched_autotune_config.restype = ctypes.c_int
        L.knnb200_batched_autotune_config.argtypes = [PP, ctypes.c_int, vp, CP,
                                                      ctypes.POINTER(ctypes.c_float)]
        L.knnb200_version.restype = ctypes.c_char_p
        L.knnb200_version.argtypes = []
        _lib = L
    return _lib


def _check_host(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index):
    for name, a, dt in (("ref", ref, np.float32), ("query", query, np.float32),
                        ("knn_dist", knn_dist, np.float32), ("knn_index", knn_index, np.int32)):
        if not isinstance(a, np.ndarray) or a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
            raise TypeError(f"{name} must be a C-contiguous numpy {np.dtype(dt).name} array")
    if ref.size < dim * ref_nb or query.size < dim * query_nb:
        raise ValueError("ref/query arrays are smaller than dim x n")
    if knn_dist.size < k * query_nb or knn_index.size < k * query_nb:
        raise ValueError("output arrays are smaller than k x query_nb")
    if not knn_dist.flags["WRITEABLE"] or not knn_index.flags["WRITEABLE"]:
        raise ValueError("outputs must be writeable")


def _host_call(name, ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) -> bool:
    if min(ref_nb, query_nb, dim, k) >= 1:
        _check_host(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index)
    fn = getattr(lib(), name)
    p = lambda a, t: a.ctypes.data_as(t) if isinstance(a, np.ndarray) else None
    return bool(fn(p(ref, _FP), ref_nb, p(query, _FP), query_nb, dim, k, p(knn_dist, _FP),
                   p(knn_index, _IP)))


def knn_cuda_global(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) -> bool:
    """Mirror of knn_cuda_global (code/knncuda.h:14-21)."""
    return _host_call("knnb200_cuda_global", ref, ref_nb, query, query_nb, dim, k, knn_dist,
                      knn_index)


def knn_cuda_texture(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) -> bool:
    """Mirror of knn_cuda_texture (code/knncuda.h:37-44)."""
    return _host_call("knnb200_cuda_texture", ref, ref_nb, query, query_nb, dim, k, knn_dist,
                      knn_index)


def knn_cublas(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) -> bool:
    """Mirror of knn_cublas (code/knncuda.h:61-68)."""
    return _host_call("knnb200_cublas", ref, ref_nb, query, query_nb, dim, k, knn_dist,
                      knn_index)


ENTRY_POINTS = {"global": knn_cuda_global, "texture": knn_cuda_texture, "cublas": knn_cublas}


def knn(ref: np.ndarray, query: np.ndarray, k: int, method: str = "global"):
    """Convenience wrapper: returns (dist, index), each k x query_nb."""
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    query = np.ascontiguousarray(query, dtype=np.float32)
    dim, ref_nb = ref.shape
    query_nb = query.shape[1]
    dist = np.empty((k, query_nb), np.float32)
    idx = np.empty((k, query_nb), np.int32)
    if not ENTRY_POINTS[method](ref, ref_nb, query, query_nb, dim, k, dist, idx):
        raise RuntimeError(f"knn_{method} failed")
    return dist, idx


def knn_device(ref, query, k: int, method: str = "global", dist=None, index=None,
               stream=None):
    """Device-resident k-NN on torch CUDA tensors shaped (dim, n).

    ``ref`` / ``query`` may be row-pitched views (stride(1) == 1, stride(0) a
    multiple of 4).  Returns (dist, index) tensors of shape (k, query_nb);
    queued on ``stream`` (default: torch's current stream), not synchronised.
    """
    import torch

    dim, ref_nb = ref.shape
    query_nb = query.shape[1]
    if ref.dtype != torch.float32 or query.dtype != torch.float32:
        raise TypeError("ref/query must be float32")
    if ref.stride(1) != 1 or query.stride(1) != 1:
        raise ValueError("ref/query rows must be contiguous")
    if dist is None:
        dist = torch.empty((k, query_nb), dtype=torch.float32, device=query.device)
    if index is None:
        index = torch.empty((k, query_nb), dtype=torch.int32, device=query.device)
    if stream is None:
        stream = torch.cuda.current_stream(query.device)
    rc = lib().knnb200_knn_device(
        ref.data_ptr(), ref_nb, ref.stride(0), query.data_ptr(), query_nb, query.stride(0),
        dim, k, METHODS[method], dist.data_ptr(), index.data_ptr(), dist.stride(0),
        ctypes.c_void_p(stream.cuda_stream))
    if rc != 0:
        raise RuntimeError(f"knnb200_knn_device failed: {status_string(rc)}")
    return dist, index


class RefSet:
    """A reference set kept resident on the current device (dim x ref_nb)."""

    def __init__(self, ref):
        import torch

        self._h = ctypes.c_void_p()
        if isinstance(ref, np.ndarray):
            ref = np.ascontiguousarray(ref, dtype=np.float32)
            self.dim, self.ref_nb = ref.shape
            rc = lib().knnb200_refset_create(ref.ctypes.data, self.ref_nb, self.ref_nb, self.dim,
                                             0, ctypes.byref(self._h))
        else:
            if ref.dtype != torch.float32 or ref.stride(1) != 1:
                raise TypeError("ref must be a float32 tensor with contiguous rows")
            self.dim, self.ref_nb = ref.shape
            rc = lib().knnb200_refset_create(ref.data_ptr(), self.ref_nb, ref.stride(0), self.dim,
                                             1, ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"knnb200_refset_create failed: {status_string(rc)}")

    @property
    def handle(self):
        return self._h

    def device_bytes(self) -> int:
        return lib().knnb200_refset_device_bytes(self._h)

    def knn(self, query, k: int, method: str = "global", dist=None, index=None, stream=None):
        """k-NN of a device tensor of queries (dim x query_nb); synchronises."""
        import torch

        query_nb = query.shape[1]
        if dist is None:
            dist = torch.empty((k, query_nb), dtype=torch.float32, device=query.device)
        if index is None:
            index = torch.empty((k, query_nb), dtype=torch.int32, device=query.device)
        if stream is None:
            stream = torch.cuda.current_stream(query.device)
        rc = lib().knnb200_refset_knn(self._h, query.data_ptr(), query_nb, query.stride(0), k,
                                      METHODS[method], dist.data_ptr(), index.data_ptr(),
                                      dist.stride(0), ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"knnb200_refset_knn failed: {status_string(rc)}")
        return dist, index

    def close(self):
        if self._h:
            lib().knnb200_refset_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching k-NN server over a RefSet (host queries in, host
    results out)."""

    def __init__(self, refset: RefSet, slots: int = 2, memory_budget: int = 8 << 30,
                 max_batch_queries: int = 4096, method: str = "cublas"):
        self.refset = refset
        self._h = ctypes.c_void_p()
        rc = lib().knnb200_server_create(refset.handle, slots, memory_budget, max_batch_queries,
                                         METHODS[method], ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"knnb200_server_create failed: {status_string(rc)}")
        self._bufs = {}

    def submit(self, query: np.ndarray, k: int) -> int:
        query = np.ascontiguousarray(query, dtype=np.float32)
        qn = query.shape[1]
        dist = np.empty((k, qn), np.float32)
        idx = np.empty((k, qn), np.int32)
        t = lib().knnb200_server_submit(self._h, query.ctypes.data, qn, k, dist.ctypes.data,
                                        idx.ctypes.data)
        if t < 0:
            raise RuntimeError(f"knnb200_server_submit failed: {status_string(-t)}")
        self._bufs[t] = (query, dist, idx)
        return t

    def wait(self, ticket: int):
        """(dist, index, latency_ms) of a submitted request."""
        lat = ctypes.c_double(0)
        rc = lib().knnb200_server_wait(self._h, ticket, ctypes.byref(lat))
        _, dist, idx = self._bufs.pop(ticket)
        if rc != 0:
            raise RuntimeError(f"request {ticket} failed: {status_string(rc)}")
        return dist, idx, lat.value

    def stats(self) -> dict:
        p50, p99, w = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
        q, b = ctypes.c_longlong(0), ctypes.c_longlong(0)
        lib().knnb200_server_stats(self._h, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(q),
                                   ctypes.byref(b), ctypes.byref(w))
        return {"p50_ms": p50.value, "p99_ms": p99.value, "queries": q.value,
                "batches": b.value, "wall_s": w.value}

    def close(self):
        if self._h:
            lib().knnb200_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def problems_from(tensors):
    """ctypes array of Problem from [(ref, query, k, dist, index)] torch tensors,
    each (dim, n) with contiguous rows."""
    arr = (Problem * len(tensors))()
    for i, (ref, query, k, dist, index) in enumerate(tensors):
        arr[i] = Problem(ref.data_ptr(), ref.shape[1], ref.stride(0), query.data_ptr(),
                         query.shape[1], query.stride(0), ref.shape[0], k, dist.data_ptr(),
                         index.data_ptr(), dist.stride(0))
    return arr


class BatchedPlan:
    """Many independent exact k-NN problems in one persistent launch.

    ``config`` (a BatchedConfig, e.g. from batched_autotune_config) overrides
    ``item_stages``."""

    def __init__(self, problems, item_stages: int = 0, config=None):
        self._arr = problems
        self._h = ctypes.c_void_p()
        if config is not None:
            rc = lib().knnb200_batched_plan_create_config(problems, len(problems),
                                                          ctypes.byref(config),
                                                          ctypes.byref(self._h))
        else:
            rc = lib().knnb200_batched_plan_create(problems, len(problems), item_stages,
                                                   ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"knnb200_batched_plan_create failed: {status_string(rc)}")
        self._graph = ctypes.c_void_p()

    def items(self) -> int:
        return lib().knnb200_batched_items(self._h)

    def config(self) -> dict:
        """The plan's configuration and how many problems it sends to the
        low-dimension kernel."""
        c, n = BatchedConfig(), ctypes.c_int(0)
        lib().knnb200_batched_plan_config(self._h, ctypes.byref(c), ctypes.byref(n))
        return dict(c.as_dict(), lowdim_problems=n.value)

    def run(self, stream=None):
        import torch

        stream = stream or torch.cuda.current_stream()
        rc = lib().knnb200_batched_run(self._h, ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"knnb200_batched_run failed: {status_string(rc)}")

    def status(self, stream=None) -> int:
        import torch

        stream = stream or torch.cuda.current_stream()
        return lib().knnb200_batched_status(self._h, ctypes.c_void_p(stream.cuda_stream))

    def capture_graph(self):
        rc = lib().knnb200_batched_graph_create(self._h, ctypes.byref(self._graph))
        if rc != 0:
            raise RuntimeError(f"knnb200_batched_graph_create failed: {status_string(rc)}")

    def replay(self, stream=None):
        import torch

        stream = stream or torch.cuda.current_stream()
        rc = lib().knnb200_graph_launch(self._graph, ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"knnb200_graph_launch failed: {status_string(rc)}")

    def close(self):
        if self._graph:
            lib().knnb200_graph_destroy(self._graph)
            self._graph = ctypes.c_void_p()
        if self._h:
            lib().knnb200_batched_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batched_autotune(problems, stream=None):
    """(best item_stages, ms per run) among the tuner's candidates."""
    import torch

    stream = stream or torch.cuda.current_stream()
    best, ms = ctypes.c_int(0), ctypes.c_float(0)
    rc = lib().knnb200_batched_autotune(problems, len(problems),
                                        ctypes.c_void_p(stream.cuda_stream), ctypes.byref(best),
                                        ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"knnb200_batched_autotune failed: {status_string(rc)}")
    return best.value, ms.value


def batched_autotune_config(problems, stream=None):
    """(best BatchedConfig, ms per run) over work-item size, tile shape and
    low-d routing."""
    import torch

    stream = stream or torch.cuda.current_stream()
    best, ms = BatchedConfig(), ctypes.c_float(0)
    rc = lib().knnb200_batched_autotune_config(problems, len(problems),
                                               ctypes.c_void_p(stream.cuda_stream),
                                               ctypes.byref(best), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"knnb200_batched_autotune_config failed: {status_string(rc)}")
    return best, ms.value


def sync_status(stream=None) -> int:
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return lib().knnb200_sync_status(ctypes.c_void_p(stream.cuda_stream))


def status_string(code: int) -> str:
    return lib().knnb200_status_string(code).decode()


def scratch_bytes(ref_nb, query_nb, dim, k, method="global") -> int:
    return lib().knnb200_scratch_bytes(ref_nb, query_nb, dim, k, METHODS[method])


def plan_splits(ref_nb, query_nb, dim, k) -> int:
    return lib().knnb200_plan_splits(ref_nb, query_nb, dim, k)


def selftest_wait_timeout(limit_ns: int = 50_000_000) -> int:
    """Run the bounded-wait self-test (a wait that nothing completes) on the
    current device's default stream; returns the KNNB200_* code
    (KNNB200_ETIMEOUT = 5 expected)."""
    return lib().knnb200_selftest_wait_timeout(int(limit_ns), None)


def measure_fp32_peak(iters: int = 4096, stream=None) -> float:
    """FP32 CUDA-core FLOP/s of the current device (packed-FMA calibration kernel)."""
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return lib().knnb200_measure_fp32_peak(iters, ctypes.c_void_p(stream.cuda_stream))


def set_phase_timing(enable: bool) -> None:
    lib().knnb200_set_phase_timing(1 if enable else 0)


def last_phase_times() -> dict:
    """{phase name: ms} for the phases the last timed call ran."""
    buf = (ctypes.c_float * len(PHASES))()
    lib().knnb200_last_phase_times(buf, len(PHASES))
    return {name: float(v) for name, v in zip(PHASES, buf) if v >= 0}


def last_tc_stats() -> dict:
    """Statistics of the last knn_cublas-method call: first-scan candidates,
    queries given a second tensor scan, queries recomputed by the exact kernel."""
    c, a, b = ctypes.c_longlong(0), ctypes.c_int(0), ctypes.c_int(0)
    lib().knnb200_last_tc_stats(ctypes.byref(c), ctypes.byref(a), ctypes.byref(b))
    return {"candidates": c.value, "second_scan": a.value, "exact": b.value}


def set_bound_check(enable: bool) -> None:
    """Turn the test-only check of the tensor path's error bound on or off."""
    rc = lib().knnb200_set_bound_check(1 if enable else 0)
    if rc != 0:
        raise RuntimeError(f"knnb200_set_bound_check failed: {status_string(rc)}")


def last_bound_check() -> tuple:
    """(max |a + |q|^2 - D| / E_q, candidates checked) of the last tensor-path
    call made while the check was on."""
    r, n = ctypes.c_double(0), ctypes.c_longlong(0)
    rc = lib().knnb200_last_bound_check(ctypes.byref(r), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"knnb200_last_bound_check failed: {status_string(rc)}")
    return r.value, n.value


def set_memory_cap(nbytes: int) -> None:
    """Cap the device memory the library assumes it may use (0 = no cap)."""
    lib().knnb200_set_memory_cap(int(nbytes))


def call_bytes(ref_nb, query_nb, dim, k, method="global", host=True) -> int:
    """The library's device-memory estimate for one call of this shape."""
    return lib().knnb200_call_bytes(ref_nb, query_nb, dim, k, METHODS[method], 1 if host else 0)


def last_query_chunks() -> int:
    """Query chunks the last host or device call ran in."""
    return lib().knnb200_last_query_chunks()


def set_tc_kind_override(kind) -> None:
    """Force the tensor path's pass-2 kind ("bf16", "bf16x3", "fp8") or
    restore the predicted choice (None).  For tests and measurements."""
    code = {None: -1, "bf16": 0, "bf16x3": 1, "fp8": 2}[kind]
    lib().knnb200_set_tc_kind_override(code)


def last_tc_kinds() -> tuple:
    """(first scan kind, second scan kind) of the last tensor-path call, as
    names: "bf16", "bf16x3" (split BF16), "fp8" or None."""
    a, b = ctypes.c_int(0), ctypes.c_int(0)
    lib().knnb200_last_tc_kinds(ctypes.byref(a), ctypes.byref(b))
    return TC_KINDS.get(a.value), TC_KINDS.get(b.value)


def last_fallback_counts() -> tuple:
    """(second_scan, exact) of the last knn_cublas-method call."""
    s = last_tc_stats()
    return s["second_scan"], s["exact"]


def version() -> str:
    return lib().knnb200_version().decode()
