"""CPU tests of the C-ABI boundary: the library loads, exports every symbol the
headers declare (including the reference's C++-mangled names), and validates
arguments with the reference's bool / "ERROR: ..." contract.  No kernel runs."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available

INCLUDE = os.path.join(ROOT, "include")


def declared_c_functions():
    src = open(os.path.join(INCLUDE, "knn_b200.h")).read()
    return sorted(set(re.findall(r"KNNB200_API\s+[\w\s\*]+?\b(knnb200_\w+)\s*\(", src)))


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_every_declared_symbol_is_exported(knncuda):
    syms = exported_symbols(knncuda.LIB_PATH)
    declared = declared_c_functions()
    assert len(declared) >= 10
    missing = [s for s in declared if s not in syms]
    assert not missing, missing
    for s in knncuda.CXX_SYMBOLS:
        assert s in syms, s
    # and the Python mirror binds exactly what the header declares
    assert set(declared) == set(knncuda.C_SYMBOLS)


def test_cxx_header_matches_reference_signatures():
    """The drop-in header declares the reference's three functions with the
    reference's parameter lists (code/knncuda.h:14-21, :37-44, :61-68)."""
    src = open(os.path.join(INCLUDE, "knncuda.h")).read()
    for name in ("knn_cuda_global", "knn_cuda_texture", "knn_cublas"):
        m = re.search(r"bool\s+" + name + r"\s*\(([^)]*)\)", src)
        assert m, name
        params = [p.strip() for p in m.group(1).replace("\n", " ").split(",")]
        types = [re.sub(r"\s+", " ", re.sub(r"\w+$", "", p)).strip() for p in params]
        assert types == ["const float *", "int", "const float *", "int", "int", "int",
                         "float *", "int *"], types


def test_mangled_names_link_from_cpp(tmp_path, knncuda):
    """A C++ program written against the reference header links unchanged."""
    prog = tmp_path / "user.cpp"
    prog.write_text('#include "knncuda.h"\n'
                    'int main() { bool (*f[3])(const float*, int, const float*, int, int, int,'
                    ' float*, int*) = {knn_cuda_global, knn_cuda_texture, knn_cublas};'
                    ' return f[0] == 0; }\n')
    lib_dir = os.path.dirname(knncuda.LIB_PATH)
    subprocess.run(["g++", str(prog), "-I", INCLUDE, "-L", lib_dir, "-lknnb200",
                    "-Wl,-rpath," + lib_dir, "-o", str(tmp_path / "user")], check=True)


def test_version_and_status_strings(knncuda):
    assert "sm_100a" in knncuda.version()
    assert knncuda.status_string(0) == "ok"
    assert knncuda.status_string(5) == "device wait timed out"


@pytest.mark.parametrize("args", [
    dict(ref_nb=10, query_nb=3, dim=2, k=0),
    dict(ref_nb=10, query_nb=3, dim=2, k=11),     # k > ref_nb (reference leaves this to callers)
    dict(ref_nb=0, query_nb=3, dim=2, k=1),
    dict(ref_nb=10, query_nb=0, dim=2, k=1),
    dict(ref_nb=10, query_nb=3, dim=0, k=1),
])
def test_invalid_sizes_return_false(knncuda, args):
    ref = np.zeros(max(1, args["dim"] * args["ref_nb"]), np.float32)
    query = np.zeros(max(1, args["dim"] * args["query_nb"]), np.float32)
    out_d = np.zeros(max(1, args["k"] * args["query_nb"]), np.float32)
    out_i = np.zeros(max(1, args["k"] * args["query_nb"]), np.int32)
    for fn in (knncuda.knn_cuda_global, knncuda.knn_cuda_texture, knncuda.knn_cublas):
        assert fn(ref, args["ref_nb"], query, args["query_nb"], args["dim"], args["k"],
                  out_d, out_i) is False


def test_null_pointers_return_false(knncuda):
    L = knncuda.lib()
    assert L.knnb200_cuda_global(None, 4, None, 4, 1, 1, None, None) == 0
    assert L.knnb200_knn_device(None, 4, 4, None, 4, 4, 1, 1, 0, None, None, 4, None) == 1


def test_device_entry_rejects_bad_pitch(knncuda):
    L = knncuda.lib()
    p = ctypes.c_void_p(256)   # never dereferenced: validation fails first
    # ref_ld not a multiple of 4
    assert L.knnb200_knn_device(p, 10, 10, p, 4, 4, 3, 2, 0, p, p, 4, None) == 1
    # out_ld < query_nb
    assert L.knnb200_knn_device(p, 10, 12, p, 8, 8, 3, 2, 0, p, p, 4, None) == 1
    # unknown method
    assert L.knnb200_knn_device(p, 10, 12, p, 8, 8, 3, 2, 9, p, p, 8, None) == 1


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_no_device_reports_error(knncuda, capfd):
    ref = np.zeros((2, 10), np.float32)
    query = np.zeros((2, 3), np.float32)
    d = np.zeros((2, 3), np.float32)
    i = np.zeros((2, 3), np.int32)
    assert knncuda.knn_cuda_global(ref, 10, query, 3, 2, 2, d, i) is False
    assert "ERROR: No CUDA device found" in capfd.readouterr().out


def test_scratch_and_split_plan_are_consistent(knncuda):
    # the exact path's scratch: the (q, q)-duplicated query copy (d rows of
    # Q rounded up to 32 pairs) + 256 B, plus splits * Q * k 8-byte keys when
    # the reference set is split
    for n, q, d, k in [(16384, 4096, 128, 16), (1 << 20, 16384, 256, 100), (1000, 5000, 8, 4)]:
        s = knncuda.plan_splits(n, q, d, k)
        assert s >= 1
        b = knncuda.scratch_bytes(n, q, d, k)
        dup = d * ((q + 31) // 32 * 32) * 8
        assert b == dup + 256 + (s * q * k * 8 if s > 1 else 0)
    # k > 256 runs in passes of 256 ranks: per-split lists of one pass plus
    # one lower-bound key per query
    for n, q, d, k in [(20000, 40, 64, 1000), (200000, 8, 16, 600), (3000, 30, 8, 3000)]:
        s = knncuda.plan_splits(n, q, d, k)
        b = knncuda.scratch_bytes(n, q, d, k)
        dup = d * ((q + 31) // 32 * 32) * 8
        assert b == dup + 256 + (s * q * 256 * 8 if s > 1 else 0) + q * 8
