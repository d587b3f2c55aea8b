"""The C ABI library loads and exports every function include/q1.h declares (no GPU calls)."""
import ctypes
import os
import re

import tpchq01_gpu_b200 as q
from tpchq01_gpu_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "q1.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(q1_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 25
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_version_and_status_strings():
    assert b"sm_100a" in q.lib().q1_version()
    assert q.lib().q1_status_string(6) == b"Q1_ERR_DOMAIN"


def test_library_links_the_cuda_runtime_statically():
    # no libcudart.so dependency, so the in-tree library runs wherever a driver is present
    import subprocess
    deps = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "libcudart.so" not in deps


def test_groupkey_scratch_sizes_follow_the_header():
    """q1_groupkey_scratch_bytes: 64 bytes a group, plus a 256-byte word block for the on-device
    path choice above 256 groups, plus the partition workspace (about 1.1 GB, independent of the
    row count) above 4096 groups."""
    f = q.lib().q1_groupkey_scratch_bytes
    for g in [1, 4, 64, 256]:
        assert f(g) == 64 * g
    for g in [257, 1024, 1025, 4096]:
        assert f(g) == ((64 * g + 255) // 256) * 256 + 256
    base = f(4097) - ((64 * 4097 + 255) // 256) * 256
    assert 0.9e9 < base < 1.3e9
    assert f(65536) - ((64 * 65536 + 255) // 256) * 256 == base


def test_host_read_probe():
    """q1_measure_host_read reads a host buffer on several threads and reports a positive rate;
    bad arguments are rejected."""
    import ctypes
    import numpy as np
    from tpchq01_gpu_b200 import _lib
    L = q.lib()
    buf = np.ones(64 << 20, dtype=np.uint8)
    g = ctypes.c_double()
    assert L.q1_measure_host_read(buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes, 2, ctypes.byref(g)) == 0
    assert g.value > 0.1
    assert L.q1_measure_host_read(buf.ctypes.data_as(ctypes.c_void_p), 100, 2, ctypes.byref(g)) == 1
    assert L.q1_measure_host_read(None, buf.nbytes, 2, ctypes.byref(g)) == 1
