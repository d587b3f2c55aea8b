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
