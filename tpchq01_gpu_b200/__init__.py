"""B200-native (sm_100a) TPC-H Query 1 filter + group-by aggregation.

The compute path is native: CUDA kernels and a C++ runtime in libq1.so behind the C ABI of
include/q1.h. This package only binds it (ctypes) and mirrors the reference's operator surface.
"""
from ._lib import Q1Error, lib  # noqa: F401
from .api import (AGG_NAMES, Q1Context, Q1Params, Q1Result, compress_host, decode_aggregates,  # noqa: F401
                  generate_host, launch_compressed, launch_uncompressed, placement_id, precompute_filter,
                  precompute_filter_host, sync_check, tbl_format, tbl_read_file)

__version__ = "1.0.0"
