"""ctypes binding of the native library libq1.so (C ABI in include/q1.h).

The library is built in-tree (tpchq01_gpu_b200/libq1.so, by __graft_entry__.build() or
`make -C tpchq01_gpu_b200`). There is no fallback: if the library is missing every entry point
raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libq1.so")

NUM_GROUPS = 6
NUM_AGGS = 6

# q1_status
OK = 0
STATUS_NAMES = {
    0: "Q1_OK", 1: "Q1_ERR_INVALID_ARGUMENT", 2: "Q1_ERR_CUDA", 3: "Q1_ERR_OUT_OF_MEMORY",
    4: "Q1_ERR_NOT_LOADED", 5: "Q1_ERR_UNSUPPORTED", 6: "Q1_ERR_DOMAIN", 7: "Q1_ERR_DEVICE_TIMEOUT",
    8: "Q1_ERR_BUSY", 9: "Q1_ERR_CPU_WORKER", 10: "Q1_ERR_INTERNAL",
}

PLACEMENTS = ["in_registers", "in_registers_per_thread", "local_mem", "shared_mem_per_thread", "global"]
LAYOUT_UNCOMPRESSED, LAYOUT_COMPRESSED = 0, 1
FLAGS_PAIR_2BIT, FLAGS_SEPARATE = 0, 1
RESIDENCY_HBM, RESIDENCY_PINNED_HOST = 0, 1


class Q1Error(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


vp = ctypes.c_void_p


class Columns(ctypes.Structure):
    _fields_ = [("shipdate", vp), ("discount", vp), ("extendedprice", vp), ("tax", vp), ("quantity", vp),
                ("returnflag", vp), ("linestatus", vp)]


class CompressedColumns(ctypes.Structure):
    _fields_ = [("shipdate", vp), ("discount", vp), ("extendedprice", vp), ("tax", vp), ("quantity", vp),
                ("flags", vp), ("returnflag", vp), ("linestatus", vp), ("filter", vp),
                ("flag_packing", ctypes.c_int32), ("num_pair_codes", ctypes.c_uint32),
                ("pair_group", ctypes.c_uint8 * 4)]


class ColumnStats(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint64), ("min_shipdate", ctypes.c_int32), ("max_shipdate", ctypes.c_int32),
                ("max_quantity", ctypes.c_uint32), ("max_discount", ctypes.c_uint32), ("max_tax", ctypes.c_uint32),
                ("max_extendedprice", ctypes.c_uint32), ("num_pair_codes", ctypes.c_uint32),
                ("pair_group", ctypes.c_uint8 * 4), ("group_present_mask", ctypes.c_uint32)]


class CompressedHostOut(ctypes.Structure):
    _fields_ = [("shipdate", vp), ("discount", vp), ("extendedprice", vp), ("tax", vp), ("quantity", vp),
                ("flags", vp), ("returnflag", vp), ("linestatus", vp)]


class I128(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_uint64), ("hi", ctypes.c_uint64)]

    def value(self):
        v = self.lo | (self.hi << 64)
        return v - (1 << 128) if v >= (1 << 127) else v


class GroupResult(ctypes.Structure):
    _fields_ = [("group", ctypes.c_int32), ("returnflag", ctypes.c_char), ("linestatus", ctypes.c_char),
                ("count", ctypes.c_uint64), ("sum_qty", I128), ("sum_base_price", I128), ("sum_disc", I128),
                ("sum_disc_price", I128), ("sum_charge", I128), ("avg_qty_e4", ctypes.c_int64),
                ("avg_price_e4", ctypes.c_int64), ("avg_disc_e4", ctypes.c_int64)]


class Result(ctypes.Structure):
    _fields_ = [("num_groups", ctypes.c_uint32), ("groups", GroupResult * NUM_GROUPS), ("rows_total", ctypes.c_uint64),
                ("rows_gpu", ctypes.c_uint64), ("rows_cpu", ctypes.c_uint64), ("ms_last_run", ctypes.c_double),
                ("ms_gpu_last_run", ctypes.c_double)]


class DeviceOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("cpu_threads", ctypes.c_int32)]


class Params(ctypes.Structure):
    _fields_ = [("placement", ctypes.c_int32), ("apply_compression", ctypes.c_int32),
                ("use_filter_pushdown", ctypes.c_int32), ("use_coprocessing", ctypes.c_int32),
                ("cpu_fraction", ctypes.c_double), ("streams", ctypes.c_int32),
                ("threads_per_block", ctypes.c_int32), ("tuples_per_thread", ctypes.c_int32),
                ("tuples_per_launch", ctypes.c_int64), ("runs", ctypes.c_int32), ("cutoff_day", ctypes.c_int32)]


class LaunchConfig(ctypes.Structure):
    _fields_ = [("threads_per_block", ctypes.c_int32), ("tuples_per_thread", ctypes.c_int32),
                ("blocks", ctypes.c_int32)]


class BatchInstance(ctypes.Structure):
    _fields_ = [("cols", CompressedColumns), ("keys", vp), ("rows", ctypes.c_uint64), ("cutoff_day", ctypes.c_int32),
                ("num_groups", ctypes.c_uint32), ("aggregates", vp)]


class BatchOpts(ctypes.Structure):
    _fields_ = [("use_graph", ctypes.c_int32), ("accumulate", ctypes.c_int32), ("chunk_tiles", ctypes.c_int32),
                ("tune", ctypes.c_int32), ("tune_cache", ctypes.c_char_p)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("instances", ctypes.c_uint32), ("items", ctypes.c_uint32), ("chunk_tiles", ctypes.c_uint32),
                ("tile_rows", ctypes.c_uint32), ("grid", ctypes.c_uint32), ("uses_graph", ctypes.c_uint32),
                ("tuned_classes", ctypes.c_uint32), ("mode_count", ctypes.c_uint32 * 3),
                ("total_rows", ctypes.c_uint64), ("total_groups", ctypes.c_uint64)]


class ColumnsOut(ctypes.Structure):
    _fields_ = [("shipdate", vp), ("returnflag", vp), ("linestatus", vp), ("discount", vp), ("tax", vp),
                ("extendedprice", vp), ("quantity", vp)]


SERVE_MAX_GROUPS = 64
SERVE_RESIDENT_KEY_GROUPS = 64
REQ_RESIDENT, REQ_ADHOC = 0, 1
GROUP_FLAGS, GROUP_KEYS = 0, 1
SERVE_BATCHED, SERVE_PLAIN = 0, 1


class Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("grouping", ctypes.c_int32), ("num_groups", ctypes.c_uint32),
                ("cutoff_day", ctypes.c_int32), ("adhoc_rows", ctypes.c_uint64), ("adhoc_seed", ctypes.c_uint64)]


class Response(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("status", ctypes.c_int32), ("num_groups", ctypes.c_uint32),
                ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("aggregates", I128 * (SERVE_MAX_GROUPS * 6))]


class ServerOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("max_inflight", ctypes.c_uint32), ("mode", ctypes.c_int32),
                ("max_rounds_in_flight", ctypes.c_uint32), ("seed", ctypes.c_uint64),
                ("resident_rows", ctypes.c_uint64), ("hbm_budget_bytes", ctypes.c_uint64),
                ("max_adhoc_rows", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("rounds", ctypes.c_uint64),
                ("pending", ctypes.c_uint64), ("logical_rows", ctypes.c_uint64), ("scanned_rows", ctypes.c_uint64),
                ("generated_rows", ctypes.c_uint64), ("cache_hits", ctypes.c_uint64), ("cache_misses", ctypes.c_uint64),
                ("evictions", ctypes.c_uint64), ("cached_tables", ctypes.c_uint64), ("cached_bytes", ctypes.c_uint64),
                ("wall_ms", ctypes.c_double), ("mean_round_size", ctypes.c_double), ("p50_ms", ctypes.c_double),
                ("p90_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("overlapped_rounds", ctypes.c_uint64),
                ("max_rounds_in_flight", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


# name -> (restype, argtypes); every symbol declared in include/q1.h
SIGNATURES = {
    "q1_last_error": (ctypes.c_char_p, []),
    "q1_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "q1_placement_from_name": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "q1_placement_name": (ctypes.c_char_p, [ctypes.c_int]),
    "q1_compress_host": (ctypes.c_int, [ctypes.POINTER(Columns), ctypes.c_uint64, ctypes.c_int,
                                        ctypes.POINTER(CompressedHostOut), ctypes.POINTER(ColumnStats)]),
    "q1_precompute_filter_host": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int32, vp]),
    "q1_finalize_groups": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.POINTER(GroupResult)]),
    "q1_open": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.POINTER(DeviceOpts)]),
    "q1_close": (ctypes.c_int, [vp]),
    "q1_load_columns": (ctypes.c_int, [vp, ctypes.POINTER(Columns), ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int]),
    "q1_load_compressed": (ctypes.c_int, [vp, ctypes.POINTER(CompressedColumns), ctypes.c_uint64, ctypes.c_int]),
    "q1_generate_table": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int]),
    "q1_params_default": (None, [ctypes.POINTER(Params)]),
    "q1_params_validate": (ctypes.c_int, [ctypes.POINTER(Params)]),
    "q1_table_columns": (ctypes.c_int, [vp, ctypes.POINTER(CompressedColumns), ctypes.POINTER(Columns),
                                        ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]),
    "q1_table_stats": (ctypes.c_int, [vp, ctypes.POINTER(ColumnStats)]),
    "q1_run_times": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                    ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "q1_run": (ctypes.c_int, [vp, ctypes.POINTER(Params), ctypes.POINTER(Result)]),
    "q1_launch_compressed": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(CompressedColumns), ctypes.c_uint64,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(LaunchConfig), vp, vp]),
    "q1_launch_uncompressed": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Columns), ctypes.c_uint64, ctypes.c_int32,
                                              ctypes.POINTER(LaunchConfig), vp, vp]),
    "q1_launch_compressed_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(CompressedColumns), ctypes.c_uint64,
                                                    ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(LaunchConfig), vp,
                                                    vp]),
    "q1_sync_check": (ctypes.c_int, [vp]),
    "q1_groupkey_scratch_bytes": (ctypes.c_uint64, [ctypes.c_uint32]),
    "q1_launch_groupkey": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(CompressedColumns), vp, ctypes.c_uint32,
                                          ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(LaunchConfig), vp, vp, vp]),
    "q1_zipf_cdf": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_double, vp]),
    "q1_generate_group_keys_device": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                                     ctypes.c_uint32, vp, vp, vp]),
    "q1_precompute_filter": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int32, vp, vp]),
    "q1_generate_host": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(Columns)]),
    "q1_generate_compressed_device": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                                     ctypes.POINTER(CompressedHostOut), vp]),
    "q1_device_describe": (ctypes.c_int, [ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t]),
    "q1_measure_host_read": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "q1_batch_create": (ctypes.c_int, [ctypes.POINTER(BatchInstance), ctypes.c_uint32, ctypes.POINTER(BatchOpts), vp,
                                       ctypes.POINTER(vp)]),
    "q1_batch_run": (ctypes.c_int, [vp, vp]),
    "q1_batch_describe": (ctypes.c_int, [vp, ctypes.POINTER(BatchDesc)]),
    "q1_batch_instance_mode": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32)]),
    "q1_batch_destroy": (ctypes.c_int, [vp]),
    "q1_server_opts_default": (None, [ctypes.POINTER(ServerOpts)]),
    "q1_server_open": (ctypes.c_int, [ctypes.POINTER(ServerOpts), ctypes.POINTER(vp)]),
    "q1_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]),
    "q1_server_wait": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(Response)]),
    "q1_server_stats_get": (ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
    "q1_server_reset_stats": (ctypes.c_int, [vp]),
    "q1_server_plain": (ctypes.c_int, [vp, ctypes.POINTER(Request), ctypes.POINTER(Response)]),
    "q1_server_resident_columns": (ctypes.c_int, [vp, ctypes.POINTER(CompressedColumns), ctypes.POINTER(vp),
                                                  ctypes.POINTER(ctypes.c_uint64)]),
    "q1_server_close": (ctypes.c_int, [vp]),
    "q1_cache_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Columns), ctypes.c_uint64]),
    "q1_cache_rows": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)]),
    "q1_cache_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ColumnsOut)]),
    "q1_cache_load": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_uint64)]),
    "q1_tbl_count_device": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), vp]),
    "q1_tbl_parse_device": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(ColumnsOut), ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_uint64), vp]),
    "q1_tbl_read_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ColumnsOut), ctypes.c_uint64,
                                        ctypes.POINTER(ctypes.c_uint64)]),
    "q1_tbl_load": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_uint64)]),
    "q1_tbl_format": (ctypes.c_int, [ctypes.POINTER(Columns), ctypes.c_uint64, ctypes.c_uint64, vp, ctypes.c_uint64,
                                     ctypes.POINTER(ctypes.c_uint64)]),
    "q1_inject_fault": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint32]),
    "q1_selftest_wait_timeout": (ctypes.c_int, [ctypes.c_uint32, vp]),
    "q1_selftest_cpu_share": (ctypes.c_int, [ctypes.POINTER(CompressedColumns), ctypes.c_uint64, ctypes.c_uint64,
                                             ctypes.c_int32, vp]),
    "q1_selftest_cpu_share_uncompressed": (ctypes.c_int, [ctypes.POINTER(Columns), ctypes.c_uint64, ctypes.c_uint64,
                                                          ctypes.c_int32, vp]),
    "q1_version": (ctypes.c_char_p, []),
}

_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"native library missing: {LIB_PATH}; build it with __graft_entry__.build() "
                               f"or `make -C tpchq01_gpu_b200` (there is no fallback implementation)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != OK:
        msg = lib().q1_last_error().decode(errors="replace")
        raise Q1Error(status, msg)
    return status
