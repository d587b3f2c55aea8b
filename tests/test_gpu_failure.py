"""Failure detection without a GPU fault: a bounded device wait that nothing completes expires and
reports Q1_ERR_DEVICE_TIMEOUT with the context still usable; host-side injected faults (a CPU
worker that raises, device and pinned allocations that fail) surface as status codes and the next
call succeeds with the same results as before."""
import ctypes

import numpy as np
import pytest
import torch

import tpchq01_gpu_b200 as q
from tpchq01_gpu_b200 import _lib

ROWS = 2_000_003
SEED = 808


def test_inject_fault_argument_checks():
    L = q.lib()
    assert L.q1_inject_fault(0, 0) == 0
    assert L.q1_inject_fault(99, 1) == 1
    assert L.q1_selftest_wait_timeout(0, None) == 1


@pytest.fixture(autouse=True)
def clear_faults():
    yield
    q.lib().q1_inject_fault(0, 0)


@pytest.mark.gpu
def test_device_wait_expires_and_context_survives(cuda):
    stream = torch.cuda.current_stream().cuda_stream
    L = q.lib()
    _lib.check(L.q1_selftest_wait_timeout(20_000, ctypes.c_void_p(stream)))   # 20 ms
    st = L.q1_sync_check(ctypes.c_void_p(stream))
    assert st == 7, L.q1_last_error()
    assert L.q1_sync_check(ctypes.c_void_p(stream)) == 0          # the status word was cleared
    with q.Q1Context() as ctx:                                      # the context still works
        ctx.generate(SEED, ROWS, layout="compressed", packing="pair")
        r = ctx.run(apply_compression=True, num_query_execution_runs=1)
        assert sum(int(g["count"]) for g in r.groups) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("pushdown", [False, True])
def test_cpu_worker_fault_is_reported_and_next_run_is_exact(cuda, pushdown):
    with q.Q1Context(cpu_threads=3) as ctx:
        ctx.generate(SEED, ROWS, layout="compressed", packing="pair", residency="pinned")
        kw = dict(apply_compression=True, use_coprocessing=True, cpu_processing_fraction=0.3,
                  use_filter_pushdown=pushdown, num_query_execution_runs=1, num_tuples_per_kernel_launch=1 << 18)
        clean = ctx.run(**kw).table()
        _lib.check(q.lib().q1_inject_fault(1, 1))
        with pytest.raises(q.Q1Error) as e:
            ctx.run(**kw)
        assert e.value.status == 9 and "injected" in str(e.value)
        assert np.array_equal(ctx.run(**kw).table(), clean)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,residency", [(2, "hbm"), (3, "pinned")])
def test_allocation_faults_are_reported_and_recoverable(cuda, kind, residency):
    with q.Q1Context() as ctx:
        _lib.check(q.lib().q1_inject_fault(kind, 1))
        with pytest.raises(q.Q1Error) as e:
            ctx.generate(SEED, ROWS, layout="compressed", packing="pair", residency=residency)
        assert e.value.status == 3
        ctx.generate(SEED, ROWS, layout="compressed", packing="pair", residency=residency)
        r = ctx.run(apply_compression=True, num_query_execution_runs=1)
        with q.Q1Context() as ref:
            ref.generate(SEED, ROWS, layout="compressed", packing="pair", residency=residency)
            assert np.array_equal(r.table(), ref.run(apply_compression=True, num_query_execution_runs=1).table())
