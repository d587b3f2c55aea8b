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
    assert L.q1_inject_fault(4, 0) == 0
    assert L.q1_inject_fault(5, 1) == 1
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


@pytest.mark.gpu
def test_failed_serving_round_fails_what_follows_and_server_reopens(cuda):
    """A serving round that fails (injected on the host while another round lane may be busy)
    fails its own requests, the rounds queued behind it and every request still waiting; the server
    then refuses submissions, closes cleanly, and a new server on the same device answers exactly."""
    from test_gpu_serve import ADHOC, FLAGS, KEYS, RES, open_server, plain, req, submit, words
    L = q.lib()
    h = open_server(slots=4, lanes=2)
    try:
        r0 = req(ADHOC, KEYS, 729999, 9, 300_000, 7)
        ok = _lib.Response()
        assert L.q1_server_wait(h, submit(h, r0), 60_000, ctypes.byref(ok)) == 0
        _lib.check(L.q1_inject_fault(4, 1))   # Q1_FAULT_SERVE_ROUND: the next round fails to enqueue
        reqs = [req(ADHOC, KEYS, 729990 + i, 9, 300_000, 7) if i % 2 else req(RES, FLAGS, 729950 + i)
                for i in range(24)]
        # Once the failed round retires the server refuses submissions (Q1_ERR_INTERNAL); until then
        # it queues them, and every request queued after the failure fails too.
        tickets, refused = [], 0
        for r in reqs:
            t = ctypes.c_uint64()
            st = L.q1_server_submit(h, ctypes.byref(r), ctypes.byref(t))
            if st == 0:
                tickets.append(t.value)
            else:
                assert st == 10, st
                refused += 1
        assert tickets, "the first request after the fault must be queued"
        statuses = []
        for t in tickets:
            resp = _lib.Response()
            statuses.append(L.q1_server_wait(h, t, 60_000, ctypes.byref(resp)))
            assert resp.status == statuses[-1]
        assert all(s == 10 for s in statuses), statuses    # the injected round and all behind it
        t = ctypes.c_uint64()
        assert L.q1_server_submit(h, ctypes.byref(r0), ctypes.byref(t)) == 10
        st = _lib.ServerStats()
        _lib.check(L.q1_server_stats_get(h, ctypes.byref(st)))
        assert st.failed == len(tickets) and st.pending == 0 and refused + len(tickets) == len(reqs)
    finally:
        _lib.check(L.q1_server_close(h))
    h2 = open_server(slots=4, lanes=2)
    try:
        resp = _lib.Response()
        assert L.q1_server_wait(h2, submit(h2, r0), 60_000, ctypes.byref(resp)) == 0
        assert np.array_equal(words(resp), words(plain(h2, r0)))
        assert np.array_equal(words(resp), words(ok))
    finally:
        _lib.check(L.q1_server_close(h2))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [2, 3])
def test_server_open_fails_cleanly_and_reopens(cuda, kind):
    """An allocation that fails while q1_server_open builds its state is reported as
    Q1_ERR_OUT_OF_MEMORY with no server made, what was built is released, and the next open on the
    same device answers exactly. The first device allocation (the resident table) fails after the
    streams exist; the first pinned one (a round lane's buffers) after the resident table, its
    per-day cubes and the ad-hoc arena are built."""
    from test_gpu_serve import FLAGS, KEYS, RES, open_server, plain, req, submit, wait, words
    L = q.lib()
    free0 = torch.cuda.mem_get_info()[0]
    _lib.check(L.q1_inject_fault(kind, 1))
    with pytest.raises(q.Q1Error) as e:
        open_server()
    assert e.value.status == 3 and "injected" in str(e.value)
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)   # the partial build was released
    h = open_server()
    try:
        for r in (req(RES, FLAGS, 729999), req(RES, KEYS, 728826, 64)):
            assert np.array_equal(words(wait(h, submit(h, r))), words(plain(h, r)))
    finally:
        _lib.check(L.q1_server_close(h))
