"""Serving loop (q1_server_*): resident table with per-day partial aggregates, ad-hoc tables
admitted under an HBM budget, continuous batching into rounds. Every response must equal the
plain one-launch path (q1_server_plain) bit for bit, alone and in a mix, and the plain path must
equal the oracle."""
import ctypes
import functools
import threading

import numpy as np
import pytest

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O
from tpchq01_gpu_b200 import _lib

pytestmark = pytest.mark.gpu

SEED = 4242
RES_ROWS = 3_000_017
ADHOC_MAX = 2_000_000
FLAGS, KEYS = _lib.GROUP_FLAGS, _lib.GROUP_KEYS
RES, ADHOC = _lib.REQ_RESIDENT, _lib.REQ_ADHOC
EDGE_CUTOFFS = [700000, 727562, 727563, 727564, 728826, 729999, 730089, 740000]


def open_server(budget=256 << 20, slots=16, mode=_lib.SERVE_BATCHED, lanes=0):
    o = _lib.ServerOpts()
    q.lib().q1_server_opts_default(ctypes.byref(o))
    o.mode = mode
    o.max_rounds_in_flight = lanes
    o.seed = SEED
    o.resident_rows = RES_ROWS
    o.hbm_budget_bytes = budget
    o.max_inflight = slots
    o.max_adhoc_rows = ADHOC_MAX
    h = ctypes.c_void_p()
    _lib.check(q.lib().q1_server_open(ctypes.byref(o), ctypes.byref(h)))
    return h


def req(kind, grouping, cutoff, groups=0, rows=0, seed=0):
    return _lib.Request(kind, grouping, groups, cutoff, rows, seed)


def words(resp):
    g = resp.num_groups
    return np.frombuffer(resp.aggregates, dtype=np.uint64)[: g * 12].copy()


def submit(h, r):
    t = ctypes.c_uint64()
    _lib.check(q.lib().q1_server_submit(h, ctypes.byref(r), ctypes.byref(t)))
    return t.value


def wait(h, t, timeout_ms=120_000):
    resp = _lib.Response()
    _lib.check(q.lib().q1_server_wait(h, t, timeout_ms, ctypes.byref(resp)))
    assert resp.status == 0 and resp.ticket == t
    return resp


def plain(h, r):
    resp = _lib.Response()
    _lib.check(q.lib().q1_server_plain(h, ctypes.byref(r), ctypes.byref(resp)))
    return resp


@functools.lru_cache(maxsize=4)
def table(seed, rows):
    cols = gen_np.generate(seed, 0, rows)
    rfc = cols["returnflag"].view(np.uint8)
    lsc = cols["linestatus"].view(np.uint8)
    rf = np.where(rfc == ord("R"), 2, 0) + np.where(rfc == ord("N"), 1, 0)
    pair_keys = ((rf << 1) + np.where(lsc == ord("F"), 0, 1)).astype(np.uint32)
    return gen_np.compress(cols), pair_keys


def oracle(kind, grouping, cutoff, groups, rows, seed):
    """int128 table of the request from the oracle (group keys = (rf << 1) + ls for FLAGS)."""
    if kind == RES:
        rows, seed = RES_ROWS, SEED
    comp, pair_keys = table(seed, rows)
    if grouping == FLAGS:
        keys, groups = pair_keys, 6
    else:
        keys = gen_np.group_keys_uniform(seed, 0, rows, groups)
    buf, flag = O.q1_groupkey(comp, keys, groups, cutoff)
    assert flag == 0
    return buf


@pytest.fixture(scope="module")
def server(cuda):
    h = open_server()
    yield h
    _lib.check(q.lib().q1_server_close(h))


def mix_requests(seed=9):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(48):
        kind = RES if i % 2 == 0 else ADHOC
        grouping = FLAGS if (i // 2) % 2 == 0 else KEYS
        cutoff = EDGE_CUTOFFS[i % len(EDGE_CUTOFFS)] if i % 3 == 0 else int(rng.integers(729906, 730090))
        groups = 64 if kind == RES else [1, 4, 7, 9, 33, 64][i % 6]
        rows = 0 if kind == RES else [0, 1, 2047, 2048, 2049, 65_537, 300_001, 1_999_999][(i // 2) % 8]
        out.append(req(kind, grouping, cutoff, groups if grouping == KEYS else 0, rows, 1000 + i))
    return out


@pytest.mark.parametrize("kind,grouping,groups,rows", [
    (RES, FLAGS, 0, 0), (RES, KEYS, 64, 0),
    (ADHOC, FLAGS, 0, 300_001), (ADHOC, KEYS, 5, 100_003), (ADHOC, KEYS, 64, 65_536)])
@pytest.mark.parametrize("cutoff", [727562, 728826, 729999, 740000])
def test_plain_equals_oracle(server, kind, grouping, groups, rows, cutoff):
    r = req(kind, grouping, cutoff, groups, rows, 77)
    got = words(plain(server, r))
    want = oracle(kind, grouping, cutoff, groups, rows, 77)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("kind,grouping,groups,rows", [
    (RES, FLAGS, 0, 0), (RES, KEYS, 64, 0), (ADHOC, FLAGS, 0, 300_001), (ADHOC, KEYS, 33, 100_003)])
def test_served_alone_equals_plain(server, kind, grouping, groups, rows):
    for cutoff in EDGE_CUTOFFS:
        r = req(kind, grouping, cutoff, groups, rows, 78)
        got = wait(server, submit(server, r))
        assert got.num_groups == (6 if grouping == FLAGS else groups)
        assert np.array_equal(words(got), words(plain(server, r))), cutoff


def test_served_mix_equals_alone_and_plain(server):
    reqs = mix_requests()
    tickets = [submit(server, r) for r in reqs]
    mixed = [words(wait(server, t)) for t in tickets]
    for r, m in zip(reqs, mixed):
        assert np.array_equal(m, words(plain(server, r)))
        assert np.array_equal(m, words(wait(server, submit(server, r))))


def test_concurrent_submitters_and_budget_admission(cuda):
    # a budget of ~2 max-size tables: rounds are limited by memory, not only by slots
    budget = 2 * 14 * ADHOC_MAX + (1 << 16)
    h = open_server(budget=budget, slots=8)
    try:
        reqs = mix_requests(seed=11) * 2
        results = [None] * len(reqs)
        errors = []

        def worker(k):
            try:
                for i in range(k, len(reqs), 4):
                    results[i] = words(wait(h, submit(h, reqs[i])))
            except Exception as e:   # reported below
                errors.append(e)

        ths = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        assert not errors, errors
        st = _lib.ServerStats()
        _lib.check(q.lib().q1_server_stats_get(h, ctypes.byref(st)))
        assert st.completed == len(reqs) and st.failed == 0 and st.pending == 0
        assert st.rounds >= 1 and st.p99_ms >= st.p50_ms > 0
        for r, m in zip(reqs, results):
            assert np.array_equal(m, words(plain(h, r)))
        # a burst larger than the slots forms rounds of more than one request
        _lib.check(q.lib().q1_server_reset_stats(h))
        tickets = [submit(h, r) for r in reqs]
        for t in tickets:
            wait(h, t)
        _lib.check(q.lib().q1_server_stats_get(h, ctypes.byref(st)))
        assert st.completed == len(reqs) and st.mean_round_size > 1.0
        assert st.logical_rows == sum(RES_ROWS if r.kind == RES else r.adhoc_rows for r in reqs)
        # the budget holds about two of the largest tables: some were evicted and made again
        assert st.evictions > 0 and st.cache_misses > 0 and st.cached_bytes <= budget
    finally:
        _lib.check(q.lib().q1_server_close(h))


def test_table_cache_hits_and_results(server):
    r1 = req(ADHOC, KEYS, 729950, 9, 123_457, 31337)
    r2 = req(ADHOC, KEYS, 730050, 9, 123_457, 31337)    # same table, other cutoff
    r3 = req(ADHOC, KEYS, 730050, 10, 123_457, 31337)   # other key column: other table
    before = _lib.ServerStats()
    _lib.check(q.lib().q1_server_stats_get(server, ctypes.byref(before)))
    got = [words(wait(server, submit(server, r))) for r in (r1, r2, r3, r1)]
    after = _lib.ServerStats()
    _lib.check(q.lib().q1_server_stats_get(server, ctypes.byref(after)))
    assert after.cache_misses - before.cache_misses == 2
    assert after.cache_hits - before.cache_hits == 2
    assert after.generated_rows - before.generated_rows == 2 * 123_457
    for r, g in zip((r1, r2, r3, r1), got):
        assert np.array_equal(g, words(plain(server, r)))
    assert np.array_equal(got[0], got[3])


def test_plain_mode_server(cuda):
    h = open_server(mode=_lib.SERVE_PLAIN)
    try:
        reqs = mix_requests(seed=13)[:24]
        tickets = [submit(h, r) for r in reqs]
        got = [words(wait(h, t)) for t in tickets]
        st = _lib.ServerStats()
        _lib.check(q.lib().q1_server_stats_get(h, ctypes.byref(st)))
        assert st.rounds == st.completed == len(reqs) and st.mean_round_size == 1.0
        for r, g in zip(reqs, got):
            assert np.array_equal(g, words(plain(h, r)))
    finally:
        _lib.check(q.lib().q1_server_close(h))


def test_rejections(server):
    L = q.lib()
    t = ctypes.c_uint64()

    def status(r):
        return L.q1_server_submit(server, ctypes.byref(r), ctypes.byref(t))

    assert status(req(RES, KEYS, 729999, 32)) == 1          # resident key column has 64 groups
    assert status(req(ADHOC, KEYS, 729999, 0, 10, 1)) == 1  # no groups
    assert status(req(ADHOC, KEYS, 729999, 65, 10, 1)) == 1
    assert status(req(ADHOC, FLAGS, 729999, 0, ADHOC_MAX + 1, 1)) == 1
    assert status(req(7, FLAGS, 729999)) == 1
    assert L.q1_server_wait(server, 123456789, 0, ctypes.byref(_lib.Response())) == 1


def test_round_lane_option_is_checked(cuda):
    o = _lib.ServerOpts()
    q.lib().q1_server_opts_default(ctypes.byref(o))
    assert o.max_rounds_in_flight == 2
    o.max_rounds_in_flight = 9
    h = ctypes.c_void_p()
    assert q.lib().q1_server_open(ctypes.byref(o), ctypes.byref(h)) == 1   # Q1_ERR_INVALID_ARGUMENT
    assert not h.value


def test_budget_refusal(cuda):
    h = open_server(budget=1 << 20, slots=4)
    try:
        t = ctypes.c_uint64()
        r = req(ADHOC, FLAGS, 729999, 0, 1_000_000, 1)
        assert q.lib().q1_server_submit(h, ctypes.byref(r), ctypes.byref(t)) == 8   # Q1_ERR_BUSY
        small = req(ADHOC, KEYS, 729999, 3, 10_000, 5)
        got = wait(h, submit(h, small))
        assert np.array_equal(words(got), words(plain(h, small)))
    finally:
        _lib.check(q.lib().q1_server_close(h))


@pytest.mark.parametrize("lanes", [1, 2, 4])
def test_rounds_overlap_on_the_device(cuda, lanes):
    """Continuous batching: a burst larger than one round's slots forms round after round, and with
    more than one round lane a round is enqueued while the previous one is still on the GPU (its
    copies and kernels queue behind it on another stream). Every response equals the plain path."""
    h = open_server(slots=4, lanes=lanes)
    try:
        rng = np.random.default_rng(lanes)
        reqs = []
        for i in range(40):
            rows = int(rng.integers(200_000, ADHOC_MAX))
            if i % 5 == 0:
                reqs.append(req(RES, FLAGS if i % 2 else KEYS, int(rng.integers(729906, 730090)), 0 if i % 2 else 64))
            else:
                reqs.append(req(ADHOC, KEYS if i % 3 else FLAGS, int(rng.integers(729906, 730090)),
                                [4, 9, 64][i % 3] if i % 3 else 0, rows, 500 + i % 7))
        # make the tables resident first, so that the burst below is all scans
        for r in reqs:
            if r.kind == ADHOC:
                wait(h, submit(h, r))
        _lib.check(q.lib().q1_server_reset_stats(h))
        tickets = [submit(h, r) for r in reqs]
        got = [words(wait(h, t)) for t in tickets]
        st = _lib.ServerStats()
        _lib.check(q.lib().q1_server_stats_get(h, ctypes.byref(st)))
        assert st.completed == len(reqs) and st.failed == 0 and st.rounds >= len(reqs) // 4
        assert st.max_rounds_in_flight <= lanes
        if lanes == 1:
            assert st.overlapped_rounds == 0
        else:
            assert st.overlapped_rounds > 0 and st.max_rounds_in_flight >= 2
        for r, g in zip(reqs, got):
            assert np.array_equal(g, words(plain(h, r)))
    finally:
        _lib.check(q.lib().q1_server_close(h))
