"""Host tests of the server's scheduling policy (continuous batching, the
device-memory budget, cancellation, failures, latency statistics).

The scheduler in cuda-sort_b200/csrc/serving_core.hpp has no CUDA in it; here
it runs over a fake device (tests/serving_fake.cpp, built with g++) that
stages and sorts batches on host threads with configurable delays and
injected failures, and that checks the scheduler's arena promises (regions
inside the budget, back to back, no overlap between batches in flight).
"""
import ctypes
import os
import subprocess
import threading
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

OK, INVALID, UNSUPPORTED, CUDA, OOM, TIMEOUT, BUDGET, BUSY, CANCELLED = range(9)
FREE, QUEUED, RUNNING, DONE, FAILED, CANCELLED_STATE = range(6)


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "submitted", "completed", "failed", "cancelled", "rejected", "batches", "keys_completed", "queued",
        "inflight_batches", "peak_arena_bytes", "arena_bytes", "max_batch_requests")] + \
        [(n, ctypes.c_double) for n in ("mean_batch_requests", "p50_us", "p99_us", "p999_us", "max_us", "mean_us",
                                        "span_s")]


@pytest.fixture(scope="module")
def fake(tmp_path_factory):
    out = tmp_path_factory.mktemp("fake") / "libserving_fake.so"
    cmd = ["g++", "-O1", "-g", "-std=c++17", "-shared", "-fPIC", "-pthread",
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(ROOT, "cuda-sort_b200", "csrc"),
           os.path.join(ROOT, "tests", "serving_fake.cpp"), "-o", str(out)]
    subprocess.run(cmd, check=True)
    lib = ctypes.CDLL(str(out))
    vp, i64, u64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64
    sig = {
        "fake_create": (vp, [ctypes.c_int, i64, ctypes.c_int, ctypes.c_int, i64, ctypes.c_int, ctypes.c_int32]),
        "fake_destroy": (None, [vp]),
        "fake_shutdown": (None, [vp]),
        "fake_submit": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32, ctypes.POINTER(u64)]),
        "fake_wait": (ctypes.c_int, [vp, u64, i64, ctypes.POINTER(ctypes.c_int)]),
        "fake_poll": (ctypes.c_int, [vp, u64]),
        "fake_cancel": (ctypes.c_int, [vp, u64]),
        "fake_drain": (ctypes.c_int, [vp, i64]),
        "fake_stats": (None, [vp, ctypes.POINTER(Stats), ctypes.c_int]),
        "fake_inject": (None, [vp, ctypes.c_int, ctypes.c_int]),
        "fake_set_delay": (None, [vp, ctypes.c_int]),
        "fake_violations": (i64, [vp]),
        "fake_last_error": (ctypes.c_char_p, []),
        "fake_arena_selftest": (i64, [u64, ctypes.c_int, i64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


class Server:
    def __init__(self, lib, eb=8, budget=1 << 20, slots=2, max_batch=64, max_queue=4096, delay_us=0,
                 max_len=65536):
        self.lib = lib
        self.h = lib.fake_create(eb, budget, slots, max_batch, max_queue, delay_us, max_len)
        self.eb = eb
        self.keep = {}

    def submit(self, arr):
        t = ctypes.c_uint64()
        out = np.empty_like(arr)
        st = self.lib.fake_submit(self.h, arr.ctypes.data, out.ctypes.data, len(arr), ctypes.byref(t))
        if st == OK:
            self.keep[t.value] = (arr, out)
        return st, t.value, out

    def wait(self, t, timeout_us=10_000_000):
        r = ctypes.c_int()
        st = self.lib.fake_wait(self.h, t, timeout_us, ctypes.byref(r))
        return st, r.value

    def stats(self, reset=False):
        s = Stats()
        self.lib.fake_stats(self.h, ctypes.byref(s), int(reset))
        return s

    def close(self):
        if self.h:
            self.lib.fake_destroy(self.h)
            self.h = None


def records(rng, n):
    a = np.empty(n, dtype=[("key", "<i4"), ("data", "<i4")])
    a["key"] = rng.integers(-50, 50, n)
    a["data"] = np.arange(n)
    return a


def test_ring_arena_invariants(fake):
    for seed in range(20):
        assert fake.fake_arena_selftest(seed, 4000, 1000 + 37 * seed) == 0


def test_requests_sorted_and_batched(fake):
    rng = np.random.default_rng(1)
    srv = Server(fake, slots=2, max_batch=32, delay_us=300)
    try:
        tickets = []
        for _ in range(400):
            arr = records(rng, int(rng.integers(1, 300)))
            st, t, out = srv.submit(arr)
            assert st == OK
            tickets.append((t, arr, out))
        for t, arr, out in tickets:
            st, res = srv.wait(t)
            assert st == OK and res == OK
            want = arr[np.argsort(arr["key"], kind="stable")]
            assert np.array_equal(out, want)
        s = srv.stats()
        assert s.completed == 400 and s.failed == 0 and s.queued == 0
        assert s.batches < 400 and s.mean_batch_requests > 1.0   # requests shared batches
        assert s.max_batch_requests <= 32
        assert fake.fake_violations(srv.h) == 0
    finally:
        srv.close()


def test_submit_from_many_threads(fake):
    srv = Server(fake, slots=3, max_batch=16, delay_us=100)
    errors = []

    def client(seed):
        rng = np.random.default_rng(seed)
        mine = []
        for _ in range(100):
            arr = records(rng, int(rng.integers(1, 64)))
            st, t, out = srv.submit(arr)
            if st != OK:
                errors.append(st)
                return
            mine.append((t, arr, out))
        for t, arr, out in mine:
            st, res = srv.wait(t)
            if st != OK or res != OK or not np.array_equal(out["key"], np.sort(arr["key"])):
                errors.append((st, res))

    try:
        th = [threading.Thread(target=client, args=(s,)) for s in range(6)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        assert not errors
        assert srv.stats().completed == 600
        assert fake.fake_violations(srv.h) == 0
    finally:
        srv.close()


def test_admission_respects_the_budget(fake):
    # 64 KiB arena; requests of 16 KiB (2048 records): at most four admitted at a time
    rng = np.random.default_rng(2)
    srv = Server(fake, budget=64 << 10, slots=8, max_batch=8, delay_us=2000)
    try:
        tickets = [srv.submit(records(rng, 2048))[1] for _ in range(16)]
        time.sleep(0.001)
        s = srv.stats()
        assert s.queued >= 8   # the rest waits for memory, not for a slot
        for t in tickets:
            assert srv.wait(t) == (OK, OK)
        s = srv.stats()
        assert s.peak_arena_bytes <= 64 << 10
        assert s.arena_bytes == 64 << 10
        assert s.completed == 16
        assert fake.fake_violations(srv.h) == 0
    finally:
        srv.close()


def test_request_larger_than_budget_is_rejected(fake):
    srv = Server(fake, budget=4096)
    try:
        st, _, _ = srv.submit(records(np.random.default_rng(3), 1000))   # 8000 bytes > 4096
        assert st == BUDGET
        assert b"budget" in fake.fake_last_error()
        assert srv.stats().rejected == 1
        st, t, _ = srv.submit(records(np.random.default_rng(3), 100))
        assert st == OK and srv.wait(t) == (OK, OK)
    finally:
        srv.close()


def test_unsupported_length_and_bad_arguments(fake):
    srv = Server(fake, max_len=1000)
    try:
        assert srv.submit(records(np.random.default_rng(4), 1001))[0] == UNSUPPORTED
        t = ctypes.c_uint64()
        assert fake.fake_submit(srv.h, None, None, 5, ctypes.byref(t)) == INVALID
        assert fake.fake_submit(srv.h, None, None, -1, ctypes.byref(t)) == INVALID
        assert srv.wait(12345)[0] == INVALID     # never issued
    finally:
        srv.close()


def test_zero_length_request_completes_at_once(fake):
    srv = Server(fake)
    try:
        st, t, _ = srv.submit(records(np.random.default_rng(5), 0))
        assert st == OK
        assert fake.fake_poll(srv.h, t) == DONE
        assert srv.wait(t, 0) == (OK, OK)
    finally:
        srv.close()


def test_queue_full_reports_busy(fake):
    rng = np.random.default_rng(6)
    srv = Server(fake, slots=1, max_batch=1, max_queue=8, delay_us=50_000)
    try:
        codes = [srv.submit(records(rng, 10))[0] for _ in range(12)]
        assert codes[:8] == [OK] * 8
        assert BUSY in codes[8:]
        assert srv.stats().rejected >= 1
        assert fake.fake_drain(srv.h, 5_000_000) == OK
    finally:
        srv.close()


def test_cancel_only_while_queued(fake):
    rng = np.random.default_rng(7)
    srv = Server(fake, slots=1, max_batch=1, delay_us=100_000)
    try:
        _, t1, _ = srv.submit(records(rng, 10))
        time.sleep(0.02)                      # t1 is admitted
        _, t2, out2 = srv.submit(records(rng, 10))
        assert fake.fake_poll(srv.h, t2) == QUEUED
        assert fake.fake_cancel(srv.h, t2) == OK
        assert srv.wait(t2) == (OK, CANCELLED)
        assert fake.fake_poll(srv.h, t2) == CANCELLED_STATE
        assert fake.fake_cancel(srv.h, t1) == INVALID     # running: cannot cancel
        assert srv.wait(t1) == (OK, OK)
        assert srv.stats().cancelled == 1
    finally:
        srv.close()


def test_launch_failure_fails_that_batch_only(fake):
    rng = np.random.default_rng(8)
    srv = Server(fake, slots=1, max_batch=1)
    try:
        fake.fake_inject(srv.h, 1, 0)
        _, t1, _ = srv.submit(records(rng, 10))
        assert srv.wait(t1) == (OK, CUDA)
        _, t2, out = srv.submit(records(rng, 10))
        assert srv.wait(t2) == (OK, OK)
        fake.fake_inject(srv.h, 0, 1)
        _, t3, _ = srv.submit(records(rng, 10))
        assert srv.wait(t3) == (OK, CUDA)
        _, t4, _ = srv.submit(records(rng, 10))
        assert srv.wait(t4) == (OK, OK)
        s = srv.stats()
        assert s.failed == 2 and s.completed == 2
    finally:
        srv.close()


def test_wait_times_out_while_pending(fake):
    srv = Server(fake, slots=1, delay_us=200_000)
    try:
        _, t, _ = srv.submit(records(np.random.default_rng(9), 10))
        assert srv.wait(t, 1000)[0] == TIMEOUT
        assert fake.fake_drain(srv.h, 1000) == TIMEOUT
        assert srv.wait(t) == (OK, OK)
    finally:
        srv.close()


def test_shutdown_cancels_queued_and_finishes_admitted(fake):
    rng = np.random.default_rng(10)
    srv = Server(fake, slots=1, max_batch=1, delay_us=50_000)
    try:
        tickets = [srv.submit(records(rng, 10))[1] for _ in range(5)]
        time.sleep(0.01)
        fake.fake_shutdown(srv.h)
        states = [fake.fake_poll(srv.h, t) for t in tickets]
        assert states[0] == DONE
        assert states[1:].count(CANCELLED_STATE) >= 3
        assert all(s in (DONE, CANCELLED_STATE) for s in states)
        t = ctypes.c_uint64()
        arr = records(rng, 4)
        out = np.empty_like(arr)
        assert fake.fake_submit(srv.h, arr.ctypes.data, out.ctypes.data, 4, ctypes.byref(t)) == INVALID
    finally:
        srv.close()


def test_latency_statistics(fake):
    rng = np.random.default_rng(11)
    srv = Server(fake, slots=1, max_batch=1, delay_us=2000)
    try:
        tickets = [srv.submit(records(rng, 10))[1] for _ in range(20)]
        for t in tickets:
            srv.wait(t)
        s = srv.stats(reset=True)
        assert s.completed == 20 and s.batches == 20
        assert 2000 <= s.p50_us <= s.p99_us <= s.p999_us <= s.max_us
        assert s.p99_us >= 20 * 2000 * 0.9       # the last request queued behind 19 others
        assert s.span_s > 0.03
        s2 = srv.stats()
        assert s2.completed == 0 and s2.p50_us == 0
    finally:
        srv.close()
