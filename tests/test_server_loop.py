"""The request loop (gpv_server_*) with a stand-in executor, on the CPU.

Admission by footprint, overtaking with its bound, session affinity and
order, timeouts, unknown ids, error propagation and the latency statistics
are host logic; a Python executor stands in for the GPU solve.
"""
import threading
import time

import numpy as np
import pytest

W, H = 64, 64


def _desc(gpv, n):
    return gpv.make_desc(np.tile([[32.0, 32.0]], (n, 1)), 10, 1)


def _footprint(h, w, n, border=20, esz=1):
    cw, ch = w + 2 * border, h + 2 * border
    pitch = (cw + 31) // 32 * 32
    # an FP64 row-pass buffer only for images with a line under 89 samples
    rowpass = 0 if min(cw, ch) >= 89 else 8 * (h * cw + 2 * 89 + 8)
    return 2 * 4 * pitch * ch + 2 * rowpass + 2 * esz * h * w + n * (120 + 200 + 4)


class Recorder:
    def __init__(self, delay=0.02, fail_n=None):
        self.lock = threading.Lock()
        self.active = 0
        self.max_active = 0
        self.log = []
        self.delay = delay
        self.fail_n = fail_n

    def __call__(self, worker, req, desc, out):
        with self.lock:
            self.active += 1
            self.max_active = max(self.max_active, self.active)
            self.log.append((worker, req["session"], req["n"], float(desc["p0"][0, 0])))
        time.sleep(self.delay)
        out["p"][:, 0] = desc["p0"][:, 0] + 1.0
        out["converged"] = 1
        out["iterations"] = req["n"]
        with self.lock:
            self.active -= 1
        return -1 if self.fail_n is not None and req["n"] == self.fail_n else 0


def _px():
    return np.zeros((H, W), np.uint8)


def test_footprint_budget_bounds_concurrency(gpv_mod):
    rec = Recorder()
    one = _footprint(H, W, 4)
    srv = gpv_mod.Server(workers=4, hbm_budget=2 * one, executor=rec)
    tickets = [srv.submit(_px(), _px(), _desc(gpv_mod, 4)) for _ in range(10)]
    for t in tickets:
        out = srv.wait(t, 10000)
        assert np.all(out["converged"] == 1)
    st = srv.stats()
    assert st["completed"] == 10 and st["failed"] == 0
    assert rec.max_active == 2  # four workers, but only two requests fit
    assert st["peak_bytes"] <= st["hbm_budget"]
    assert st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def test_request_larger_than_budget_runs_alone(gpv_mod):
    rec = Recorder()
    srv = gpv_mod.Server(workers=3, hbm_budget=1000, executor=rec)
    tickets = [srv.submit(_px(), _px(), _desc(gpv_mod, 2)) for _ in range(4)]
    for t in tickets:
        srv.wait(t, 10000)
    assert rec.max_active == 1
    srv.close()


def test_small_requests_overtake_a_large_one_boundedly(gpv_mod):
    rec = Recorder(delay=0.05)
    small = _footprint(H, W, 1)
    big_h = 256
    srv = gpv_mod.Server(workers=2, hbm_budget=_footprint(big_h, big_h, 1) + 10, executor=rec)
    t0 = srv.submit(_px(), _px(), _desc(gpv_mod, 1))  # running: the big one no longer fits beside it
    time.sleep(0.01)
    big = srv.submit(np.zeros((big_h, big_h), np.uint8), np.zeros((big_h, big_h), np.uint8), _desc(gpv_mod, 3))
    smalls = [srv.submit(_px(), _px(), _desc(gpv_mod, 1)) for _ in range(20)]
    for t in [t0, big] + smalls:
        srv.wait(t, 20000)
    order = [n for _, _, n, _ in rec.log]
    pos = order.index(3)
    assert 1 <= pos <= 1 + 8 + 1  # overtaken, but by at most the bypass bound (+ the one already running)
    assert small < _footprint(big_h, big_h, 3)
    srv.close()


def test_sessions_are_served_in_order_on_one_worker(gpv_mod):
    rec = Recorder(delay=0.005)
    srv = gpv_mod.Server(workers=4, executor=rec, hbm_budget=1 << 30)
    tickets = []
    for k in range(6):
        for s in (11, 12, 13):
            d = _desc(gpv_mod, 2)
            d["p0"][:, 0] = k
            tickets.append(srv.submit(_px(), _px(), d, session=s))
    for t in tickets:
        srv.wait(t, 10000)
    for s in (11, 12, 13):
        mine = [(w, p) for w, ss, _, p in rec.log if ss == s]
        assert len({w for w, _ in mine}) == 1
        assert [p for _, p in mine] == sorted(p for _, p in mine)
    srv.close()


def test_wait_timeout_unknown_id_and_errors(gpv_mod):
    rec = Recorder(delay=0.3, fail_n=7)
    srv = gpv_mod.Server(workers=1, executor=rec, hbm_budget=1 << 30)
    t = srv.submit(_px(), _px(), _desc(gpv_mod, 7))
    rc, _, _ = srv.wait_raw(t.id, 10)
    assert rc == -5  # GPV_ERR_TIMEOUT
    with pytest.raises(gpv_mod.GpvError, match="failed"):
        srv.wait(t, 10000)
    assert srv.wait_raw(t.id, 0)[0] == -6  # collected: GPV_ERR_NOT_FOUND
    assert srv.wait_raw(12345, 0)[0] == -6
    assert srv.stats()["failed"] == 1
    srv.close()


def test_submit_argument_checks(gpv_mod):
    srv = gpv_mod.Server(workers=1, executor=Recorder(), hbm_budget=1 << 30)
    with pytest.raises(gpv_mod.GpvError, match="session"):
        srv.submit(_px(), _px(), _desc(gpv_mod, 1), reuse_reference=True)
    with pytest.raises(gpv_mod.GpvError):
        srv.submit(_px(), _px(), _desc(gpv_mod, 1), border=2)
    with pytest.raises(ValueError):
        srv.submit(np.zeros((8, 8), np.uint8), _px(), _desc(gpv_mod, 1))
    srv.close()


def test_close_serves_what_is_queued(gpv_mod):
    rec = Recorder(delay=0.01)
    srv = gpv_mod.Server(workers=2, executor=rec, hbm_budget=1 << 30)
    for _ in range(8):
        srv.submit(_px(), _px(), _desc(gpv_mod, 1))
    srv.close()
    assert len(rec.log) == 8


def test_priority_lane_routes_by_size(gpv_mod):
    """With a priority lane, requests of at most priority_subsets subsets run
    on the priority workers only, larger ones on the others, and session
    requests stay on their session's worker whatever their size."""
    rec = Recorder(delay=0.005)
    srv = gpv_mod.Server(workers=5, executor=rec, hbm_budget=1 << 30, priority_workers=2, priority_subsets=8)
    tickets = []
    for k in range(24):
        tickets.append(srv.submit(_px(), _px(), _desc(gpv_mod, 3 + (k % 3) * 5)))  # 3, 8, 13 subsets
    for k in range(4):
        tickets.append(srv.submit(_px(), _px(), _desc(gpv_mod, 20), session=5))  # large, pinned to worker 0
    for t in tickets:
        srv.wait(t, 10000)
    srv.close()
    plain = [(w, n) for w, s, n, _ in rec.log if s == 0]
    assert len(plain) == 24
    assert all(w < 2 for w, n in plain if n <= 8) and all(w >= 2 for w, n in plain if n > 8)
    assert {w for w, s, _, _ in rec.log if s == 5} == {5 % 5}


def test_priority_lane_config_checks(gpv_mod):
    for pw, ps in ((3, 10), (-1, 10), (1, 0)):
        with pytest.raises(gpv_mod.GpvError, match="priority"):
            gpv_mod.Server(workers=3, executor=Recorder(), hbm_budget=1 << 30, priority_workers=pw,
                           priority_subsets=ps)


def test_prepare_reaches_every_worker_and_is_not_a_request(gpv_mod):
    rec = Recorder(delay=0.001)
    srv = gpv_mod.Server(workers=3, executor=rec, hbm_budget=1 << 30)
    srv.prepare((H, W), np.uint8)
    srv.prepare((H, W), np.uint16)
    st = srv.stats()
    assert st["completed"] == 0 and st["submitted"] == 0 and not rec.log
    with pytest.raises(gpv_mod.GpvError, match="border"):
        srv.prepare((H, W), np.uint8, border=1)
    srv.wait(srv.submit(_px(), _px(), _desc(gpv_mod, 2)), 10000)
    assert srv.stats()["completed"] == 1
    srv.close()
