"""CPU tests of the serving loop's policy: admission under a slot limit and a memory budget,
continuous admission as work finishes, bounded bypass of a large request, rejection of
requests larger than the budget, and the latency statistics.  A fake executor stands in for
the GPU (completion after a simulated duration)."""
import time

import numpy as np
import pytest

from directsht_b200.serve import Admission, Request, Server, cap_points, poisson_requests


class FakeExecutor:
    def __init__(self, sec_per_byte=2e-10):
        self.sec_per_byte = sec_per_byte
        self.log = []

    def footprint(self, req):
        return int(req.N) * 100

    def start(self, req):
        self.log.append(("start", req.rid, time.perf_counter()))
        return {"t_end": time.perf_counter() + self.footprint(req) * self.sec_per_byte}

    def done(self, h):
        return time.perf_counter() >= h["t_end"]

    def result(self, req, h):
        return np.full((req.nmaps, 3), float(req.rid))


def _req(N, maps=1):
    return Request(32, 64, np.zeros(N), np.zeros(N), np.ones((maps, N)))


def test_admission_slots_and_budget():
    a = Admission(budget_bytes=1000, slots=2)
    for fp in (400, 400, 400, 100):
        a.push(object(), fp)
    start, rej = a.pop_admissible()
    assert [fp for _, fp in start] == [400, 400] and not rej     # slot limit
    a.release(400)
    start, _ = a.pop_admissible()
    assert [fp for _, fp in start] == [400]                       # freed slot, fits in 600
    assert a.used == 800 and a.running == 2


def test_admission_bypass_is_bounded_and_oversize_rejected():
    a = Admission(budget_bytes=1000, slots=100, max_bypass=2)
    a.push("big0", 900)
    a.push("huge", 5000)
    start, rej = a.pop_admissible()
    assert [r for r, _ in start] == ["big0"] and rej == ["huge"]
    a.push("big1", 900)           # head, waits for memory
    for i in range(5):
        a.push(f"s{i}", 10)
    start, _ = a.pop_admissible()
    assert [r for r, _ in start] == ["s0", "s1"]                   # two may pass, then the head blocks
    a.release(900)
    start, _ = a.pop_admissible()
    assert [r for r, _ in start][0] == "big1"


def test_server_continuous_admission_and_results():
    ex = FakeExecutor()
    srv = Server(ex, budget_bytes=10_000_000, slots=3, poll_s=1e-4).start()
    futs = [srv.submit(_req(n, maps=2)) for n in (20000, 1000, 50000, 3000, 7000, 100)]
    srv.stop(drain=True, timeout=30)
    for i, f in enumerate(futs):
        out = f.result(timeout=1)
        assert out.shape == (2, 3) and np.all(out == i)
    st = srv.stats()
    assert st["requests"] == 6 and st["max_concurrent"] <= 3 and st["p99_ms"] >= st["p50_ms"] > 0
    # a request was started while others were still running (not queue-then-batch)
    starts = [t for kind, _, t in ex.log if kind == "start"]
    assert len(starts) == 6


def test_server_rejects_oversize():
    srv = Server(FakeExecutor(), budget_bytes=1000, slots=2).start()
    f = srv.submit(_req(50))
    srv.stop(drain=True, timeout=10)
    with pytest.raises(MemoryError):
        f.result(timeout=1)


def test_cap_points_stay_in_cap():
    rng = np.random.default_rng(0)
    th, ph, (t0, p0) = cap_points(rng, 5000, 0.3, return_centre=True)
    v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    c = np.array([np.sin(t0) * np.cos(p0), np.sin(t0) * np.sin(p0), np.cos(t0)])
    cosd = c @ v
    assert np.all(cosd >= np.cos(0.3) - 1e-9)
    # uniform in the cap: cos(distance) uniform on [cos 0.3, 1]
    assert abs(np.mean(cosd) - (1 + np.cos(0.3)) / 2) < 2e-3
    assert np.all((th >= 0) & (th <= np.pi) & (ph >= 0) & (ph < 2 * np.pi))


def test_poisson_requests_shape():
    rng = np.random.default_rng(1)
    reqs = poisson_requests(rng, 20, 200.0, Nls=(16, 32), n_range=(100, 1000), maps=(1, 3))
    ts = np.array([t for t, _ in reqs])
    assert np.all(np.diff(ts) > 0) and 0.01 < ts[-1] < 1.0
    for _, r in reqs:
        assert r.Nx == 2 * r.Nl and 1 <= r.nmaps <= 3 and 100 <= r.N <= 1000
