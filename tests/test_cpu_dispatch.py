"""Serving over several GPUs as replicas: the dispatcher's assignment and its
per-device worker processes, on the CPU with a stand-in server (no GPU): two
worker processes each 'serve' their share by sleeping for its work at a fixed
rate; every request comes back exactly once with its latency."""

import time

import numpy as np

from hemepure_b200 import serving


class FakeServer:
    """Serves requests one after the other at `rate` site updates per second,
    each no earlier than its arrival (a stand-in with the Server interface)."""

    def __init__(self, device, rate=2e9):
        self.device, self.rate, self.completed, self.wall_s = device, rate, [], 0.0

    def run(self, reqs):
        t0 = time.perf_counter()
        for r in sorted(reqs, key=lambda q: q.arrival):
            now = time.perf_counter() - t0
            if now < r.arrival:
                time.sleep(r.arrival - now)
            r.admitted = time.perf_counter() - t0
            time.sleep(r.sites * r.steps / self.rate)
            r.finished = time.perf_counter() - t0
            r.steps_done = r.steps
            self.completed.append(r)
        self.wall_s = time.perf_counter() - t0

    def report(self):
        return {"wall_s": self.wall_s, "requests": len(self.completed)}


def make_fake(device):
    return FakeServer(device)


def _requests(n, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for i in range(n):
        t += float(rng.exponential(0.01))
        out.append(serving.Request(rid=i, xml="", kernel="LBGK", wall="SBB", steps=int(rng.integers(1000, 5000)),
                                   sites=int(rng.integers(1000, 20000)), arrival=t))
    return out


def test_least_work_assignment_balances_and_keeps_arrival_order():
    reqs = _requests(200)
    shares = serving.assign_least_work(reqs, 3)
    assert sorted(r.rid for s in shares for r in s) == list(range(200))
    loads = [sum(r.sites * r.steps for r in s) for s in shares]
    biggest = max(r.sites * r.steps for r in reqs)
    assert max(loads) - min(loads) <= biggest
    for s in shares:
        arr = [r.arrival for r in s]
        assert arr == sorted(arr)


def test_dispatcher_two_worker_processes():
    reqs = _requests(24)
    d = serving.Dispatcher([0, 1], budget_bytes=1 << 30, server_factory=make_fake)
    rep = d.run(reqs)
    assert rep["devices"] == 2 and rep["requests"] == 24 and rep["failed"] == 0
    assert set(rep["per_device"]) == {0, 1}
    assert all(r.finished is not None and r.finished >= r.admitted >= r.arrival - 1e-3 for r in reqs)
    assert sum(p["requests"] for p in rep["per_device"].values()) == 24
    work = sum(r.sites * r.steps for r in reqs)
    assert rep["aggregate_MLUPS"] > 0 and abs(sum(rep["assigned_work"]) - work) == 0


def test_saturated_window_excludes_the_drain():
    """The sustained rate counts the blocks run while at least half of the peak
    resident set was resident: the drain at the end (one long request alone)
    is left out, the blocks of the loaded server are in."""
    log = [(0.5, 5e6, 8), (0.5, 5e6, 8), (0.5, 4e6, 6), (0.5, 2e6, 4), (1.0, 1e6, 1), (1.0, 1e6, 1)]
    w = serving.saturated_window(log)
    assert w["peak_resident"] == 8 and w["blocks"] == 4
    assert w["wall_s"] == 2.0
    assert abs(w["MLUPS"] - 16e6 / 2.0 / 1e6) < 1e-12
    assert serving.saturated_window([])["blocks"] == 0
