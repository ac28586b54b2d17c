"""Serving loop over the batched form: continuous batching of solve requests.

Requests (geometry, relaxation time, inlet profile, step count) arrive over
time; the server admits each as soon as the batch has a free slot and room in
its HBM budget, keeps every admitted lattice resident on the device, steps all
of them together in CUDA-graph blocks, and retires each at its step count with
its extractions (density, velocity, wall shear stress of the last step).
Latency is arrival to retirement; throughput is site updates per second over
the run.
"""

from __future__ import annotations

import math
import os
import tempfile
import time
from collections import deque
from concurrent.futures import Future, ProcessPoolExecutor, ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import lbm, vessels


@dataclass
class Request:
    rid: int
    xml: str
    kernel: str
    wall: str
    steps: int
    sites: int
    arrival: float = 0.0
    shape: str = ""
    # filled by the server
    admitted: Optional[float] = None
    finished: Optional[float] = None
    steps_done: int = 0      # time steps the lattice made (its step count unless it went unstable)
    result: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None
    status: int = 0          # status bits of the run (1 unstable, 2 iolet radius), or a negative error code
    error: str = ""

    @property
    def latency(self) -> Optional[float]:
        return None if self.finished is None else self.finished - self.arrival


# ---------------------------------------------------------------------------
# The request mix: seeded random vessels
# ---------------------------------------------------------------------------

def _make_request(args) -> Tuple[int, str, str, str, int, int, str]:
    (rid, out_dir, seed, r_range, l_range, step_range, re_max) = args
    rng = np.random.default_rng([seed, rid])
    shape = ["pipe", "bifurcation", "stenosis"][int(rng.integers(0, 3))]
    r = float(rng.uniform(*r_range))
    length = float(rng.uniform(*l_range)) * r
    kernel = "LBGK" if rng.random() < 0.5 else "TRT"
    tau = float(rng.uniform(0.51, 1.0))
    nu = (tau - 0.5) / 3.0
    sev = float(rng.uniform(0.5, 0.75))              # stenosis area reduction
    # peak inflow velocity at Re <= re_max (on the inlet diameter), capped so the
    # fastest section (the stenosis throat) stays below 0.03 lattice units
    narrowing = (1.0 - sev) if shape == "stenosis" else 1.0
    u = min(re_max * nu / (2.0 * r), 0.03 * narrowing) * float(rng.uniform(0.5, 1.0))
    steps = int(rng.integers(step_range[0], step_range[1] + 1))
    ri = max(3, int(round(r)))
    li = max(8, int(round(length)))
    if shape == "pipe":
        v = vessels.Pipe(ri, li)
    elif shape == "stenosis":
        rmin = max(2.0, ri * math.sqrt(1.0 - sev))
        v = vessels.Stenosis(ri, li, rmin, max(4.0, 2.0 * ri))
    else:
        rd = max(3, int(round(ri * 0.8)))
        v = vessels.YBifurcation(ri, li // 2, rd, li // 2, 35.0)
    d = os.path.join(out_dir, f"req{rid:05d}")
    os.makedirs(d, exist_ok=True)
    gmy = os.path.join(d, "geom.gmy")
    xml = os.path.join(d, "case.xml")
    info = vessels.voxelise(v, gmy)
    units = vessels.CaseUnits(tau=tau)
    n_out = len([io for io in v.iolets if io.kind == "outlet"])
    # Either inlet kind is ramped in over the reference's warm-up (extra_warmup_steps:
    # the parabolic peak grows linearly, the cosine density moves linearly from the
    # lowest iolet density to its target); a pressure step applied at once from rest
    # sends a wave that low-viscosity cases do not survive.
    warm = int(min(1000, steps // 4))
    if rng.random() < 0.5:
        inlet = [vessels.VelocityBC(u)]
    else:
        # pressure drop that drives about u through a Poiseuille tube of this size
        drho = 3.0 * 8.0 * nu * u * length / (r * r) / 2.0
        inlet = [vessels.PressureBC(1.0 + drho)]
    outlets = [vessels.PressureBC(1.0)] * n_out
    vessels.write_case_xml(xml, "geom.gmy", v, units, max(1, steps - warm), inlet, outlets, warmup=warm,
                           relaxation_parameter=3.0 / 16.0 if kernel == "TRT" else None)
    wall = "BFL" if rng.random() < 0.5 else "SBB"
    return rid, xml, kernel, wall, steps, info.fluid_sites, shape


def generate_requests(n: int, out_dir: Optional[str] = None, seed: int = 2024,
                      radius: Tuple[float, float] = (6.0, 32.0), length_radii: Tuple[float, float] = (10.0, 40.0),
                      steps: Tuple[int, int] = (1000, 20000), re_max: float = 300.0,
                      workers: int = 0) -> List[Request]:
    """Seeded random vessels: straight pipe, Y-bifurcation at +-35 degrees, or
    50-75 % cosine stenosis with equal probability; radius U[r0, r1], length
    U[l0, l1] radii; LBGK or TRT with tau ~ U[0.51, 1.0]; pressure or parabolic
    velocity inlet at Re <= re_max; step count U[s0, s1]."""
    out_dir = out_dir or tempfile.mkdtemp(prefix="hemeb200_requests_")
    jobs = [(i, out_dir, seed, radius, length_radii, steps, re_max) for i in range(n)]
    workers = workers or min(16, os.cpu_count() or 1)
    if workers > 1 and n > 1:
        import multiprocessing as mp
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            made = list(ex.map(_make_request, jobs))
    else:
        made = [_make_request(j) for j in jobs]
    return [Request(rid=m[0], xml=m[1], kernel=m[2], wall=m[3], steps=m[4], sites=m[5], shape=m[6]) for m in made]


def poisson_arrivals(requests: Sequence[Request], rate_per_s: float, seed: int = 7) -> None:
    rng = np.random.default_rng(seed)
    t = 0.0
    for r in requests:
        t += float(rng.exponential(1.0 / rate_per_s))
        r.arrival = t


# ---------------------------------------------------------------------------
# Autotuner
# ---------------------------------------------------------------------------

@dataclass
class Tuning:
    sites_per_thread: int
    block: int
    precision: str
    mlups: float
    table: Dict[str, float] = field(default_factory=dict)
    form: str = "persistent"


def autotune(probe: Sequence[Request], tolerance: float = 1e-4, device: int = 0, block_steps: int = 100,
             site_capacity: Optional[int] = None) -> Tuning:
    """Pick the step form (persistent or split), sites per thread, threads per
    block and storage precision, and measure the batch's capacity in MLUPS.

    Precision: FP16 storage is only eligible when the tolerance allows its error
    (about 1e-3 relative in velocity against FP64); otherwise FP32.  Each launch
    shape is timed on a probe batch holding all the given requests at once (the
    device time of a block of steps after a warm-up block), so the probe should
    hold enough sites to fill the device, as a loaded server does."""
    precisions = ["fp32"] + (["fp16"] if tolerance >= 5e-3 else [])
    total = sum(r.sites for r in probe)
    cap = site_capacity or int(total * 1.1) + 64 * len(probe) + 1024
    best = None
    table = {}
    for prec in precisions:
        b = lbm.Batch(cap, cap, max(8, len(probe)), precision=prec, device=device)
        for r in probe:
            b.add_xml(r.xml, r.kernel, r.wall, 10 ** 9)
        for form in ("persistent", "split"):
            for spt in (1, 2):
                for block in (128, 256):
                    b.set_tuning(spt, block, form)
                    b.run(block_steps)          # capture + warm
                    b.run(block_steps)
                    ms, act, _ = b.stats()
                    mlups = act * block_steps / (ms * 1e-3) / 1e6
                    table[f"{prec}/{form}/spt{spt}/b{block}"] = mlups
                    if best is None or mlups > best.mlups:
                        best = Tuning(spt, block, prec, mlups, form=form)
        b.close()
    best.table = table
    return best


def capacity_probe(requests: Sequence[Request], min_sites: int = 8_000_000, max_requests: int = 64) -> List[Request]:
    """The first requests of the stream whose sites add up to min_sites (a
    loaded server's resident set), for the autotuner's capacity measurement."""
    out, n = [], 0
    for r in requests:
        if n >= min_sites or len(out) >= max_requests:
            break
        out.append(r)
        n += r.sites
    return out


# ---------------------------------------------------------------------------
# Server
# ---------------------------------------------------------------------------

class Server:
    """Continuous batching of solve requests on one GPU under an HBM budget.

    Each request is prepared (case parsed, geometry read, storage layout built)
    on a pool of host threads as soon as it arrives, while the device steps the
    resident lattices; admission between blocks is then an upload.  Requests are
    admitted in arrival order as slots and memory free up."""

    def __init__(self, budget_bytes: int, device: int = 0, tuning: Optional[Tuning] = None, block_steps: int = 100,
                 max_lattices: int = 256, general_fraction: float = 0.6, prep_workers: int = 0):
        precision = tuning.precision if tuning else "fp32"
        # Largest site capacity whose arena fits the budget.
        lo, hi = 1024, 1 << 31
        while lo < hi:
            mid = (lo + hi + 1) // 2
            need = lbm.Batch.bytes_for(mid, int(mid * general_fraction), max_lattices, precision)
            if need <= budget_bytes:
                lo = mid
            else:
                hi = mid - 1
        self.site_capacity = lo
        self.batch = lbm.Batch(lo, int(lo * general_fraction), max_lattices, precision=precision, device=device)
        if tuning:
            self.batch.set_tuning(tuning.sites_per_thread, tuning.block, tuning.form)
        self.block_steps = block_steps
        self.queue: deque = deque()
        self.prepared: Dict[int, Future] = {}
        self.pool = ThreadPoolExecutor(max_workers=prep_workers or min(8, os.cpu_count() or 1))
        self.running: Dict[int, Request] = {}
        self.completed: List[Request] = []
        self.site_updates = 0
        self.device_ms = 0.0
        self.blocks = 0
        # Per block: wall seconds since the previous block ended (host work
        # included), site updates made, members resident at its start.
        self.block_log: List[Tuple[float, float, int]] = []
        # Host wall seconds: inside batch.run (launch, graph capture when the
        # membership changed, the wait), admissions, retirements.
        self.host_s = {"run": 0.0, "admit": 0.0, "retire": 0.0}

    def submit(self, r: Request) -> None:
        self.prepared[r.rid] = self.pool.submit(lbm.PreparedLattice, r.xml, r.kernel, r.wall, r.steps)
        self.queue.append(r)

    def _admit(self, now: float) -> None:
        while self.queue:
            r = self.queue[0]
            fut = self.prepared[r.rid]
            if not fut.done() and self.running:
                return                     # keep stepping; admit it after the next block
            try:
                prep = fut.result()
            except lbm.HemeLBError as e:   # the case itself is invalid: retire it as failed
                r.status, r.error = e.code, str(e)
                r.admitted = r.finished = now
                self.completed.append(r)
                self.queue.popleft()
                del self.prepared[r.rid]
                continue
            try:
                slot = self.batch.add_prepared(prep)
            except lbm.HemeLBError as e:
                if e.code == -5:           # no room yet: wait for a retirement (FIFO)
                    if not self.running:
                        raise RuntimeError(f"request {r.rid} ({r.sites} sites) exceeds the whole budget") from e
                    return
                raise
            prep.close()
            del self.prepared[r.rid]
            r.admitted = now
            self.running[slot] = r
            self.queue.popleft()

    def run(self, requests: Sequence[Request], keep_results: bool = False, clock=time.perf_counter) -> None:
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = clock()
        last_end = 0.0
        try:
            while pending or self.queue or self.running:
                now = clock() - t0
                while pending and pending[0].arrival <= now:
                    self.submit(pending.popleft())
                ta = clock()
                self._admit(now)
                self.host_s["admit"] += clock() - ta
                if not self.running:
                    if pending and not self.queue:
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - (clock() - t0))))
                    last_end = clock() - t0  # idle time between requests is no block's
                    continue
                resident = len(self.running)
                updates = 0
                for r in self.running.values():
                    k = min(self.block_steps, r.steps - r.steps_done)
                    r.steps_done += k
                    updates += r.sites * k
                tr = clock()
                done = self.batch.run(self.block_steps)
                self.host_s["run"] += clock() - tr
                ms = self.batch.stats()[0]
                self.device_ms += ms
                self.blocks += 1
                now = clock() - t0
                self.block_log.append((now - last_end, float(updates), resident))
                tt = clock()
                for slot in done:
                    r = self.running.pop(slot)
                    n, t, st = self.batch.info(slot)
                    r.status = st
                    # Work up to the member's own last step, not to the block's end.
                    r.steps_done = r.steps if st == 0 else max(0, min(r.steps, int(t) - 1))
                    self.site_updates += r.sites * r.steps_done
                    if st == 0:          # an unstable lattice is handed back early, without fields
                        res = self.batch.macro(slot)
                        if keep_results:
                            r.result = res
                    r.finished = now
                    self.batch.remove(slot)
                    self.completed.append(r)
                self.host_s["retire"] += clock() - tt
                last_end = now
        finally:
            self.pool.shutdown(wait=True)
        self.wall_s = clock() - t0

    def close(self) -> None:
        """Release the batch's device memory."""
        self.batch.close()

    def report(self) -> Dict[str, float]:
        """Latency percentiles over all requests and over the first and second
        halves of the stream (by arrival: a stationary queue gives the two halves
        the same latencies); aggregate MLUPS counts the site updates of the
        requests that completed (a request whose lattice went unstable is
        retired at once and counted as failed, not as work); device-busy MLUPS
        counts every member's steps up to its own end over the device time."""
        lat = np.array([r.latency for r in self.completed])
        work = sum(r.sites * r.steps for r in self.completed if not r.status)
        failed = [r for r in self.completed if r.status]
        by_arrival = sorted(self.completed, key=lambda r: r.arrival)
        half = len(by_arrival) // 2
        halves = {}
        for name, part in (("first_half", by_arrival[:half]), ("second_half", by_arrival[half:])):
            if part:
                lh = np.array([r.latency for r in part])
                halves[name] = {"requests": len(part), "p50_latency_s": float(np.percentile(lh, 50)),
                                "p99_latency_s": float(np.percentile(lh, 99))}
        return {"requests": len(self.completed), "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
                "halves": halves,
                "aggregate_MLUPS": work / self.wall_s / 1e6, "wall_s": self.wall_s,
                "device_busy_MLUPS": self.site_updates / (self.device_ms * 1e-3) / 1e6 if self.device_ms else 0.0,
                "device_busy_fraction": self.device_ms * 1e-3 / self.wall_s if self.wall_s else 0.0,
                "blocks": self.blocks, "host_s": dict(self.host_s), "device_s": self.device_ms * 1e-3,
                "site_capacity": self.site_capacity, "failed": len(failed),
                "failed_requests": [{"rid": r.rid, "status": r.status, "shape": r.shape, "sites": r.sites}
                                    for r in failed]}


def saturated_window(block_log: Sequence[Tuple[float, float, int]]) -> Dict[str, float]:
    """Rate over the blocks run while at least half of the most members ever
    resident were resident: block_log holds (wall seconds since the previous
    block ended, site updates, members resident) per block."""
    peak = max((b[2] for b in block_log), default=0)
    sat = [b for b in block_log if peak > 0 and b[2] * 2 >= peak]
    wall = sum(b[0] for b in sat)
    return {"MLUPS": sum(b[1] for b in sat) / wall / 1e6 if wall > 0 else 0.0, "blocks": len(sat),
            "wall_s": wall, "peak_resident": peak}


def sustained_rate(requests: Sequence[Request], budget_bytes: int, tuning: Optional[Tuning] = None, device: int = 0,
                   block_steps: int = 200) -> Dict[str, float]:
    """Closed-loop saturation pass: the given requests (the head of the stream)
    all arrive at once and the server runs them to completion under the same
    budget, block length and tuning as the open-loop run.  The sustained rate is
    their work over the wall time of the blocks run while at least half of the
    most members ever resident were still resident -- admissions, retirements
    and block boundaries included, the drain at the end (a few long requests
    left alone on the device) excluded: the rate an arrival process must stay
    below for the queue to be stationary.  The whole pass's rate is reported
    beside it."""
    import copy
    reqs = [copy.copy(r) for r in requests]
    for r in reqs:
        r.arrival = 0.0
        r.admitted = r.finished = None
        r.result = None
        r.status, r.steps_done, r.error = 0, 0, ""
    srv = Server(budget_bytes, device=device, tuning=tuning, block_steps=block_steps)
    srv.run(reqs)
    rep = srv.report()
    srv.close()
    sat = saturated_window(srv.block_log)
    return {"MLUPS": sat["MLUPS"] if sat["wall_s"] > 0 else rep["aggregate_MLUPS"],
            "saturated_blocks": sat["blocks"], "saturated_wall_s": sat["wall_s"], "peak_resident": sat["peak_resident"],
            "whole_pass_MLUPS": rep["aggregate_MLUPS"], "requests": len(reqs), "wall_s": rep["wall_s"],
            "device_busy_MLUPS": rep["device_busy_MLUPS"], "host_s": rep["host_s"], "device_s": rep["device_s"],
            "blocks": rep["blocks"]}


def solve_sequential_fp64(requests: Sequence[Request], device: int = 0) -> Dict[str, float]:
    """The same requests one at a time on the FP64 plain path (create, step, extract)."""
    t0 = time.perf_counter()
    work = 0
    for r in requests:
        sim = lbm.LBM(r.xml, kernel=r.kernel, wall=r.wall, device=device)
        sim.step(r.steps, macro=True)
        sim.GetPropertyCache()
        sim.close()
        work += r.sites * r.steps
    dt = time.perf_counter() - t0
    return {"requests": len(requests), "MLUPS": work / dt / 1e6, "wall_s": dt}


def _main(argv=None) -> None:
    """Resident-batch probe: the first requests of the seeded stream admitted at
    once and stepped for a few blocks; prints the device time per block.

        python -m hemepure_b200.serving --requests 8 --blocks 3 --block-steps 20
    """
    import argparse
    import json
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--requests", type=int, default=8)
    ap.add_argument("--blocks", type=int, default=3)
    ap.add_argument("--block-steps", type=int, default=20)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16"])
    ap.add_argument("--sites-per-thread", type=int, default=2)
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--form", default="persistent", choices=sorted(lbm.BATCH_FORMS))
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    reqs = generate_requests(a.requests, a.out, seed=a.seed)
    total = sum(r.sites for r in reqs)
    b = lbm.Batch(total + 64 * len(reqs) + 1024, total + 1024, max(8, len(reqs)), precision=a.precision)
    b.set_tuning(a.sites_per_thread, a.block, a.form)
    for r in reqs:
        b.add_xml(r.xml, r.kernel, r.wall, 10 ** 9)
    rows = []
    for _ in range(a.blocks):
        b.run(a.block_steps)
        ms, act, _ = b.stats()
        rows.append({"block_ms": ms, "active_sites": act, "MLUPS": act * a.block_steps / (ms * 1e-3) / 1e6})
    print(json.dumps({"requests": len(reqs), "sites": total, "blocks": rows}))
    b.close()


if __name__ == "__main__":
    _main()


# ---------------------------------------------------------------------------
# Several GPUs: independent servers, one per device
# ---------------------------------------------------------------------------

def assign_least_work(requests: Sequence[Request], n_devices: int) -> List[List[Request]]:
    """Each request, in arrival order, to the device with the least work (sites x
    steps) assigned so far; ties to the lower device index.  Independent
    lattices need no exchange, so the devices serve their shares apart."""
    shares: List[List[Request]] = [[] for _ in range(n_devices)]
    load = [0] * n_devices
    for r in sorted(requests, key=lambda q: (q.arrival, q.rid)):
        d = min(range(n_devices), key=lambda k: (load[k], k))
        shares[d].append(r)
        load[d] += r.sites * r.steps
    return shares


def _serve_share(args):
    """One device's share, in its own process: its own CUDA context and server."""
    (device, share, budget_bytes, tuning, block_steps, factory) = args
    make = factory or (lambda dev: Server(budget_bytes, device=dev, tuning=tuning, block_steps=block_steps))
    srv = make(device)
    srv.run(share)
    out = [(r.rid, r.admitted, r.finished, r.status, r.steps_done) for r in srv.completed]
    rep = srv.report()
    if hasattr(srv, "close"):
        srv.close()
    return device, out, rep


class Dispatcher:
    """Spreads a request stream over the GPUs of one node as replicas: one
    `Server` per device, each in its own process (one CUDA context per GPU, as
    one process per GPU), each request assigned on arrival order to the device
    with the least assigned work.  All devices start at the same time, so the
    arrival times keep their meaning; latencies and work come back per request.
    `server_factory(device)` builds a server (a stand-in without a GPU in tests)."""

    def __init__(self, devices: Sequence[int], budget_bytes: int, tuning: Optional[Tuning] = None,
                 block_steps: int = 200, server_factory=None):
        self.devices = list(devices)
        self.budget_bytes, self.tuning, self.block_steps = budget_bytes, tuning, block_steps
        self.factory = server_factory

    def run(self, requests: Sequence[Request]) -> Dict[str, object]:
        import multiprocessing as mp
        shares = assign_least_work(requests, len(self.devices))
        jobs = [(dev, share, self.budget_bytes, self.tuning, self.block_steps, self.factory)
                for dev, share in zip(self.devices, shares)]
        by_rid = {r.rid: r for r in requests}
        t0 = time.perf_counter()
        with ProcessPoolExecutor(max_workers=len(jobs), mp_context=mp.get_context("spawn")) as ex:
            results = list(ex.map(_serve_share, jobs))
        wall = time.perf_counter() - t0
        per_device = {}
        for dev, out, rep in results:
            per_device[dev] = rep
            for rid, admitted, finished, status, steps_done in out:
                r = by_rid[rid]
                r.admitted, r.finished, r.status, r.steps_done = admitted, finished, status, steps_done
        done = [r for r in requests if r.finished is not None]
        lat = np.array([r.latency for r in done]) if done else np.zeros(1)
        work = sum(r.sites * r.steps for r in done if not r.status)
        span = max((rep["wall_s"] for rep in per_device.values()), default=wall)
        return {"devices": len(self.devices), "requests": len(done), "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)), "aggregate_MLUPS": work / span / 1e6 if span else 0.0,
                "wall_s": span, "failed": sum(1 for r in done if r.status),
                "assigned_work": [sum(r.sites * r.steps for r in s) for s in shares], "per_device": per_device}
