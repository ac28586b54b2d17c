"""Benchmark: D3Q19 collide-and-stream on the 4M-site pipe, FP64 plain form.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

A step is one time step over the whole lattice.  The default workload is the
large straight pipe (radius 40, length 800, 4,019,200 fluid sites; LBGK
tau=0.55, BFL walls, parabolic inlet ramped over 1000 steps, Nash pressure
outlet), generated synthetically with the same shapes as the reference's
configuration.  With N > 1 (torchrun), every rank runs its own replica: the
plain form does not shard, so there is no collective on the data path.

Rank 0 prints one JSON line.  `value` is whole-job MLUPS (site updates per
second over all ranks / 1e6) timed with CUDA events on the library's stream,
max over ranks; `e2e` is the same metric measured through the C ABI one
step at a time as a HemePure host drives it (the host hands over the step's
pressure-iolet densities, hb_step(1) uploads the step's iolet row and reads
back the stability word, with a host synchronisation).

The CPU baseline and the reference arm (`--impl reference`) run HemePure's
own code, compiled from its sources into oracle/_ref (single-rank: no MPI
library exists on these machines), as one copy of the lattice per host core
side by side, on a bounded number of steps; where those executables are not
built, the oracle's C restatement runs on all host threads instead.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS & % HBM roofline, FP64 plain vs mixed/batched; p50/p99 solve latency"
WORKLOADS = {
    # name: (description, kernel, wall, algorithmic bytes per site update)
    "pipe_r40": ("straight rigid pipe r=40 L=800 (4,019,200 sites), LBGK tau=0.55, BFL walls, parabolic inlet "
                 "u=0.02 ramped over 1000 steps, Nash pressure outlet rho=1, FP64 plain", "LBGK", "BFL", 304),
    "pipe_r40_short": ("straight rigid pipe r=40 L=200 (1,004,800 sites), same physics as pipe_r40; the case "
                       "the kernel profiles capture", "LBGK", "BFL", 304),
    "pipe_r8": ("straight rigid pipe r=8 L=64 (13,312 sites), LBGK tau=0.8, bounce-back walls, Nash pressure "
                "iolets rho 1.001/0.999, FP64 plain", "LBGK", "SBB", 304),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, dist, device) -> float:
    """The largest of the ranks' values (device timings are reported as the
    slowest rank's); `dist` is torch.distributed or None for one rank."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_mlups(world: int, n_sites: int, steps: int, ms_max: float) -> float:
    """Whole-job MLUPS of `world` replicas each stepping `n_sites` sites `steps`
    times, over the slowest rank's device time `ms_max`."""
    return world * n_sites * steps / (ms_max * 1e-3) / 1e6


def make_workload(name: str, out_dir: str):
    from hemepure_b200 import vessels
    xml, gmy, info = vessels.make_case(name, out_dir)
    return xml, info


def reference_cpu(xml: str, kernel: str, wall: str, n_sites: int, budget_s: float, max_steps: int,
                  warmup: int = 1):
    """HemePure itself (compiled from its own sources, single-rank) on the host
    cores: one copy of the lattice per core side by side, `warmup` untimed
    steps each, then a bounded number of timed steps sized to about `budget_s`
    seconds from a single-copy rate probe.  None when the executables are not
    built on this machine."""
    from oracle import reference as R
    try:
        combo = R.combo_for(xml, kernel, wall)
    except (KeyError, ValueError):
        return None
    if not R.available(combo):
        return None
    probe = R.timed_replicas(xml, kernel, wall, 2, procs=1, warmup=0)
    per_step_s = probe["span_s"] / 2
    # Side by side the copies share memory bandwidth: 16 copies of the 4M-site
    # pipe each step about 1.3x slower than one copy alone on the 16-core hosts.
    steps = int(max(1, min(max_steps, budget_s / max(per_step_s * 1.5, 1e-6))))
    r = R.timed_replicas(xml, kernel, wall, steps, warmup=warmup)
    return {"value": r["MLUPS"], "unit": "MLUPS", "cores": r["procs"], "kind": "reference",
            "cpu_model": r["cpu_model"],
            "sample": f"HemePure's own code (single-rank build, {combo}) as {r['procs']} copies of the full "
                      f"{r['sites']}-site lattice side by side, one per core, {warmup} untimed step(s) then "
                      f"{r['steps']} timed steps each ({r['procs'] * r['sites'] * r['steps']} site updates over "
                      f"{r['span_s']:.1f} s from the first copy's loop start to the last one's end)",
            "single_copy_MLUPS": n_sites / per_step_s / 1e6}


def cpu_baseline(xml: str, kernel: str, wall: str, n_sites: int, budget_s: float = 12.0, threads: int = 0):
    """The oracle (the reference's algorithm restated in C) on the host cores,
    used when the reference's own executables are not built here."""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    sim = O.Simulation(xml, kernel, wall, threads=threads)
    t0 = time.perf_counter()
    sim.run(1)
    one = time.perf_counter() - t0
    steps = max(1, int(budget_s / max(one, 1e-6)))
    t0 = time.perf_counter()
    rc = sim.run(steps)
    dt = time.perf_counter() - t0
    return {"value": n_sites * steps / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{steps} full time steps of the same lattice after 1 warm-up step "
                      f"({n_sites * steps} site updates, {dt:.1f} s, {threads} threads, status {rc})"}


def serving_leg(n_requests: int, device: int, case_root: str):
    """Continuous batching of a seeded stream of vessel solves (FP32-shifted batched
    form): Poisson arrivals at 80% of the sustained rate under a 150 GB budget.

    The autotuner picks the launch shape on a batch holding the stream's first
    requests up to 8M sites (a loaded server's resident set).  The sustained rate
    is measured closed-loop: the stream's first 16 requests all arriving at once,
    served by the same server (admissions, retirements and block boundaries
    included) over the blocks run while it is saturated; the open-loop arrival
    rate is 80% of it, so the open-loop aggregate is bounded by 80% of the
    server's capacity, while the FP64 comparison runs back to back.  The FP64
    comparison solves an evenly spaced sample of the same requests one at a time
    through the plain path, each end to end (case read, layout, upload, steps,
    extraction)."""
    from hemepure_b200 import serving
    budget = 150 * 10 ** 9
    t0 = time.perf_counter()
    reqs = serving.generate_requests(n_requests, os.path.join(case_root, "serving"), seed=2024)
    gen_s = time.perf_counter() - t0
    probe = serving.capacity_probe(reqs)
    tuning = serving.autotune(probe, tolerance=1e-4, device=device)
    sustained = serving.sustained_rate(reqs[:min(16, len(reqs))], budget, tuning, device=device, block_steps=200)
    works = np.array([r.sites * r.steps for r in reqs], dtype=np.float64)
    rate = 0.8 * sustained["MLUPS"] * 1e6 / float(works.mean())
    serving.poisson_arrivals(reqs, rate)
    srv = serving.Server(budget, device=device, tuning=tuning, block_steps=200)
    srv.run(reqs)
    rep = srv.report()
    srv.close()
    sample = reqs[::max(1, len(reqs) // 16)][:16]
    seq = serving.solve_sequential_fp64(sample, device=device)
    rep.update({"stream": f"{n_requests} seeded vessels (pipe / Y-bifurcation / 50-75% stenosis), r~U[6,32], "
                          f"L~U[10,40]r, LBGK/TRT tau~U[0.51,1], pressure or parabolic inlet Re<=300, "
                          f"1000-20000 steps", "storage": tuning.precision,
                "tuning": {"form": tuning.form, "sites_per_thread": tuning.sites_per_thread, "block": tuning.block,
                           "capacity_MLUPS": tuning.mlups, "probe_requests": len(probe),
                           "probe_sites": int(sum(r.sites for r in probe)), "table": tuning.table},
                "sustained": sustained, "arrival_rate_per_s": rate, "offered_MLUPS": 0.8 * sustained["MLUPS"],
                "geometry_generation_s": gen_s,
                "fp64_one_at_a_time_MLUPS": seq["MLUPS"], "fp64_sample_requests": seq["requests"],
                "speedup_vs_fp64_one_at_a_time": rep["aggregate_MLUPS"] / seq["MLUPS"],
                # Both sides closed-loop (requests back to back, no arrival gaps): the
                # server saturated against the plain path solving one after another.
                "saturated_speedup_vs_fp64_one_at_a_time": sustained["MLUPS"] / seq["MLUPS"]})
    return rep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pipe_r40", choices=sorted(WORKLOADS))
    ap.add_argument("--case-dir", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=64,
                    help="requests in the serving leg (0 skips it; 512 is the full stream)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    desc, kernel, wall, bytes_per_site = WORKLOADS[args.workload]
    warmup = max(3, args.warmup)

    if args.impl == "reference" and rank != 0:
        return  # the reference arm runs on rank 0 only; the other ranks exit without work
    case_root = args.case_dir or os.path.join(tempfile.gettempdir(), f"hemeb200_bench_{os.getuid()}")
    case_dir = os.path.join(case_root, f"{args.workload}_rank{rank}")
    xml, info = make_workload(args.workload, case_dir)
    n_sites = info.fluid_sites
    config = {"workload": args.workload + ": " + desc, "sites": n_sites, "kernel": kernel, "wall": wall,
              "storage": "fp64", "l2": "inputs larger than L2: two 19-plane FP64 buffers of %.2f GB each"
              % (19 * n_sites * 8 / 1e9), "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}

    if args.impl == "reference":
        # HemePure itself, compiled from its own sources (oracle/_ref), one copy per
        # host core; its C restatement on all host threads where it is not built.
        base = reference_cpu(xml, kernel, wall, n_sites, budget_s=60.0, max_steps=args.steps, warmup=warmup)
        if base is None:
            base = cpu_baseline(xml, kernel, wall, n_sites, budget_s=120.0)
        v = base["value"]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": warmup, "ms_per_step": n_sites / (v * 1e6) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config, "cpu_baseline": base,
                "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod
        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from hemepure_b200 import lbm

    sim = lbm.LBM(xml, kernel=kernel, wall=wall, device=local)
    sim.step(warmup)

    # Timed region: K steps, CUDA events on the library's stream.
    sampler = ClockSampler(local)
    sampler.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.step(args.steps)
    wall_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    ms, launches = sim.last_step_timing()
    clocks = sampler.stop()
    ms = max_over_ranks(ms, dist, f"cuda:{local}")
    value = replica_mlups(world, n_sites, args.steps, ms)

    # Roofline of the dominant kernel (the plain-bulk kernel, three quarters of the
    # step): per-launch CUDA events.  The step's launch pair (bulk and boundary
    # kernels side by side, as hb_step issues them) is timed beside it.
    prof_steps = 200
    s_ms, b_ms, g_ms = sim.profile_steps(prof_steps)
    from hemepure_b200.lbm import Geometry, read_case
    p_case, gmy = read_case(xml, kernel)
    lay = Geometry(gmy).layout(p_case, wall)
    step_launch_ms = s_ms / prof_steps
    bulk_launch_ms = b_ms / prof_steps
    achieved = bytes_per_site * lay["bulk_sites"] / (bulk_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as fh:
            tj = json.load(fh)
        if tj.get("workload") == args.workload and tj.get("kernel") == "k_bulk":
            traffic = tj.get("bytes_per_launch")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "k_bulk (plain bulk sites)", "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": bytes_per_site * lay["bulk_sites"], "launch_ms": bulk_launch_ms,
                "boundary_kernel_alone_ms": g_ms / prof_steps,
                "step_launches": {"kernels": "k_bulk + k_general_walls + k_general side by side", "ms": step_launch_ms,
                                  "achieved": bytes_per_site * n_sites / (step_launch_ms * 1e-3) / 1e9},
                "whole_step_frac": (bytes_per_site * n_sites / (ms / args.steps * 1e-3) / 1e9) / peak}

    # End to end through the C ABI, as a HemePure host drives it: per step the
    # host's BoundaryValues hand over the pressure-iolet densities
    # (hb_set_iolet_densities from host memory), hb_step(1) uploads that step's
    # iolet row (96 doubles) and reads back the stability word, host-synchronised.
    e2e_steps = min(args.steps, 500)
    din = np.ones(max(1, p_case.n_inlets))[:p_case.n_inlets]
    dout = np.ones(max(1, p_case.n_outlets))[:p_case.n_outlets]
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.SetIoletDensities(din, dout)
        sim.step(1)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    sim.SetIoletDensities()
    e2e = {"value": world * n_sites * e2e_steps / e2e_s / 1e6, "unit": "MLUPS", "h2d_bytes_per_step": 96 * 8,
           "d2h_bytes_per_step": 4, "steps": e2e_steps,
           "note": "per step: hb_set_iolet_densities (the outlet's density from host memory), hb_step(1) "
                   "uploading that step's 96-double iolet row, 4-byte stability word read back, host sync"}

    # The shifted low-precision forms on the same lattice (same step count).
    forms = {"fp64": {"MLUPS": value / world, "bytes_per_site": 304,
                      "whole_step_frac": roofline["whole_step_frac"]}}
    for prec, nbytes in (("fp32", 152), ("fp16", 76)):
        try:
            ms_p = lbm.LBM(xml, kernel=kernel, wall=wall, precision=prec, device=local)
            ms_p.step(warmup)
            ms_p.step(args.steps)
            t_ms, _ = ms_p.last_step_timing()
            _, b_p, _ = ms_p.profile_steps(prof_steps)
            ms_p.close()
            per = t_ms / args.steps
            forms[prec] = {"MLUPS": n_sites / (per * 1e-3) / 1e6, "ms_per_step": per, "bytes_per_site": nbytes,
                           "whole_step_frac": nbytes * n_sites / (per * 1e-3) / 1e9 / peak,
                           "bulk_kernel_GBs": nbytes * lay["bulk_sites"] / (b_p / prof_steps * 1e-3) / 1e9}
        except Exception as e:  # report, do not hide
            forms[prec] = {"error": str(e)}

    serving_rep = None
    if world == 1 and args.serving_requests > 0:
        try:
            serving_rep = serving_leg(args.serving_requests, local, case_root)
        except Exception as e:  # report, do not hide
            serving_rep = {"error": repr(e)}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = reference_cpu(xml, kernel, wall, n_sites, budget_s=15.0, max_steps=args.steps)
        if base is None:
            base = cpu_baseline(xml, kernel, wall, n_sites)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "roofline": roofline, "cpu_baseline": base, "e2e": e2e, "clocks": clocks, "forms": forms,
                "serving": serving_rep,
                "gpu_launches": int(launches), "wall_s": wall_s}
        print(json.dumps(line), flush=True)
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
