"""HemePure itself, compiled from its own sources, as the parity oracle.

Test infrastructure only: the tests, the smoke check and the benchmark's
reference arm run it as the checker or as the timed CPU baseline; the product
library never imports it.

`oracle/ref/build_ref.sh` compiles the reference's translation units, unmodified
and where they lie in the reference tree, into one single-rank executable per
kernel / boundary-condition combination (the reference fixes those at compile
time, src/lb/lb.h:37-48), with the stand-ins in `oracle/ref/shim` for MPI,
boost, ParMETIS, ctemplate and XDR.  `oracle/ref/harness.cc` wires the solver
together as SimulationMaster::Initialise does (src/SimulationMaster.cc:126-285),
steps it, and dumps the distributions and the density, velocity and wall shear
stress caches of the last step in the reference's own contiguous site order.
The executables land in `oracle/_ref/<combo>/hemepure_ref`; they are built
where the reference sources exist and travel with the repository snapshot.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
import time
import xml.etree.ElementTree as ET
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SCRIPT = os.path.join(HERE, "ref", "build_ref.sh")
DEFAULT_SOURCES = "/root/reference"

# (kernel, wall, inlet streamer, outlet streamer) -> build folder.  The inlet and
# outlet streamers follow the iolets' XML condition types: pressure -> Nash
# zeroth-order pressure, velocity -> Ladd (src/configuration/SimConfig.cc:238-260
# rejects a case whose conditions do not match the build).
COMBOS = {
    ("LBGK", "SBB", "NASH", "NASH"): "lbgk_sbb_nash",
    ("LBGK", "SBB", "LADD", "NASH"): "lbgk_sbb_ladd_nash",
    ("LBGK", "BFL", "LADD", "NASH"): "lbgk_bfl_ladd_nash",
    ("TRT", "GZS", "NASH", "NASH"): "trt_gzs_nash",
    ("TRT", "GZS", "LADD", "NASH"): "trt_gzs_ladd_nash",
    ("LBGKLESSL", "BFL", "LADD", "NASH"): "les_bfl_ladd_nash",
}


def sources() -> Optional[str]:
    """The reference source tree, if this machine has it."""
    p = os.environ.get("HEMEPURE_REFERENCE", DEFAULT_SOURCES)
    return p if os.path.isdir(os.path.join(p, "src")) else None


def binary(combo: str) -> str:
    return os.path.join(OUT, combo, "hemepure_ref")


def available(combo: str) -> bool:
    return os.access(binary(combo), os.X_OK)


def build(combos=None) -> bool:
    """Compile the reference executables (all combos by default).  Returns False
    when the reference sources are not on this machine; prebuilt executables
    are then used as they are."""
    src = sources()
    if src is None:
        return False
    env = dict(os.environ, HEMEPURE_REFERENCE=src)
    subprocess.run(["bash", SCRIPT] + list(combos or []), check=True, env=env,
                   stdout=subprocess.DEVNULL)
    return True


def _streamer(group: ET.Element) -> str:
    kinds = {c.get("type") for c in group.iter("condition")}
    if kinds <= {"pressure"}:
        return "NASH"
    if kinds == {"velocity"}:
        return "LADD"
    raise ValueError(f"mixed iolet condition types {sorted(kinds)}: the reference needs one streamer per group")


def combo_for(xml_path: str, kernel: str, wall: str) -> str:
    root = ET.parse(xml_path).getroot()
    key = (kernel, wall, _streamer(root.find("inlets")), _streamer(root.find("outlets")))
    if key not in COMBOS:
        raise KeyError(f"no reference build for {key}")
    return COMBOS[key]


def load_dump(path: str) -> Dict[str, np.ndarray]:
    """Read the harness's dump (layout in oracle/ref/harness.cc)."""
    raw = open(path, "rb").read()
    if raw[:8] != b"HBREFDMP":
        raise ValueError(f"{path}: not a reference dump")
    n, steps, stability = (int(v) for v in np.frombuffer(raw, np.int64, 3, 8))
    off = 32
    out: Dict[str, np.ndarray] = {"n": n, "steps": steps, "stability": stability}
    for name, dt, k in (("coords", np.int64, 3), ("f", np.float64, 19), ("rho", np.float64, 1),
                        ("u", np.float64, 3), ("wss", np.float64, 1)):
        cnt = n * k
        a = np.frombuffer(raw, dt, cnt, off)
        off += cnt * 8
        out[name] = a.reshape(n, k) if k > 1 else a
    if off != len(raw):
        raise ValueError(f"{path}: {len(raw) - off} trailing bytes")
    return out


class Run:
    """One run of the reference solver: `steps` time steps of the case file."""

    def __init__(self, xml_path: str, kernel: str, wall: str, steps: int, combo: Optional[str] = None,
                 timeout: float = 3600.0):
        self.combo = combo or combo_for(xml_path, kernel, wall)
        exe = binary(self.combo)
        if not os.access(exe, os.X_OK):
            raise FileNotFoundError(f"{exe} is not built (oracle/ref/build_ref.sh {self.combo})")
        work = tempfile.mkdtemp(prefix="hemepure_ref_")
        try:
            dump = os.path.join(work, "dump.bin")
            t0 = time.perf_counter()
            p = subprocess.run([exe, os.path.abspath(xml_path), os.path.join(work, "out"), str(int(steps)), dump],
                               cwd=os.path.dirname(os.path.abspath(xml_path)), capture_output=True, text=True,
                               timeout=timeout)
            self.wall_seconds = time.perf_counter() - t0
            if p.returncode != 0:
                raise RuntimeError(f"hemepure_ref failed ({p.returncode}): {p.stderr[-2000:]}")
            self.log = p.stderr
            self.data = load_dump(dump)
        finally:
            shutil.rmtree(work, ignore_errors=True)
        self.mlups = None
        for line in self.log.splitlines():
            if line.startswith("hemepure_ref:") and "MLUPS" in line:
                self.mlups = float(line.split(",")[-1].split()[0])

    def __getitem__(self, key):
        return self.data[key]


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _mem_available_bytes() -> int:
    try:
        with open("/proc/meminfo") as fh:
            for line in fh:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def timed_replicas(xml_path: str, kernel: str, wall: str, steps: int, procs: int = 0, bytes_per_site: int = 700,
                   warmup: int = 1, timeout: float = 1800.0) -> Dict[str, object]:
    """Aggregate throughput of HemePure on the host cores.

    The reference is built single-rank here (there is no MPI library on these
    machines), so the host's cores are used by `procs` independent copies of the
    same lattice run side by side, one process per core: every copy reads and
    sets up the case and runs `warmup` untimed steps, all wait at a common
    start barrier, then each steps `steps` times.  The result is all copies'
    site updates over the span from the first loop start to the last loop end.
    Every copy does the per-site work of an MPI rank over the same cores
    without its halo exchange.  `procs` defaults to the
    core count, capped so the copies fit in half the available memory
    (`bytes_per_site` per copy and site: two FP64 distribution arrays, the
    64-bit neighbour table and the site data)."""
    combo = combo_for(xml_path, kernel, wall)
    exe = binary(combo)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"{exe} is not built")
    root = ET.parse(xml_path).getroot()
    cores = os.cpu_count() or 1
    work = tempfile.mkdtemp(prefix="hemepure_ref_rep_")
    try:
        # Site count from a one-step probe (also warms the page cache for the geometry).
        probe = subprocess.run([exe, os.path.abspath(xml_path), os.path.join(work, "probe"), "1", "-"],
                               cwd=os.path.dirname(os.path.abspath(xml_path)), capture_output=True, text=True,
                               timeout=timeout)
        if probe.returncode != 0:
            raise RuntimeError(f"hemepure_ref failed: {probe.stderr[-2000:]}")
        n_sites = int(probe.stderr.strip().splitlines()[-1].split()[1])
        if procs <= 0:
            mem = _mem_available_bytes()
            fit = max(1, int(0.5 * mem // max(1, n_sites * bytes_per_site))) if mem else cores
            procs = max(1, min(cores, fit))
        ready = os.path.join(work, "sync")
        os.makedirs(ready)
        env = dict(os.environ, HB_REF_READY=ready)
        ps = [subprocess.Popen([exe, os.path.abspath(xml_path), os.path.join(work, f"o{i}"), str(int(steps)), "-",
                                str(int(warmup))],
                               cwd=os.path.dirname(os.path.abspath(xml_path)), env=env,
                               stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True)
              for i in range(procs)]
        t_end = time.monotonic() + timeout
        while len([f for f in os.listdir(ready) if f.startswith("ready.")]) < procs:
            if any(p.poll() not in (None, 0) for p in ps) or time.monotonic() > t_end:
                for p in ps:
                    p.kill()
                raise RuntimeError("a reference copy failed before the start barrier")
            time.sleep(0.01)
        open(os.path.join(ready, "go"), "w").close()
        starts, ends = [], []
        for p in ps:
            _, err = p.communicate(timeout=max(1.0, t_end - time.monotonic()))
            if p.returncode != 0:
                raise RuntimeError(f"hemepure_ref failed: {err[-2000:]}")
            words = err.strip().splitlines()[-1].replace(",", " ").split()
            k = words.index("loop")
            starts.append(float(words[k + 1]))
            ends.append(float(words[k + 2]))
        span = max(ends) - min(starts)
        return {"MLUPS": procs * n_sites * steps / span / 1e6, "procs": procs, "sites": n_sites, "steps": steps,
                "warmup": warmup,
                "span_s": span, "per_copy_s": [e - s for s, e in zip(starts, ends)], "combo": combo,
                "cpu_model": cpu_model()}
    finally:
        shutil.rmtree(work, ignore_errors=True)
