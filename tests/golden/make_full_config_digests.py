"""Digests of HemePure's own results on the full-size workloads (test fixtures).

Runs the reference solver compiled from its sources (oracle/_ref, built by
oracle/ref/build_ref.sh where the reference tree is present) on the synthetic
workloads at their stated sizes, and records SHA-256 digests of the
distributions, density, velocity and wall shear stress after the step count,
in the reference's contiguous site order and native byte order (float64
little-endian).  The GPU tests hash their own FP64 results the same way, so a
match means bit-for-bit equality with HemePure at full size without carrying
gigabytes of fixtures.

    python tests/golden/make_full_config_digests.py [c2] [c3]

C2: straight pipe r=40 L=800 (4,019,200 sites), LBGK, BFL, parabolic Ladd inlet,
Nash outlet, 1000 steps (the step the parity target names).  C3: Y-bifurcation
(parent r=32, daughters r=25 at +-35 degrees), TRT, GZS, cosine inlet, two WK3
outlets, 1000 steps.  Single-rank runs take about 8 and 20 minutes.
"""

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hemepure_b200 import vessels  # noqa: E402
from oracle import reference as R  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "full_config_digests.json")

CONFIGS = {
    # key: (workload, kernel, wall, steps)
    "c2": ("pipe_r40", "LBGK", "BFL", 1000),
    "c3": ("bifurcation", "TRT", "GZS", 1000),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def fields_digest(f, rho, u, wss) -> dict:
    return {"f": digest(f), "rho": digest(rho), "u": digest(u), "wss": digest(wss)}


def main(keys):
    R.build()
    for key in keys:
        workload, kernel, wall, steps = CONFIGS[key]
        d = tempfile.mkdtemp(prefix=f"full_{key}_")
        xml, gmy, info = vessels.make_case(workload, d)
        run = R.Run(xml, kernel, wall, steps, timeout=6 * 3600)
        rec = fields_digest(run["f"], run["rho"], run["u"], run["wss"])
        rec.update({"workload": workload, "kernel": kernel, "wall": wall, "steps": steps, "sites": int(run["n"]),
                    "max_abs_u": float(np.max(np.abs(run["u"]))), "sum_f": float(np.sum(run["f"])),
                    "seconds": run.wall_seconds, "combo": run.combo})
        have = json.load(open(OUT)) if os.path.exists(OUT) else {}  # runs of other keys may have finished
        have[key] = rec
        with open(OUT + ".tmp", "w") as fh:
            json.dump(have, fh, indent=1, sort_keys=True)
        os.replace(OUT + ".tmp", OUT)
        print(key, json.dumps(rec), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CONFIGS))
