"""The workloads at their stated sizes and step counts (opt-in: they take minutes).

    HEMEB200_FULL_CONFIGS=1 [HEMEB200_FULL_CONFIGS_REPORT=path.json] pytest -m gpu tests/test_gpu_full_configs.py

* Straight pipe r=40 L=800 (4,019,200 sites; LBGK, BFL, parabolic inlet ramped
  over 1000 steps, Nash outlet), FP64: after 1000 steps the distributions,
  density, velocity and wall shear stress equal HemePure's own results bit for
  bit (SHA-256 digests of the reference's run, tests/golden/full_config_digests.json,
  made by tests/golden/make_full_config_digests.py).
* Y-bifurcation (parent r=32 L=400, daughters r=25 L=400 at +-35 degrees; TRT
  with magic parameter 3/16, GZS, cosine inlet, two WK3 outlets), FP64 equal to
  HemePure after 1000 steps the same way.  As stated (tau+ = 0.52) the run
  diverges before step 8000 (the reference's scheme, FP64 bit-identical to it),
  so FP32-shifted storage is compared with FP64 at 4000 steps, and again at the
  full 8000 steps with tau+ = 0.55: velocity and wall shear stress within 1e-4.
* Stenosed artery r=48 L=1200 narrowing to r=24 (LBGK+LES, sponge layer at the
  outlet, pulsatile parabolic inlet).  As stated FP64 diverges near step 4300,
  so FP32- and FP16-shifted storage are compared with FP64 at 3000 steps, and
  for the full 20,000 steps on a variant that is stable (tau 0.6, half the
  inflow); errors stated (FP32 within 1e-3 of FP64 in velocity on the
  variant), FP16 reported (stable or not, error stated).

Errors are max |a - b| / max |b| over the field (pressure as (rho - 1) cs^2,
wall shear stress over wall sites).  With a report path, each test writes its
figures there.
"""

import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.environ.get("HEMEB200_FULL_CONFIGS"),
                                 reason="full-size workloads take minutes: set HEMEB200_FULL_CONFIGS=1"),
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

HERE = os.path.dirname(os.path.abspath(__file__))


def digests() -> dict:
    with open(os.path.join(HERE, "golden", "full_config_digests.json")) as fh:
        return json.load(fh)


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def rel(a, b) -> float:
    s = float(np.max(np.abs(b)))
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / s) if s > 0 else 0.0


def errors(fields, ref):
    (rho, u, w), (r0, u0, w0) = fields, ref
    wall = w0 < 1e300
    return {"u": rel(u, u0), "p": rel((rho - 1.0) / 3.0, (r0 - 1.0) / 3.0), "wss": rel(w[wall], w0[wall])}


def report(key, rec):
    print(key, json.dumps(rec))
    path = os.environ.get("HEMEB200_FULL_CONFIGS_REPORT")
    if path:
        have = json.load(open(path)) if os.path.exists(path) else {}
        have[key] = rec
        with open(path, "w") as fh:
            json.dump(have, fh, indent=1, sort_keys=True)


def _case(name, **variant):
    from hemepure_b200 import vessels
    d = tempfile.mkdtemp(prefix=f"full_{name}_")
    return vessels.make_case(name, d, **variant)


def _equals_reference(key, xml, kernel, wall, steps):
    import time

    from hemepure_b200 import lbm
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    t0 = time.perf_counter()
    sim.step(steps, macro=True)
    gpu_s = time.perf_counter() - t0
    f = sim.GetFOld()
    rho, u, w = sim.GetPropertyCache()
    got = {"f": digest(f), "rho": digest(rho), "u": digest(u), "wss": digest(w)}
    want = digests()[key]
    rec = {"sites": int(sim.n), "steps": steps, "gpu_seconds": gpu_s,
           "equal_to_reference": {k: got[k] == want[k] for k in got}, "max_abs_u": float(np.max(np.abs(u)))}
    sim.close()
    return rec, got, want, (rho, u, w)


def test_c2_pipe_fp64_equals_hemepure_at_step_1000():
    xml, gmy, info = _case("pipe_r40")
    rec, got, want, _ = _equals_reference("c2", xml, "LBGK", "BFL", 1000)
    report("c2_pipe_r40_fp64", rec)
    assert info.fluid_sites == digests()["c2"]["sites"] == 4019200
    assert got == {k: want[k] for k in got}


def _divergence_step(xml, kernel, wall, limit, chunk):
    """FP64 steps until the run goes unstable (or `limit`): the last step it was
    stable at, in multiples of `chunk`."""
    from hemepure_b200 import lbm
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    t = 0
    try:
        while t < limit:
            sim.step(chunk)
            t += chunk
    except lbm.Unstable:
        pass
    sim.close()
    return t


def _fields_at(xml, kernel, wall, steps, precisions):
    from hemepure_b200 import lbm
    out, status = {}, {}
    for prec in precisions:
        sim = lbm.LBM(xml, kernel=kernel, wall=wall, precision=prec)
        try:
            sim.step(steps, macro=True)
            out[prec] = sim.GetPropertyCache()
            status[prec] = "stable"
        except lbm.Unstable:
            status[prec] = "unstable"
        sim.close()
    return out, status


def test_c3_bifurcation_fp64_and_fp32():
    """As stated (tau+ = 0.52): FP64 equals HemePure at step 1000; the run
    diverges before its 8000 steps through the Nash pressure inlet's own-velocity
    mode at the inlet plane's centre (the reference's scheme, FP64 bit-identical
    to it), so FP32 is compared with FP64 at 4000 steps.  With tau+ = 0.55 the
    same vessel is stable and FP32 is compared at the full 8000 steps."""
    xml, gmy, info = _case("bifurcation")
    rec, got, want, _ = _equals_reference("c3", xml, "TRT", "GZS", 1000)
    assert got == {k: want[k] for k in got}
    rec["fp64_last_stable_step"] = _divergence_step(xml, "TRT", "GZS", 8000, 250)
    fields, status = _fields_at(xml, "TRT", "GZS", 4000, ("fp64", "fp32"))
    rec["status_at_4000"] = status
    err = errors(fields["fp32"], fields["fp64"])
    rec["fp32_vs_fp64_at_4000"] = err
    assert err["u"] <= 1e-4 and err["wss"] <= 1e-4, err
    xml2, gmy2, info2 = _case("bifurcation", tau=0.55)
    fields2, status2 = _fields_at(xml2, "TRT", "GZS", 8000, ("fp64", "fp32"))
    assert status2 == {"fp64": "stable", "fp32": "stable"}, status2
    err2 = errors(fields2["fp32"], fields2["fp64"])
    rec["variant_tau_0.55_fp32_vs_fp64_at_8000"] = err2
    report("c3_bifurcation", rec)
    assert err2["u"] <= 1e-4 and err2["wss"] <= 1e-4, err2


# Stable in FP64 for the full 20000 steps (checked every 4000 steps); tau 0.55
# with a quarter of the inflow, the same Reynolds number, is stable too, while
# tau 0.502 / 0.51 / 0.52 with 0.1 / 0.25 / 0.5 of the inflow diverge by step
# 8000 / 8000 / 12000.
C4_VARIANT = {"tau": 0.6, "inflow_scale": 0.5}


def test_c4_stenosis_les_fp64_fp32_fp16():
    """As stated (tau = 0.502, inlet peak 0.05 (1 + sin/2), 75 % area reduction):
    the throat speed passes Mach 0.5 and FP64 diverges near step 4300, so FP32
    and FP16 are compared with FP64 at 3000 steps.  A variant with a larger
    relaxation time and a lower inflow is stable for the full 20000 steps in
    FP64, and FP32 and FP16 are compared there.

    The errors are stated, not held to the laminar configs' 1e-4: with the
    relaxation rate at 1.992 and an LES eddy viscosity that depends on the
    non-equilibrium part itself, rounding of the stored deviations grows in the
    jet (measured FP32: u 9.2e-4, WSS 1.1e-2 at step 3000 as stated; u 4.3e-4,
    WSS 9.4e-4 at step 20000 on the variant).  The bounds below hold the
    measured figures with a factor of two of margin, so that a regression shows."""
    xml, gmy, info = _case("stenosis")
    rec = {"sites": info.fluid_sites}
    rec["fp64_last_stable_step"] = _divergence_step(xml, "LBGKLESSL", "BFL", 20000, 250)
    fields, status = _fields_at(xml, "LBGKLESSL", "BFL", 3000, ("fp64", "fp32", "fp16"))
    rec["status_at_3000"] = status
    assert status["fp64"] == "stable" and status["fp32"] == "stable", status
    for prec in ("fp32", "fp16"):
        if prec in fields:
            rec[f"{prec}_vs_fp64_at_3000"] = errors(fields[prec], fields["fp64"])
    if C4_VARIANT["tau"] is not None:
        xml2, gmy2, info2 = _case("stenosis", tau=C4_VARIANT["tau"], inflow_scale=C4_VARIANT["inflow_scale"])
        fields2, status2 = _fields_at(xml2, "LBGKLESSL", "BFL", 20000, ("fp64", "fp32", "fp16"))
        rec["variant"] = dict(C4_VARIANT)
        rec["variant_status_at_20000"] = status2
        for prec in ("fp32", "fp16"):
            if prec in fields2:
                rec[f"variant_{prec}_vs_fp64_at_20000"] = errors(fields2[prec], fields2["fp64"])
    report("c4_stenosis", rec)
    assert rec["fp32_vs_fp64_at_3000"]["u"] <= 2e-3 and rec["fp32_vs_fp64_at_3000"]["wss"] <= 2.5e-2, rec
    if C4_VARIANT["tau"] is not None:
        assert rec["variant_status_at_20000"]["fp64"] == "stable"
        assert rec["variant_status_at_20000"]["fp32"] == "stable"
        assert rec["variant_fp32_vs_fp64_at_20000"]["u"] <= 1e-3, rec
        assert rec["variant_fp32_vs_fp64_at_20000"]["wss"] <= 2e-3, rec
