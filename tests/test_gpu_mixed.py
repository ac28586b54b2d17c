"""Shifted low-precision storage (FP32, FP16) against the FP64 oracle.

The error of velocity, pressure and wall shear stress is stated per
configuration (printed, and bounded here): each is the largest absolute
difference divided by the field's largest magnitude (pressure as the deviation
p - p0 = (rho - 1) cs^2).  FP32 storage must stay within 1e-4 of FP64 for
velocity and wall shear stress."""

import numpy as np
import pytest

from conftest import SMALL_CASES, make_small_case
from hemepure_b200 import lbm
from oracle import oracle as O

pytestmark = pytest.mark.gpu

BOUNDS = {"fp32": 1e-4, "fp16": 5e-2}
_oracle_cache = {}


def rel(a, b):
    s = np.max(np.abs(b))
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / s) if s > 0 else 0.0


def oracle_fields(case_dir, key):
    if key not in _oracle_cache:
        xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
        orc = O.Simulation(xml, kernel, wall)
        assert orc.run(steps, macro=True) == 0
        _oracle_cache[key] = orc.macro()
    return _oracle_cache[key]


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_shifted_storage_error(case_dir, key, precision):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall, precision=precision)
    gpu.step(steps, macro=True)
    rho_g, u_g, w_g = gpu.GetPropertyCache()
    rho_o, u_o, w_o = oracle_fields(case_dir, key)
    wall_sites = w_o < 1e300
    err = {"u": rel(u_g, u_o), "p": rel((rho_g - 1.0) / 3.0, (rho_o - 1.0) / 3.0),
           "wss": rel(w_g[wall_sites], w_o[wall_sites]) if wall_sites.any() else 0.0}
    print(f"{key} {precision} after {steps} steps: error vs FP64 {err}")
    assert err["u"] <= BOUNDS[precision] and err["wss"] <= BOUNDS[precision], err
    # distributions round-trip through the shifted storage
    f = gpu.GetFOld()
    assert np.all(np.isfinite(f))


def test_fp32_set_get_round_trip(case_dir):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_r8")
    a = lbm.LBM(xml, kernel=kernel, wall=wall, precision="fp32")
    a.step(10)
    f = a.GetFOld()
    b = lbm.LBM(xml, kernel=kernel, wall=wall, precision="fp32")
    b.SetFs(f)
    b.time_step = a.time_step
    a.step(5)
    b.step(5)
    assert np.max(np.abs(a.GetFOld() - b.GetFOld())) < 1e-7
