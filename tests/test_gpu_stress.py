"""Stress caches and the stress-type .xtr fields on the GPU path.

The reference fills its MacroscopicPropertyCache stress entries in
BaseStreamer::UpdateMinsAndMaxes (src/lb/streamers/BaseStreamer.h:123-217) from
the momentum flux tensor of the step's collision (Lattice.h:983-1180, 1353-1383),
and LocalPropertyOutput::Write converts them with the UnitConverter
(src/extraction/LocalPropertyOutput.cc:255-326, src/util/UnitConverter.h:52-96).
FP64: the library's caches equal the oracle's bit for bit on every physics
combination; the .xtr values equal the caches converted as the reference does.
"""

import numpy as np
import pytest

from conftest import SMALL_CASES, make_small_case
from hemepure_b200 import lbm
from oracle import oracle as O
from test_gpu_extraction import read_xtr, units

pytestmark = pytest.mark.gpu

FIELDS = list(lbm.STRESS_FIELDS)
STEPS = 200


@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_stress_caches_bit_exact(case_dir, key):
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, key)
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall)
    orc = O.Simulation(xml, kernel, wall)
    gpu.step(STEPS, macro=True, stress=True)
    assert orc.run(STEPS, macro=True) == 0
    _, _, wss = orc.macro()
    walls = wss < 1e300
    for f in FIELDS:
        g, o = gpu.GetStress(f), orc.stress(f)
        assert g.shape == o.shape
        differ = int(np.sum(~((g == o) | (np.isnan(g) & np.isnan(o)))))
        assert differ == 0, (key, f, differ)
        if f.endswith("traction"):
            assert np.all(g[~walls] == 0.0)
    assert np.max(gpu.GetStress("vonmisesstress")) > 0.0


def test_stress_needs_a_stress_step(case_dir):
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_r8")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(5, macro=True)
    with pytest.raises(lbm.HemeLBError):
        sim.GetStress("vonmisesstress")
    # the phase API fills the caches the same way as hb_step
    sim.RequestComms()
    sim.PreSend()
    sim.PreReceive(macro=True, stress=True)
    sim.PostReceive()
    sim.EndIteration()
    ref = lbm.LBM(xml, kernel=kernel, wall=wall)
    ref.step(6, macro=True, stress=True)
    for f in FIELDS:
        assert np.array_equal(sim.GetStress(f), ref.GetStress(f))
    # a later step without stress invalidates them
    sim.step(1, macro=True)
    with pytest.raises(lbm.HemeLBError):
        sim.GetStress("shearrate")


def test_xtr_stress_fields(case_dir, tmp_path):
    """Every OutputField type in one record, converted as the reference converts it."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(60, macro=True, stress=True)
    types = ["pressure", "velocity", "shearstress", "vonmisesstress", "shearrate", "stresstensor", "traction",
             "tangentialprojectiontraction", "normalprojectiontraction", "wallextension", "distributions", "mpirank"]
    path = tmp_path / "all.xtr"
    sim.WriteXtr(path, types)
    x = read_xtr(path)
    assert [(n, w) for n, w, _ in x["fields"]] == [
        ("pressure", 1), ("velocity", 3), ("shearstress", 1), ("vonmisesstress", 1), ("shearrate", 1),
        ("stresstensor", 6), ("traction", 3), ("tangentialprojectiontraction", 3), ("normalprojectiontraction", 3),
        ("wallextension", 1), ("distributions", 19), ("mpirank", 1)]
    (label, coords, vals), = x["records"]
    dx, dt, p_unit, v_unit = units(xml, kernel)
    st = {f: sim.GetStress(f) for f in FIELDS}
    normal = lbm.Geometry(gmy).tables()["wall_normal"]
    ref_p_mmhg = 0.0
    mmhg = 133.3223874
    with np.errstate(over="ignore", invalid="ignore"):
        expect = {
            "vonmisesstress": st["vonmisesstress"] * p_unit,
            "shearrate": st["shearrate"] / dt,
            "stresstensor": st["stresstensor"] * p_unit + np.array([1, 0, 0, 1, 0, 1]) * (-ref_p_mmhg * mmhg),
            "traction": st["traction"] * (v_unit * v_unit * 1000.0) - normal * ref_p_mmhg * mmhg,
            "tangentialprojectiontraction": st["tangentialprojectiontraction"] * p_unit,
            "normalprojectiontraction": st["normalprojectiontraction"] * p_unit,
        }
        for f, e in expect.items():
            assert np.array_equal(vals[f], e.astype(np.float32), equal_nan=True), f
    assert np.all(vals["wallextension"] == 0.0) and np.all(vals["mpirank"] == 0.0)
    # the reference's traction conversion leaves sites without a wall normal non-finite
    no_normal = ~np.isfinite(normal[:, 0])
    assert np.any(no_normal) and np.all(np.isnan(vals["traction"][no_normal]))
    walls = np.isfinite(normal[:, 0])
    assert np.all(np.isfinite(vals["traction"][walls]))
    # tangential + normal projection = traction at the wall (lattice units)
    t = st["traction"][walls]
    assert np.allclose(st["tangentialprojectiontraction"][walls] + st["normalprojectiontraction"][walls], t,
                       rtol=1e-12, atol=1e-15 * np.max(np.abs(t)))


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_mixed_precision_stress(case_dir, precision):
    """Shifted storage: stress caches within the form's error of the FP64 oracle
    (relative to each field's largest magnitude)."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall, precision=precision)
    orc = O.Simulation(xml, kernel, wall)
    gpu.step(STEPS, macro=True, stress=True)
    assert orc.run(STEPS, macro=True) == 0
    tol = 1e-3 if precision == "fp32" else 3e-2
    devs = {}
    for f in FIELDS:
        g, o = gpu.GetStress(f), orc.stress(f)
        devs[f] = float(np.max(np.abs(g - o)) / np.max(np.abs(o)))
    print(precision, devs)
    for f, d in devs.items():
        assert d <= tol, (f, d)
