"""Edge cases on the GPU path.

* The reference's own unit-test geometry (four_cube.gmy, 64 sites): every site
  is a wall or iolet site, so the plain-bulk kernel has nothing to do and the
  whole lattice runs through the boundary rules.  FP64 must stay bit-exact with
  the oracle; the batched form must run it too.
* A batch member that goes unstable is handed back at the end of the block
  with its status set and stops stepping; the others are unaffected.
* A case whose geometry file is missing is refused by both forms.
"""

import os
import shutil
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import ROOT
from hemepure_b200 import lbm, vessels
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FOUR_CUBE = os.path.join(ROOT, "tests", "golden", "four_cube.gmy")


def four_cube_case(tmp, tau=0.8, kernel="LBGK", steps=300, rho_in=1.001, name=None):
    d = os.path.join(str(tmp), name or f"four_cube_{kernel}")
    os.makedirs(d, exist_ok=True)
    shutil.copy(FOUR_CUBE, os.path.join(d, "four_cube.gmy"))
    # Inlet below z = 1 and outlet above z = 4 (iolet id 0 each), normals into the fluid.
    v = SimpleNamespace(iolets=[
        vessels.Iolet("inlet", np.array([2.5, 2.5, 0.5]), np.array([0.0, 0.0, 1.0]), 2.0),
        vessels.Iolet("outlet", np.array([2.5, 2.5, 4.5]), np.array([0.0, 0.0, -1.0]), 2.0)])
    xml = os.path.join(d, "case.xml")
    vessels.write_case_xml(xml, "four_cube.gmy", v, vessels.CaseUnits(tau=tau), steps,
                           [vessels.PressureBC(rho_in)], [vessels.PressureBC(0.999)],
                           relaxation_parameter=3.0 / 16.0 if kernel == "TRT" else None)
    return xml


@pytest.mark.parametrize("kernel,wall", [("LBGK", "SBB"), ("TRT", "BFL")])
def test_four_cube_fp64_bit_exact(tmp_path, kernel, wall):
    xml = four_cube_case(tmp_path, kernel=kernel)
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall)
    orc = O.Simulation(xml, kernel, wall)
    gpu.step(300, macro=True)
    assert orc.run(300, macro=True) == 0
    assert np.array_equal(gpu.GetFOld(), orc.f())
    rho_g, u_g, w_g = gpu.GetPropertyCache()
    rho_o, u_o, w_o = orc.macro()
    assert np.array_equal(rho_g, rho_o) and np.array_equal(u_g, u_o) and np.array_equal(w_g, w_o)
    assert np.max(np.abs(u_o)) > 0  # the pressure drop drives a flow


def test_four_cube_in_a_batch(tmp_path):
    xml = four_cube_case(tmp_path, kernel="LBGK")
    b = lbm.Batch(4096, 4096, 4)
    slot = b.add_xml(xml, "LBGK", "SBB", 300)
    done = []
    while not done:
        done = b.run(64)
    rho_b, u_b, w_b = b.macro(slot)
    orc = O.Simulation(xml, "LBGK", "SBB")
    assert orc.run(300, macro=True) == 0
    rho_o, u_o, w_o = orc.macro()
    assert np.max(np.abs(u_b - u_o)) <= 1e-4 * np.max(np.abs(u_o))
    walls = w_o < 1e300
    assert np.max(np.abs(w_b[walls] - w_o[walls])) <= 1e-4 * np.max(np.abs(w_o[walls]))


def test_missing_geometry_is_refused(tmp_path):
    xml = four_cube_case(tmp_path)
    os.remove(os.path.join(os.path.dirname(xml), "four_cube.gmy"))
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.LBM(xml)
    assert e.value.code == -2
    b = lbm.Batch(4096, 4096, 2)
    with pytest.raises(lbm.HemeLBError) as e:
        b.add_xml(xml, "LBGK", "SBB", 10)
    assert e.value.code == -2


def test_unstable_member_is_retired_early(tmp_path):
    """An inlet density of 1.5 at tau 0.51 drives FourCube unstable within 15 steps
    (the oracle agrees); the batch returns it after the first block with status
    bit 1, while a stable member beside it finishes with the result it has alone."""
    stable = four_cube_case(tmp_path, kernel="LBGK")
    wild = four_cube_case(tmp_path, tau=0.51, steps=100000, rho_in=1.5, name="four_cube_unstable")
    alone = lbm.Batch(4096, 4096, 4)
    s0 = alone.add_xml(stable, "LBGK", "SBB", 300)
    while not alone.run(64):
        pass
    ref = alone.macro(s0)
    b = lbm.Batch(8192, 8192, 4)
    s1 = b.add_xml(stable, "LBGK", "SBB", 300)
    s2 = b.add_xml(wild, "LBGK", "SBB", 100000)
    first = b.run(64)
    assert first == [s2]
    n, t, st = b.info(s2)
    assert st & 1 and t <= 1 + 64
    b.remove(s2)
    done = []
    while not done:
        done = b.run(64)
    assert done == [s1] and b.info(s1)[2] == 0
    for a, m in zip(ref, b.macro(s1)):
        assert np.array_equal(a, m)
