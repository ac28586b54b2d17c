"""Velocity iolets on the host: Womersley, file velocity, and the fileWK pressure iolet.

* The oracle's Bessel series is pinned by the reference's BesselTests::TestUsedRange
  table of J0(i^(3/2) x), x = 0 .. 20 (tests/golden/bessel_j0_table.json, parsed by
  make_golden.py), at the test's absolute 1e-6.
* The Womersley profile repeats InOutLetTests::TestWomersleyVelocityConstruct
  (src/unittests/lbtests/iolets/InOutLetTests.h:200-262) on its fixture
  config_new_velocity_inlets.xml: the values read from the case, zero velocity at
  the wall, and the Poiseuille limit at a small Womersley number a quarter and
  three quarters into the period.
* The file velocity profile repeats TestFileVelocityConstruct (:264-332) on
  config_file_velocity_inlet.xml and velocity_inlet.txt: 0.01 m/s on the axis
  and 0.0075 m/s half way to the wall at t = 3 s.
* The library's host evaluation (hb_iolet_velocity, the values the kernels impose)
  equals the oracle's bit for bit at random points and steps, and its file
  velocity table equals the oracle's.

The fixtures give iolet positions in metres, as the reference's tests were
written for an older reader; the reference's SimConfig takes them in lattice
units (src/configuration/SimConfig.cc:648-650), so the tests rewrite the
position element before reading.
"""

import json
import math
import os
import re
import shutil

import numpy as np
import pytest

from conftest import ROOT
from hemepure_b200 import lbm
from oracle import case as ocase
from oracle import oracle as O

GOLDEN = os.path.join(ROOT, "tests", "golden")
MMHG = 133.3223874


def _lattice_position_copy(src: str, dst_dir, voxel: float, extra=()) -> str:
    text = open(src).read()

    def conv(m):
        v = [float(a) / voxel for a in m.group(1).split(",")]
        return '<position value="(' + ",".join(repr(a) for a in v) + ')" units="lattice" />'

    text = re.sub(r'<position value="\(([^)]*)\)" units="m" />', conv, text)
    dst = os.path.join(str(dst_dir), os.path.basename(src))
    with open(dst, "w") as fh:
        fh.write(text)
    for name in extra:
        shutil.copy(os.path.join(GOLDEN, name), os.path.join(str(dst_dir), name))
    return dst


def test_bessel_j0_against_the_reference_table():
    d = json.load(open(os.path.join(GOLDEN, "bessel_j0_table.json")))
    th = 1.5 * math.atan2(1.0, 0.0)          # i^(3/2) = exp(1.5 i pi/2)
    i32 = complex(math.cos(th), math.sin(th))
    assert len(d["x"]) == 201
    for x, (re_, im_) in zip(d["x"], d["j0"]):
        j = O.bessel_j0(i32 * x)
        assert abs(j.real - re_) <= d["abs_tol"] and abs(j.imag - im_) <= d["abs_tol"], x


def _womersley(tmp_path):
    xml = _lattice_position_copy(os.path.join(GOLDEN, "config_new_velocity_inlets.xml"), tmp_path, 0.01)
    p, _ = lbm.read_case(xml)
    cfg = ocase.load_case(xml)
    return p.inlets[0], cfg.inlets[0]


def test_womersley_construct(tmp_path):
    io, oc = _womersley(tmp_path)
    assert io.kind == lbm.IOLET_KINDS["womersley"] and oc.kind == "womersley"
    assert io.radius == 10.0 and oc.radius == 10.0
    assert io.pressure_gradient_amplitude == pytest.approx(MMHG * 1e-6, rel=1e-15)
    assert io.pressure_gradient_amplitude == oc.pressure_gradient_amplitude
    assert io.period == pytest.approx(5.0, rel=1e-15) and io.period == oc.period
    assert io.womersley_number == 2.0 and oc.womersley_number == 2.0
    assert list(io.position) == pytest.approx([0.0, 0.0, -5.0]) and list(io.normal) == [0.0, 0.0, 1.0]
    # Zero at the wall (r = R) at t = 0.
    wall = np.array([10.0, 0.0, -5.0])
    for v in (lbm.iolet_velocity(io, wall, 0), O.iolet_velocity(oc, wall, 0)):
        assert np.all(np.abs(v) <= 1e-9)


def test_womersley_poiseuille_limit(tmp_path):
    io, oc = _womersley(tmp_path)
    alpha, eta, nu = 1e-4, 1.0, 1.0
    for c in (io, oc):
        c.womersley_number = alpha
        c.period = 2 * math.pi * io.radius ** 2 / (alpha * alpha * nu)
    poiseuille = io.pressure_gradient_amplitude * io.radius ** 2 / (4 * eta)
    centre = np.array(io.position[:])
    for frac, sign in ((0.25, 1.0), (0.75, -1.0)):
        t = int(frac * io.period)  # GetVelocity takes a LatticeTimeStep
        vl = lbm.iolet_velocity(io, centre, t)
        vo = O.iolet_velocity(oc, centre, t)
        assert np.array_equal(vl, vo)
        assert abs(vl[0]) <= 1e-9 and abs(vl[1]) <= 1e-9
        assert vl[2] == pytest.approx(sign * poiseuille, abs=1e-9)


def _file_velocity(tmp_path):
    xml = _lattice_position_copy(os.path.join(GOLDEN, "config_file_velocity_inlet.xml"), tmp_path, 0.01,
                                 extra=("velocity_inlet.txt",))
    p, _ = lbm.read_case(xml)
    cfg = ocase.load_case(xml)
    io = p.inlets[0]
    table = lbm.read_case_iolet_table(xml, "LBGK", False, 0, io.table_steps)
    io.table = table.ctypes.data
    return io, cfg, table


def test_file_velocity_construct(tmp_path):
    io, cfg, table = _file_velocity(tmp_path)
    oc = cfg.inlets[0]
    assert io.kind == lbm.IOLET_KINDS["file_velocity"] and oc.kind == "file_velocity"
    assert io.radius == pytest.approx(20.0) and io.radius == oc.radius
    assert io.table_steps == 4001 and np.array_equal(table, np.array(oc.table))
    dt, voxel = 0.001, 0.01
    t = int(3.0 / dt)
    centre = np.array(io.position[:])
    half = centre.copy()
    half[0] -= io.radius / 2.0
    for x, want in ((centre, 0.01), (half, 0.0075)):
        vl = lbm.iolet_velocity(io, x, t)
        assert np.array_equal(vl, O.iolet_velocity(oc, x, t))
        phys = vl * (voxel / dt)
        assert abs(phys[0]) <= 1e-9 and abs(phys[1]) <= 1e-9
        assert phys[2] == pytest.approx(want, abs=1e-9)
    outside = centre.copy()
    outside[1] += 1.01 * io.radius
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.iolet_velocity(io, outside, t)
    assert e.value.code == -8
    with pytest.raises(ValueError):
        O.iolet_velocity(oc, outside, t)


def test_random_points_bit_exact(tmp_path):
    rng = np.random.default_rng(7)
    os.makedirs(tmp_path / "w")
    os.makedirs(tmp_path / "f")
    wio, woc = _womersley(tmp_path / "w")
    fio, fcfg, ftable = _file_velocity(tmp_path / "f")   # fio.table points into ftable
    foc = fcfg.inlets[0]
    # A tilted Womersley iolet with a larger Womersley number (r / R beyond 1 included).
    for c in (wio, woc):
        c.womersley_number = 7.3
        c.period = 850.0
    n = np.array([0.3, -0.2, 0.93])
    n /= np.linalg.norm(n)
    wio.normal[:] = list(n)
    woc.normal = list(n)
    for _k in range(300):
        x = np.array(wio.position[:]) + rng.uniform(-12, 12, 3)
        t = int(rng.integers(0, 5000))
        assert np.array_equal(lbm.iolet_velocity(wio, x, t), O.iolet_velocity(woc, x, t))
        xf = np.array(fio.position[:]) + np.append(rng.uniform(-13, 13, 2), rng.uniform(-2, 2))
        assert np.array_equal(lbm.iolet_velocity(fio, xf, t), O.iolet_velocity(foc, xf, t))
    assert ftable.size == fio.table_steps


def test_file_wk_reads_as_wk2(tmp_path):
    from hemepure_b200 import vessels
    v = vessels.Pipe(4, 16)
    units = vessels.CaseUnits(tau=0.8)
    xml = str(tmp_path / "case.xml")
    vessels.write_case_xml(xml, "p.gmy", v, units, 100, [vessels.PressureBC(1.001)],
                           [vessels.FileWKBC("weights.txt", r=4.0, c=2.5e5, area=50.0)])
    p, _ = lbm.read_case(xml)
    oc = ocase.load_case(xml).outlets[0]
    io = p.outlets[0]
    assert io.kind == lbm.IOLET_KINDS["wk2"] and oc.kind == "wk2"
    assert (io.rp, io.cp, io.area) == (oc.rp, oc.cp, oc.area)
    assert io.rp == pytest.approx(4.0, rel=1e-12) and io.cp == pytest.approx(2.5e5, rel=1e-12)
    assert io.area == pytest.approx(50.0, rel=1e-12) and io.radius == 0.0


def velocity_pipe_case(tmp_path, inlet: str, steps: int = 300, relaxation_parameter=None):
    """A pipe (radius 5, length 20) driven by a Womersley inlet into a fileWK outlet,
    or by a file-velocity inlet into a fixed-pressure outlet."""
    from hemepure_b200 import vessels
    d = os.path.join(str(tmp_path), inlet)
    os.makedirs(d, exist_ok=True)
    v = vessels.Pipe(5, 20)
    vessels.voxelise(v, os.path.join(d, "p.gmy"))
    units = vessels.CaseUnits(tau=0.8)
    xml = os.path.join(d, "case.xml")
    if inlet == "womersley":
        vessels.write_case_xml(xml, "p.gmy", v, units, steps,
                               [vessels.WomersleyBC(pressure_gradient=3e-4, period_steps=200, womersley_number=3.0)],
                               [vessels.FileWKBC("weights.txt", r=4.0, c=2.5e5, area=math.pi * 25)],
                               relaxation_parameter=relaxation_parameter)
    else:
        T = steps * units.dt
        rows = [(0.0, 0.0), (0.3 * T, 0.01), (0.7 * T, 0.006), (1.2 * T, 0.012)]
        with open(os.path.join(d, "velocity.txt"), "w") as fh:
            fh.write("\n".join(f"{t!r} {units.speed_to_phys(u)!r}" for t, u in rows) + "\n")
        vessels.write_case_xml(xml, "p.gmy", v, units, steps, [vessels.FileVelocityBC("velocity.txt")],
                               [vessels.PressureBC(1.0)], relaxation_parameter=relaxation_parameter)
    return xml, steps


@pytest.mark.parametrize("inlet,wall", [("womersley", "SBB"), ("womersley", "GZS"), ("file", "BFL"), ("file", "GZS")])
def test_oracle_runs_velocity_inlets(tmp_path, inlet, wall):
    """The oracle steps both inlets stably and drives a flow along the inlet normal."""
    kernel = "TRT" if wall == "GZS" else "LBGK"
    xml, _ = velocity_pipe_case(tmp_path, inlet, relaxation_parameter=3.0 / 16.0 if kernel == "TRT" else None)
    orc = O.Simulation(xml, kernel, wall)
    assert orc.run(60, macro=True) == 0
    _, u, _ = orc.macro()
    assert np.all(np.isfinite(u)) and np.max(np.abs(u)) > 1e-5
