"""File-pressure and two-element Windkessel iolets on the host.

* The oracle's restatement of InOutLetFile::CalculateTable is pinned by the
  reference's own unit test InOutLetTests::TestFileConstruct
  (src/unittests/lbtests/iolets/InOutLetTests.h:117-162) on its fixture
  iolet.txt (tests/golden/, copied by make_golden.py): the density at step 0 and
  at half the run, and the minimum, against the pressures 78 and 82 mmHg.
* The library's table (its own C++ reader) equals the oracle's bit for bit, for
  a file that ends after its last number and for one that ends with a newline
  (the reference's read loop makes one more pass over such a file).
* A WK2 condition is read into lattice units the same way by both.
"""

import os
import shutil

import numpy as np
import pytest

from conftest import ROOT
from hemepure_b200 import lbm, vessels
from oracle import case as ocase

GOLDEN = os.path.join(ROOT, "tests", "golden")
MMHG = 133.3223874
CS2 = 1.0 / 3.0


def test_file_table_known_answers():
    dt, voxel, steps = 1e-4, 0.01, 40000     # config_file_inlet.xml
    u = ocase.Units(dt, voxel, [0.0, 0.0, 0.0])
    table, dmin = ocase.file_density_table(os.path.join(GOLDEN, "iolet.txt"), steps, dt, u)
    temp = dt / voxel

    def target(p):
        return 1 + (p - 0.0) * MMHG * temp * temp / (CS2 * 1000.0)

    assert len(table) == steps + 1
    assert table[0] == pytest.approx(target(78.0), abs=1e-6)
    assert table[steps // 2] == pytest.approx(target(82.0), abs=1e-6)
    assert dmin == pytest.approx(target(78.0), abs=1e-6)


def _pipe_case(tmp_path, trailing_newline: bool):
    v = vessels.Pipe(4, 16)
    vessels.voxelise(v, str(tmp_path / "p.gmy"))
    units = vessels.CaseUnits(tau=0.8)
    steps = 300
    T = steps * units.dt
    rows = [(0.0, units.density_to_mmHg(1.0)), (0.3 * T, units.density_to_mmHg(1.002)),
            (0.7 * T, units.density_to_mmHg(1.001)), (1.2 * T, units.density_to_mmHg(1.0015))]
    text = "\n".join(f"{t!r} {p!r}" for t, p in rows) + ("\n" if trailing_newline else "")
    (tmp_path / "inlet.txt").write_text(text)
    area = np.pi * 4 * 4
    xml = tmp_path / "case.xml"
    vessels.write_case_xml(str(xml), "p.gmy", v, units, steps, [vessels.FilePressureBC("inlet.txt")],
                           [vessels.WK2BC(r=4.0, c=2.5e5, area=area)])
    return str(xml), steps


@pytest.mark.parametrize("trailing_newline", [False, True])
def test_library_file_table_equals_the_oracle(tmp_path, trailing_newline):
    xml, steps = _pipe_case(tmp_path, trailing_newline)
    cfg = ocase.load_case(xml, "LBGK")
    ref = np.asarray(cfg.inlets[0].table)
    got = lbm.read_case_iolet_table(xml, "LBGK", False, 0, len(ref))
    assert np.array_equal(got, ref)
    p, _ = lbm.read_case(xml, "LBGK")
    assert p.inlets[0].kind == lbm.IOLET_KINDS["file"] and p.inlets[0].table_steps == len(ref)
    assert p.inlets[0].density_min == cfg.inlets[0].density_min


def test_wk2_condition_in_lattice_units(tmp_path):
    xml, _ = _pipe_case(tmp_path, False)
    cfg = ocase.load_case(xml, "LBGK")
    p, _ = lbm.read_case(xml, "LBGK")
    o, r = p.outlets[0], cfg.outlets[0]
    assert o.kind == lbm.IOLET_KINDS["wk2"] and r.kind == "wk2"
    assert (o.rp, o.cp, o.area, o.radius) == (r.rp, r.cp, r.area, r.radius)
    assert o.rp == pytest.approx(4.0) and o.cp == pytest.approx(2.5e5)
