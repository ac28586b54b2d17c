"""The storage layout built on the GPU (layout_device.cu) against the host build.

The host build (layout.cpp) is the one the parity tests pin: every case steps
bit-exactly with the oracle and with HemePure through it.  The device passes
must give the same layout bit for bit -- storage order, run axis and offsets,
the plain/general split, every general record, the Windkessel couplings --
which the digests of each array check, on the reference's FourCube geometry
and on the four scaled cases, under each wall rule the case can take.  A case
created through the device reader (which lays the lattice out on the device)
then steps to the same distributions as one created through the host reader.
"""

import os

import numpy as np
import pytest

from conftest import ROOT, SMALL_CASES, make_small_case
from hemepure_b200 import lbm

pytestmark = pytest.mark.gpu

FOUR_CUBE = os.path.join(ROOT, "tests", "golden", "four_cube.gmy")
FIELDS = ["scalars", "st2ref", "ref2st", "meta", "run_off", "g_site", "g_run", "g_src", "g_io", "g_cpl", "g_xyz",
          "g_kind", "g_wall", "g_iolet", "g_q", "g_nrm", "couplings"]


def assert_same_layout(g, params, wall):
    host = g.layout_digest(params, wall, device=-1)
    dev = g.layout_digest(params, wall, device=0)
    diff = [FIELDS[k] for k in range(len(FIELDS)) if host[k] != dev[k]]
    assert not diff, f"device layout differs from the host's in {diff}"
    assert np.array_equal(host, dev)


def four_cube_params():
    g = lbm.Geometry(FOUR_CUBE)
    t = g.tables()
    p = lbm.Params()
    p.tau = 0.8
    p.initial_density = 1.0
    for st, attr in ((1, "n_inlets"), (2, "n_outlets")):
        ids = t["iolet_id"][t["site_type"] == st]
        setattr(p, attr, int(ids.max()) + 1 if ids.size else 0)
    for k in range(p.n_inlets):
        p.inlets[k].normal[:] = [0.0, 0.0, 1.0]
    for k in range(p.n_outlets):
        p.outlets[k].normal[:] = [0.0, 0.0, -1.0]
    return g, p


@pytest.mark.parametrize("wall", ["SBB", "BFL", "GZS"])
def test_four_cube_layout(wall):
    g, p = four_cube_params()
    try:
        host = g.layout_digest(p, wall, device=-1)
    except lbm.HemeLBError as e:  # a lattice the host refuses, the device must refuse alike
        with pytest.raises(lbm.HemeLBError) as d:
            g.layout_digest(p, wall, device=0)
        assert d.value.code == e.code
        return
    assert np.array_equal(host, g.layout_digest(p, wall, device=0))


@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_cases_layout(case_dir, key):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    p, _ = lbm.read_case(xml, kernel)
    for reader in (None, 0):
        g = lbm.Geometry(gmy, device=reader)
        for w in sorted({wall, "SBB", "BFL"}):
            assert_same_layout(g, p, w)


@pytest.mark.parametrize("key", ["bifurcation", "stenosis"])
def test_created_with_device_layout_steps_alike(case_dir, key):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    a = lbm.LBM(xml, kernel=kernel, wall=wall, geometry_reader="host")
    b = lbm.LBM(xml, kernel=kernel, wall=wall, geometry_reader="device")
    a.step(40, macro=True)
    b.step(40, macro=True)
    assert np.array_equal(a.GetFOld(), b.GetFOld())
    for x, y in zip(a.GetPropertyCache(), b.GetPropertyCache()):
        assert np.array_equal(x, y, equal_nan=True)


def test_setup_timing_phases(case_dir):
    """hb_setup_timing reports the case, geometry and solver phases of a creation
    from a case file, and they add up to its total."""
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_bfl")
    for reader in ("device", "host"):
        sim = lbm.LBM(xml, kernel=kernel, wall=wall, geometry_reader=reader)
        t = sim.setup_timing()
        assert t["geometry"] > 0.0 and t["solver"] > 0.0 and t["case"] >= 0.0
        assert abs(t["case"] + t["geometry"] + t["solver"] - t["total"]) < 1e-6 * max(1.0, t["total"]) + 1e-9
        sim.close()
