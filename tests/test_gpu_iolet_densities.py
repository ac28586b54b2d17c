"""Iolet densities supplied by the caller (hb_set_iolet_densities): a HemePure
host that keeps its own BoundaryValues hands the library each step's
GetBoundaryDensity instead of the library computing it from the case.

Two cases on one pipe differ only in their Nash pressure iolets.  Running case A
with case B's densities supplied must give case B's oracle result bit for bit,
and clearing the override must give case A's again."""

import os

import numpy as np
import pytest

from hemepure_b200 import lbm, vessels
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEPS = 300


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("iolet_override"))
    v = vessels.Pipe(6, 40)
    vessels.voxelise(v, os.path.join(d, "p.gmy"))
    out = {}
    for name, (rin, rout) in {"a": (1.001, 0.999), "b": (1.003, 0.997)}.items():
        xml = os.path.join(d, name + ".xml")
        vessels.write_case_xml(xml, "p.gmy", v, vessels.CaseUnits(tau=0.8), STEPS, [vessels.PressureBC(rin)],
                               [vessels.PressureBC(rout)])
        out[name] = xml
    return out


def densities(xml):
    p = lbm.LBM(xml, kernel="LBGK", wall="SBB").GetLbmParams()
    return ([p.inlets[k].density_mean for k in range(p.n_inlets)],
            [p.outlets[k].density_mean for k in range(p.n_outlets)])


def test_supplied_densities_replace_the_case(cases):
    din, dout = densities(cases["b"])
    assert din[0] != densities(cases["a"])[0][0]
    sim = lbm.LBM(cases["a"], kernel="LBGK", wall="SBB")
    sim.SetIoletDensities(din, dout)
    sim.step(STEPS, macro=True)
    orc = O.Simulation(cases["b"], "LBGK", "SBB")
    assert orc.run(STEPS, macro=True) == 0
    assert np.array_equal(sim.GetFOld(), orc.f())
    rho, u, _ = sim.GetPropertyCache()
    rho_o, u_o, _ = orc.macro()
    assert np.array_equal(rho, rho_o) and np.array_equal(u, u_o)


def test_clearing_returns_to_the_case(cases):
    din, dout = densities(cases["b"])
    sim = lbm.LBM(cases["a"], kernel="LBGK", wall="SBB")
    sim.SetIoletDensities(din, dout)
    sim.SetIoletDensities()
    sim.step(STEPS)
    ref = lbm.LBM(cases["a"], kernel="LBGK", wall="SBB")
    ref.step(STEPS)
    assert np.array_equal(sim.GetFOld(), ref.GetFOld())


def test_counts_must_match_the_case(cases):
    sim = lbm.LBM(cases["a"], kernel="LBGK", wall="SBB")
    with pytest.raises(lbm.HemeLBError):
        sim.SetIoletDensities([1.0, 1.0], [1.0])
