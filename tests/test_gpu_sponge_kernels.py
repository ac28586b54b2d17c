"""The LBGK and TRT sponge-layer kernels (the reference's HEMELB_KERNEL choices
LBGKSL and TRTSL, src/lb/kernels/LBGKSpongeLayer.h, TRTSpongeLayer.h) in FP64:
bit-exact with the oracle through the sponge's whole schedule (its own time for
the first half of the lifetime, the linear return to tau0, then tau0), with
bounce-back and BFL walls, a velocity inlet and a Nash pressure outlet."""

import os

import numpy as np
import pytest

from hemepure_b200 import lbm, vessels
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEPS = 300


def sponge_case(d, kernel):
    v = vessels.Pipe(6, 40)
    gmy = os.path.join(d, "p.gmy")
    if not os.path.exists(gmy):
        vessels.voxelise(v, gmy)
    xml = os.path.join(d, kernel + ".xml")
    vessels.write_case_xml(xml, "p.gmy", v, vessels.CaseUnits(tau=0.6), STEPS, [vessels.VelocityBC(0.02)],
                           [vessels.PressureBC(1.0)], warmup=50,
                           relaxation_parameter=3.0 / 16.0 if kernel == "TRTSL" else None,
                           sponge={"viscosity_ratio": 10.0, "width": 12.0, "lifetime": 200})
    return xml


@pytest.mark.parametrize("kernel,wall", [("LBGKSL", "SBB"), ("LBGKSL", "BFL"), ("TRTSL", "SBB"), ("TRTSL", "BFL")])
def test_sponge_kernels_bit_exact(tmp_path, kernel, wall):
    xml = sponge_case(str(tmp_path), kernel)
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall)
    orc = O.Simulation(xml, kernel, wall)
    gpu.step(STEPS, macro=True)
    assert orc.run(STEPS, macro=True) == 0
    f_g, f_o = gpu.GetFOld(), orc.f()
    assert int(np.sum(f_g != f_o)) == 0
    for a, b in zip(gpu.GetPropertyCache(), orc.macro()):
        assert np.array_equal(a, b)


def test_sponge_kernels_refuse_gzs_and_low_precision(tmp_path):
    xml = sponge_case(str(tmp_path), "LBGKSL")
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.LBM(xml, kernel="LBGKSL", wall="GZS")
    assert e.value.code == -7
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.LBM(xml, kernel="LBGKSL", wall="SBB", precision="fp32")
    assert e.value.code == -7
