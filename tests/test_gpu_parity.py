"""FP64 parity of the B200 kernels with the CPU oracle (the reference's algorithm).

Each case runs the same case file on the GPU (through the C ABI) and on the
oracle, then compares the distributions entering the next step, density,
velocity and wall shear stress.  The bar: at most 1e-12 deviation relative to
the field's largest magnitude; the kernels are written to be bit-exact, and the
number of differing values is reported.
"""

import numpy as np
import pytest

from conftest import SMALL_CASES, make_small_case
from hemepure_b200 import lbm
from oracle import oracle as O

TOL = 1e-12
pytestmark = pytest.mark.gpu


def rel_dev(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a - b)))


def run_pair(case_dir, key, steps=None):
    xml, gmy, info, kernel, wall, nsteps = make_small_case(case_dir, key)
    steps = steps or nsteps
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall)
    orc = O.Simulation(xml, kernel, wall)
    gpu.step(steps, macro=True)
    assert orc.run(steps, macro=True) == 0
    return gpu, orc


@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_fp64_parity(case_dir, key):
    gpu, orc = run_pair(case_dir, key)
    assert gpu.time_step == orc.time_step
    f_g, f_o = gpu.GetFOld(), orc.f()
    rho_g, u_g, w_g = gpu.GetPropertyCache()
    rho_o, u_o, w_o = orc.macro()
    wall = w_o < 1e300
    assert np.array_equal(wall, w_g < 1e300)
    devs = {"f": rel_dev(f_g, f_o), "rho": rel_dev(rho_g, rho_o), "u": rel_dev(u_g, u_o),
            "p": rel_dev((rho_g - 1.0) / 3.0, (rho_o - 1.0) / 3.0), "wss": rel_dev(w_g[wall], w_o[wall])}
    exact = int(np.sum(f_g != f_o))
    print(f"{key}: deviations {devs}; {exact} of {f_o.size} distributions differ in any bit")
    for k, v in devs.items():
        assert v <= TOL, (k, v)


def test_phase_api_matches_step(case_dir):
    """RequestComms/PreSend/PreReceive/PostReceive/EndIteration == one hb_step."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_r8")
    a = lbm.LBM(xml, kernel=kernel, wall=wall)
    b = lbm.LBM(xml, kernel=kernel, wall=wall)
    for _ in range(5):
        a.RequestComms()
        a.PreSend()
        a.PreReceive()
        a.PostReceive()
        a.EndIteration()
    b.step(5)
    assert a.time_step == b.time_step == 6
    assert np.array_equal(a.GetFOld(), b.GetFOld())


def test_get_set_fs_round_trip(case_dir):
    """GetFOld mid-run does not perturb the run; SetFs restores a state exactly."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    a = lbm.LBM(xml, kernel=kernel, wall=wall)
    b = lbm.LBM(xml, kernel=kernel, wall=wall)
    a.step(7)
    mid = a.GetFOld()
    a.step(6)
    b.step(13)
    assert np.array_equal(a.GetFOld(), b.GetFOld())
    c = lbm.LBM(xml, kernel=kernel, wall=wall)
    c.SetFs(mid)
    c.time_step = 8
    c.step(6)
    assert np.array_equal(c.GetFOld(), b.GetFOld())


def test_windkessel_state(case_dir):
    gpu, orc = run_pair(case_dir, "bifurcation", steps=300)
    for k in range(2):
        g = gpu.GetWK3(1, k)
        o = orc.wk3(1, k)
        assert rel_dev(g, o) <= TOL, (g, o)


def test_instability_is_reported(case_dir):
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_r8")
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall)
    f = gpu.GetFOld()
    f[17, 3] = -1.0
    gpu.SetFs(f)
    with pytest.raises(lbm.Unstable):
        gpu.step(2)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_moment_sums_match_distributions(case_dir, precision):
    """hb_moment_sums equals the density and momentum summed from GetFOld on the host."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    g = lbm.LBM(xml, kernel=kernel, wall=wall, precision=precision)
    g.step(40)
    sums = g.moment_sums()
    f = g.GetFOld()
    cx = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0], float)
    cy = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1], float)
    cz = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1], float)
    ref = np.array([f.sum(), (f * cx).sum(), (f * cy).sum(), (f * cz).sum()])
    assert abs(sums[0] - ref[0]) <= 1e-12 * abs(ref[0])
    assert np.max(np.abs(sums[1:] - ref[1:])) <= 1e-12 * abs(ref[0])


def test_file_inlet_and_wk2_outlet_bit_exact(tmp_path):
    """A file-pressure inlet (InOutLetFile) and a two-element Windkessel outlet
    (InOutLetWK2): FP64 bit-exact with the oracle, the Windkessel state included;
    the FP32 form within 1e-4."""
    from test_cpu_iolets import _pipe_case
    xml, steps = _pipe_case(tmp_path, trailing_newline=True)
    gpu = lbm.LBM(xml, kernel="LBGK", wall="SBB")
    orc = O.Simulation(xml, "LBGK", "SBB")
    gpu.step(steps, macro=True)
    assert orc.run(steps, macro=True) == 0
    assert np.array_equal(gpu.GetFOld(), orc.f())
    rho_g, u_g, w_g = gpu.GetPropertyCache()
    rho_o, u_o, w_o = orc.macro()
    assert np.array_equal(rho_g, rho_o) and np.array_equal(u_g, u_o)
    assert np.array_equal(gpu.GetWK3(1, 0), orc.wk3(1, 0))
    assert np.max(np.abs(u_o)) > 0
    f32 = lbm.LBM(xml, kernel="LBGK", wall="SBB", precision="fp32")
    f32.step(steps, macro=True)
    assert rel_dev(f32.GetPropertyCache()[1], u_o) <= 1e-4


@pytest.mark.parametrize("inlet,kernel,wall", [("womersley", "LBGK", "SBB"), ("womersley", "TRT", "GZS"),
                                               ("file", "LBGK", "BFL"), ("file", "TRT", "GZS")])
def test_velocity_inlets_bit_exact(tmp_path, inlet, kernel, wall):
    """Womersley (InOutLetWomersleyVelocity) into a fileWK outlet, and file velocity
    (InOutLetFileVelocity) into a pressure outlet, under the Ladd rule, with the GZS
    walls' extrapolation from a velocity iolet: FP64 bit-exact with the oracle (the
    Windkessel state included); the FP32 form within 1e-4."""
    from test_cpu_velocity_iolets import velocity_pipe_case
    xml, steps = velocity_pipe_case(tmp_path, inlet, relaxation_parameter=3.0 / 16.0 if kernel == "TRT" else None)
    gpu = lbm.LBM(xml, kernel=kernel, wall=wall)
    orc = O.Simulation(xml, kernel, wall)
    gpu.step(steps, macro=True)
    assert orc.run(steps, macro=True) == 0
    assert np.array_equal(gpu.GetFOld(), orc.f())
    rho_g, u_g, w_g = gpu.GetPropertyCache()
    rho_o, u_o, w_o = orc.macro()
    assert np.array_equal(rho_g, rho_o) and np.array_equal(u_g, u_o) and np.array_equal(w_g, w_o)
    if inlet == "womersley":
        assert np.array_equal(gpu.GetWK3(1, 0), orc.wk3(1, 0))
    assert np.max(np.abs(u_o)) > 1e-3
    f32 = lbm.LBM(xml, kernel=kernel, wall=wall, precision="fp32")
    f32.step(steps, macro=True)
    assert rel_dev(f32.GetPropertyCache()[1], u_o) <= 1e-4
