"""The batched form: many lattices in one arena, stepped by persistent kernels
in CUDA-graph blocks.  Each lattice's result must be the same alone and in a
mix (members admitted at different times, of different sizes and physics),
and within 1e-4 of the FP64 oracle in velocity and wall shear stress."""

import os

import numpy as np
import pytest

from hemepure_b200 import lbm, vessels
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mix(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("mix"))
    cases = []
    # (name, vessel, units tau, inlet bc, outlet bc, kernel, wall, steps, warmup)
    specs = [
        ("a", vessels.Pipe(6, 40), 0.8, [vessels.PressureBC(1.001)], [vessels.PressureBC(0.999)], "LBGK", "SBB", 600, 0),
        ("b", vessels.Pipe(9, 60), 0.6, [vessels.VelocityBC(0.02)], [vessels.PressureBC(1.0)], "LBGK", "BFL", 400, 200),
        ("c", vessels.Stenosis(8, 80, 5, 20), 0.55, [vessels.PressureBC(1.0, 1e-3, 400.0)], [vessels.PressureBC(1.0)],
         "TRT", "BFL", 500, 0),
    ]
    for name, v, tau, inl, outl, kernel, wall, steps, warm in specs:
        gmy = os.path.join(d, name + ".gmy")
        xml = os.path.join(d, name + ".xml")
        vessels.voxelise(v, gmy)
        vessels.write_case_xml(xml, name + ".gmy", v, vessels.CaseUnits(tau=tau), steps, inl, outl, warmup=warm,
                               relaxation_parameter=3.0 / 16.0 if kernel == "TRT" else None)
        cases.append((name, xml, kernel, wall, steps + warm))
    return cases


def run_alone(xml, kernel, wall, steps, tuning=None):
    b = lbm.Batch(400_000, 200_000, 8)
    if tuning:
        b.set_tuning(*tuning)
    slot = b.add_xml(xml, kernel, wall, steps)
    done = []
    while not done:
        done = b.run(64)
    n, t, st = b.info(slot)
    assert st == 0 and t == 1 + steps
    return b.macro(slot)


def test_same_alone_and_in_the_mix(mix):
    alone = {name: run_alone(xml, k, w, s) for name, xml, k, w, s in mix}
    b = lbm.Batch(800_000, 400_000, 8)
    slots = {}
    results = {}
    # staggered admission: a joins at block 0, b after 2 blocks, c after 3
    order = {0: [mix[0]], 2: [mix[1]], 3: [mix[2]]}
    block = 0
    while len(results) < len(mix):
        for name, xml, k, w, s in order.get(block, []):
            slots[b.add_xml(xml, k, w, s)] = name
        for slot in b.run(50):
            results[slots[slot]] = b.macro(slot)
            b.remove(slot)
        block += 1
        assert block < 200
    for name in alone:
        ra, rm = alone[name], results[name]
        for a, m in zip(ra, rm):
            assert np.array_equal(a, m), name


def test_batch_matches_fp64_oracle(mix):
    for name, xml, kernel, wall, steps in mix:
        rho_b, u_b, w_b = run_alone(xml, kernel, wall, steps)
        orc = O.Simulation(xml, kernel, wall)
        assert orc.run(steps, macro=True) == 0
        rho_o, u_o, w_o = orc.macro()
        wall_sites = w_o < 1e300
        eu = np.max(np.abs(u_b - u_o)) / np.max(np.abs(u_o))
        ew = np.max(np.abs(w_b[wall_sites] - w_o[wall_sites])) / np.max(np.abs(w_o[wall_sites]))
        print(f"batch {name} ({kernel}/{wall}, {steps} steps) FP32 error vs FP64: velocity {eu:.2e}, wss {ew:.2e}")
        assert eu <= 1e-4 and ew <= 1e-4


def test_batch_matches_single_lattice_fp32(mix):
    name, xml, kernel, wall, steps = mix[1]
    rho_b, u_b, w_b = run_alone(xml, kernel, wall, steps)
    single = lbm.LBM(xml, kernel=kernel, wall=wall, precision="fp32")
    single.step(steps, macro=True)
    rho_s, u_s, w_s = single.GetPropertyCache()
    assert np.max(np.abs(u_b - u_s)) <= 1e-6 * np.max(np.abs(u_s))


def test_admission_beyond_capacity_is_refused(mix):
    b = lbm.Batch(10_000, 10_000, 2)
    name, xml, kernel, wall, steps = mix[1]
    with pytest.raises(lbm.HemeLBError) as e:
        b.add_xml(xml, kernel, wall, steps)
    assert e.value.code == -5


def test_prepared_admission_matches_and_survives_refusal(mix):
    """A lattice prepared on the host gives the same result as add_xml, and a
    prepared lattice refused for lack of room can be admitted later."""
    name, xml, kernel, wall, steps = mix[0]
    ref = run_alone(xml, kernel, wall, steps)
    prep = lbm.PreparedLattice(xml, kernel, wall, steps)
    small = lbm.Batch(prep.sites // 2, prep.sites // 2, 2)
    with pytest.raises(lbm.HemeLBError) as e:
        small.add_prepared(prep)
    assert e.value.code == -5
    b = lbm.Batch(400_000, 200_000, 8)
    slot = b.add_prepared(prep)
    prep.close()
    done = []
    while not done:
        done = b.run(64)
    for a, m in zip(ref, b.macro(slot)):
        assert np.array_equal(a, m)


def test_prepared_on_the_device_matches(mix):
    """A lattice decoded and laid out on the device steps as one prepared on the host."""
    name, xml, kernel, wall, steps = mix[0]
    out = []
    for device in (None, 0):
        prep = lbm.PreparedLattice(xml, kernel, wall, steps, device=device)
        b = lbm.Batch(400_000, 200_000, 8)
        slot = b.add_prepared(prep)
        prep.close()
        done = []
        while not done:
            done = b.run(64)
        out.append(b.macro(slot))
    for a, m in zip(*out):
        assert np.array_equal(a, m)


@pytest.mark.parametrize("tuning", [(1, 256, "split"), (2, 128, "split"), (2, 256, "persistent"),
                                    (1, 128, "persistent")])
def test_every_launch_shape_gives_the_same_result(mix, tuning):
    """The autotuner's choices (step form, sites per thread, block) change the
    launch and, between kernel instantiations, where the compiler fuses FP32
    multiply-adds: results agree to FP32 rounding (1e-5 of each field's largest
    value), far inside the form's 1e-4 tolerance against FP64."""
    for name, xml, kernel, wall, steps in mix:
        ref = run_alone(xml, kernel, wall, steps)
        got = run_alone(xml, kernel, wall, steps, tuning)
        for a, m in zip(ref, got):
            fin = a < 1e300
            assert np.array_equal(fin, m < 1e300)
            assert np.max(np.abs(a[fin] - m[fin])) <= 1e-5 * np.max(np.abs(a[fin])), (name, tuning)
