"""The C++ host class (include/hemeb200_lbm.hpp) over the C ABI, built and run the
way a HemePure build would use it: compiled with g++ against the header and
linked to libhemeb200.so."""

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, make_small_case, gpu_available
from hemepure_b200 import lbm
from oracle import oracle as O

SRC = os.path.join(ROOT, "tests", "cpp", "lbm_shim_main.cpp")
LIBDIR = os.path.join(ROOT, "hemepure_b200")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    lbm.library()  # the library must be built
    exe = str(tmp_path_factory.mktemp("cpp") / "lbm_shim_main")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe,
                           "-L" + LIBDIR, "-lhemeb200", "-Wl,-rpath," + LIBDIR])
    return exe


def test_shim_reports_library_errors(shim, tmp_path):
    """A missing case file surfaces as hemeb200::Error with the C ABI's message."""
    r = subprocess.run([shim, str(tmp_path / "missing.xml"), "1", "0", "0", str(tmp_path / "o.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 2 and "hemeb200 error" in r.stderr


def test_shim_without_gpu_fails_cleanly(shim, case_dir, tmp_path):
    if gpu_available():
        pytest.skip("a GPU is present")
    xml = make_small_case(case_dir, "pipe_r8")[0]
    r = subprocess.run([shim, xml, "1", "0", "0", str(tmp_path / "o.bin")], capture_output=True, text=True)
    assert r.returncode == 2 and "error -4" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["pipe_r8", "pipe_bfl"])
def test_shim_phases_match_the_oracle(shim, case_dir, tmp_path, key):
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, key)
    steps = 120
    out = tmp_path / "o.bin"
    r = subprocess.run([shim, xml, str(steps), str(O.KERNELS[kernel]), str(O.WALLS[wall]), str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.uint8)
    n, t = np.frombuffer(raw[:16].tobytes(), dtype=np.int64)
    body = np.frombuffer(raw[16:].tobytes(), dtype=np.float64)
    f, rho, u, wss, tensor, traction = np.split(body, [19 * n, 20 * n, 23 * n, 24 * n, 30 * n])
    orc = O.Simulation(xml, kernel, wall)
    assert orc.run(steps, macro=True) == 0
    assert t == orc.time_step
    assert np.array_equal(f.reshape(n, 19), orc.f())
    rho_o, u_o, w_o = orc.macro()
    assert np.array_equal(rho, rho_o) and np.array_equal(u.reshape(n, 3), u_o) and np.array_equal(wss, w_o)
    assert np.array_equal(tensor.reshape(n, 6), orc.stress("stresstensor"))
    assert np.array_equal(traction.reshape(n, 3), orc.stress("traction"))
