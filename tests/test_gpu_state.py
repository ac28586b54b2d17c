"""Exact restart from the FP64 state file (hb_write_state / hb_read_state).

A run stopped after some steps, written out and restored into a fresh handle
continues bit for bit: distributions, macroscopic fields and the Windkessel
state after further steps equal those of the run that never stopped.  The
reference's own checkpoint (float32 distributions in an .xtr file) cannot do
that; hb_read_checkpoint keeps reading it."""

import numpy as np
import pytest

from conftest import make_small_case
from hemepure_b200 import lbm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("key,split", [("pipe_r8", 137), ("bifurcation", 333), ("stenosis", 250)])
def test_state_file_resumes_bit_for_bit(case_dir, tmp_path, key, split):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    path = tmp_path / "state.bin"
    a = lbm.LBM(xml, kernel=kernel, wall=wall)
    a.step(split)
    a.WriteState(path)
    t_written = a.time_step
    a.step(200, macro=True)
    b = lbm.LBM(xml, kernel=kernel, wall=wall)
    b.ReadState(path)
    assert b.time_step == t_written
    b.step(200, macro=True)
    assert np.array_equal(a.GetFOld(), b.GetFOld())
    for x, y in zip(a.GetPropertyCache(), b.GetPropertyCache()):
        assert np.array_equal(x, y)
    if key == "bifurcation":
        for k in range(2):
            assert np.array_equal(a.GetWK3(1, k), b.GetWK3(1, k))


def test_state_file_refuses_another_lattice(case_dir, tmp_path):
    x1 = make_small_case(case_dir, "pipe_r8")
    x2 = make_small_case(case_dir, "pipe_bfl")
    a = lbm.LBM(x1[0], kernel=x1[3], wall=x1[4])
    a.step(5)
    a.WriteState(tmp_path / "s.bin")
    b = lbm.LBM(x2[0], kernel=x2[3], wall=x2[4])
    with pytest.raises(lbm.HemeLBError) as e:
        b.ReadState(tmp_path / "s.bin")
    assert e.value.code == -3
    c = lbm.LBM(x1[0], kernel=x1[3], wall=x1[4], precision="fp32")
    with pytest.raises(lbm.HemeLBError):
        c.WriteState(tmp_path / "t.bin")
