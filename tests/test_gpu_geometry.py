"""The `.gmy` reader with its decode on the GPU (hb_geometry_open_device).

* Same tables as the host reader, bit for bit (neighbour table, masks, types,
  iolet ids, coordinates, type counts, cut distances, normals), on the
  reference's own FourCube geometry and on the synthetic pipe, bifurcation and
  stenosis cases; the host reader is pinned by the oracle and by the reference's
  GeometryReaderTests (tests/test_cpu_geometry.py).
* A block whose header declares more or fewer fluid sites than its records hold
  is refused with HB_ERR_FORMAT by both readers.
* A case created with either reader steps to the same distributions.
"""

import os
import shutil
import struct

import numpy as np
import pytest

from conftest import ROOT, SMALL_CASES, make_small_case
from hemepure_b200 import lbm

pytestmark = pytest.mark.gpu

FOUR_CUBE = os.path.join(ROOT, "tests", "golden", "four_cube.gmy")


def assert_same_tables(path):
    host = lbm.Geometry(path).tables()
    dev_g = lbm.Geometry(path, device=0)
    dev = dev_g.tables()
    for k in host:
        assert host[k].dtype == dev[k].dtype and np.array_equal(host[k], dev[k]), k
    return dev_g


def test_four_cube_same_tables():
    assert_same_tables(FOUR_CUBE)


@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_cases_same_tables(case_dir, key):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    g = assert_same_tables(gmy)
    assert g.n == info.fluid_sites
    assert g.read_timing()["device"] > 0.0


def _edit_first_block_count(src, dst, delta):
    data = bytearray(open(src, "rb").read())
    bx, by, bz, bs = struct.unpack(">IIII", data[12:28])
    nb = bx * by * bz
    for b in range(nb):
        fluid = struct.unpack(">I", data[32 + 12 * b: 36 + 12 * b])[0]
        if fluid:
            data[32 + 12 * b: 36 + 12 * b] = struct.pack(">I", fluid + delta)
            break
    open(dst, "wb").write(bytes(data))


@pytest.mark.parametrize("delta", [1, -1])
def test_block_count_mismatch_is_refused(tmp_path, delta):
    bad = str(tmp_path / "bad.gmy")
    _edit_first_block_count(FOUR_CUBE, bad, delta)
    for dev in (None, 0):
        with pytest.raises(lbm.HemeLBError) as e:
            lbm.Geometry(bad, device=dev)
        assert e.value.code == -3


def test_create_with_either_reader(case_dir):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_bfl")
    a = lbm.LBM(xml, kernel=kernel, wall=wall, geometry_reader="host")
    b = lbm.LBM(xml, kernel=kernel, wall=wall, geometry_reader="device")
    a.step(50)
    b.step(50)
    assert np.array_equal(a.GetFOld(), b.GetFOld())
