"""Host front-end (C++ in libhemeb200.so) against the CPU oracle, no GPU needed.

Bit-exact integer tables (site order, neighbour indices, site data, counts)
and identical lattice-unit parameters from the case reader."""

import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT, SMALL_CASES, make_small_case
from hemepure_b200 import lbm
from oracle import case as ocase
from oracle import oracle as O


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "hemeb200.h")).read()
    declared = set(re.findall(r"\b(hb_[a-z0-9_]+)\s*\(", header))
    L = lbm.library()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    assert declared == set(lbm.EXPORTS)


@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_tables_bit_exact_vs_oracle(case_dir, key):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    g = lbm.Geometry(gmy)
    t = g.tables()
    lat = O.Lattice(gmy)
    assert g.n == lat.n == info.fluid_sites
    assert np.array_equal(t["type_counts"], lat.type_counts())
    assert np.array_equal(t["coords"], lat.coords())
    assert np.array_equal(t["neighbours"], lat.neighbours())
    w, io, ty, ii = lat.sitedata()
    assert np.array_equal(t["wall_mask"], w)
    assert np.array_equal(t["iolet_mask"], io)
    assert np.array_equal(t["site_type"], ty)
    assert np.array_equal(t["iolet_id"], ii)
    assert np.array_equal(t["wall_distance"], lat.wall_distance())
    assert np.array_equal(t["wall_normal"], lat.wall_normal())


@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_case_reader_matches_oracle(case_dir, key):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    p, gpath = lbm.read_case(xml, kernel)
    c = ocase.load_case(xml, kernel)
    assert os.path.abspath(gpath) == os.path.abspath(c.gmy_path)
    assert p.tau == c.tau
    assert p.initial_density == c.initial_density
    assert p.relaxation_parameter == c.relaxation_parameter
    assert p.viscosity_ratio == c.viscosity_ratio and p.sponge_width == c.sponge_width
    assert p.sponge_lifetime == c.sponge_lifetime
    assert p.n_inlets == len(c.inlets) and p.n_outlets == len(c.outlets)
    for group, ref in ((p.inlets, c.inlets), (p.outlets, c.outlets)):
        for k, r in enumerate(ref):
            g = group[k]
            assert g.kind == O.IOLET_KINDS[r.kind]
            assert list(g.position) == r.position and list(g.normal) == r.normal
            for f in ("density_mean", "density_amp", "phase", "period", "radius", "max_speed", "rc", "rp", "cp", "area"):
                assert getattr(g, f) == getattr(r, f), f
            assert g.warmup == r.warmup


@pytest.mark.parametrize("key", list(SMALL_CASES))
def test_layout_streams_exactly(case_dir, key):
    """Every slot has exactly one writer; most sites take the plain bulk path."""
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    p, _ = lbm.read_case(xml, kernel)
    st = lbm.Geometry(gmy).layout(p, wall)
    assert st["bulk_sites"] + st["general_sites"] == info.fluid_sites
    assert st["bulk_sites"] > 0


def test_create_without_gpu_fails_cleanly(case_dir):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_r8")
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.LBM(xml, kernel=kernel, wall=wall)
    assert e.value.code == -4  # HB_ERR_CUDA


def test_malformed_inputs_are_rejected(tmp_path):
    bad = tmp_path / "bad.gmy"
    bad.write_bytes(b"\x00" * 40)
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.Geometry(str(bad))
    assert e.value.code == -3
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.Geometry(str(tmp_path / "missing.gmy"))
    assert e.value.code == -2
    xml = tmp_path / "bad.xml"
    xml.write_text('<?xml version="1.0"?><hemelbsettings version="2"></hemelbsettings>')
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.read_case(str(xml))
    assert e.value.code == -3


def test_batch_preparation_is_host_only(case_dir):
    """hb_batch_prepare_xml parses, reads and lays out a lattice without a device,
    and refuses physics the batched form does not run."""
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_bfl")
    prep = lbm.PreparedLattice(xml, kernel, wall, 100)
    assert prep.sites == info.fluid_sites
    prep.close()
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "stenosis")
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.PreparedLattice(xml, kernel, wall, 100)     # LBGK+LES is not run batched
    assert e.value.code == -7


def test_empty_lattice_is_refused():
    """A lattice with no sites is an argument error, raised before any device work."""
    empty = {"coords": np.zeros((0, 3), np.int64), "dims": [1, 1, 1], "wall_mask": np.zeros(0, np.uint32),
             "iolet_mask": np.zeros(0, np.uint32), "site_type": np.zeros(0, np.int32),
             "iolet_id": np.zeros(0, np.int32)}
    with pytest.raises(lbm.HemeLBError) as e:
        lbm.LBM(lattice=empty, params=lbm.Params())
    assert e.value.code == -1
