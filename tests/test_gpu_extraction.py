"""Extraction and checkpoint output on the GPU path (.xtr v4, .off v1).

The files are decoded here with an independent XDR reader and checked against
the library's own state (property cache, distributions, lattice tables) with the
reference's unit conversions (src/util/UnitConverter.cc) and record semantics
(src/extraction/LocalPropertyOutput.cc, LocalDistributionInput.cc).
"""

import struct

import numpy as np
import pytest

from conftest import make_small_case
from hemepure_b200 import lbm
from oracle import case as ocase

pytestmark = pytest.mark.gpu

CS2 = 1.0 / 3.0
MMHG = 133.3223874


def read_xtr(path):
    data = open(path, "rb").read()
    pos = 0

    def take(fmt):
        nonlocal pos
        v = struct.unpack_from(">" + fmt, data, pos)
        pos += struct.calcsize(">" + fmt)
        return v if len(v) > 1 else v[0]

    magic, xmagic, version = take("III")
    voxel = take("d")
    origin = take("ddd")
    nsites = take("Q")
    nfields, fhl = take("II")
    fields = []
    for _ in range(nfields):
        ln = take("I")
        name = data[pos:pos + ln].decode()
        pos += (ln + 3) // 4 * 4
        width = take("I")
        offset = take("d")
        fields.append((name, width, offset))
    header_len = pos
    per_site = 3 + sum(w for _, w, _ in fields)
    rec_len = 8 + 4 * per_site * nsites
    records = []
    while pos < len(data):
        label = take("Q")
        body = np.frombuffer(data, dtype=">u4", count=per_site * nsites, offset=pos).reshape(nsites, per_site)
        pos += 4 * per_site * nsites
        coords = body[:, :3].astype(np.int64)
        vals = body[:, 3:].copy().view(">f4").astype(np.float32)
        out, c = {}, 0
        for name, width, _ in fields:
            out[name] = vals[:, c:c + width]
            c += width
        records.append((label, coords, out))
    return {"magic": (magic, xmagic, version), "voxel": voxel, "origin": origin, "nsites": nsites,
            "fields": fields, "header_len": header_len, "rec_len": rec_len, "records": records}


def units(xml, kernel):
    cfg = ocase.load_case(xml, kernel)
    dx, dt = cfg.dx, cfg.dt
    mass = 1000.0 * dx * dx * dx
    return dx, dt, mass / (dx * dt * dt), dx / dt


def test_xtr_fields_match_state(case_dir, tmp_path):
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(40, macro=True)
    rho, u, wss = sim.GetPropertyCache()
    path, off = tmp_path / "out.xtr", tmp_path / "out.off"
    sim.WriteXtr(path, ["pressure", "velocity", "shearstress", "distributions"], off)
    x = read_xtr(path)
    assert x["magic"] == (0x686C6221, 0x78747204, 4)
    dx, dt, p_unit, v_unit = units(xml, kernel)
    assert x["voxel"] == dx and x["nsites"] == sim.n
    assert [(n, w) for n, w, _ in x["fields"]] == [("pressure", 1), ("velocity", 3), ("shearstress", 1),
                                                   ("distributions", 19)]
    (label, coords, vals), = x["records"]
    assert label == sim.time_step - 1
    assert np.array_equal(coords, sim.tables()["coords"])
    with np.errstate(over="ignore"):
        assert np.array_equal(vals["pressure"][:, 0], ((rho * CS2 - CS2) * p_unit / MMHG).astype(np.float32))
        assert np.array_equal(vals["velocity"], (u * v_unit).astype(np.float32))
        assert np.array_equal(vals["shearstress"][:, 0], (wss * p_unit).astype(np.float32))
    walls = wss < 1e300
    assert np.all(np.isfinite(vals["shearstress"][walls, 0])) and np.all(np.isinf(vals["shearstress"][~walls, 0]))
    # .off: start of the first record and its end
    o = struct.unpack(">IIIIQQ", open(off, "rb").read())
    assert o[:4] == (0x686C6221, 0x6F666604, 1, 1)
    assert o[4] == x["header_len"] and o[5] == x["header_len"] + x["rec_len"]


def test_xtr_field_names(case_dir, tmp_path):
    """A <field type= name=> is written under its name, with the type's values."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_r8")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(5, macro=True)
    sim.WriteXtr(tmp_path / "a.xtr", ["velocity", "pressure"])
    sim.WriteXtr(tmp_path / "b.xtr", ["velocity:inflow", "pressure:p"])
    a, b = read_xtr(tmp_path / "a.xtr"), read_xtr(tmp_path / "b.xtr")
    assert [(n, w) for n, w, _ in b["fields"]] == [("inflow", 3), ("p", 1)]
    (_, _, va), = a["records"]
    (_, _, vb), = b["records"]
    assert np.array_equal(va["velocity"], vb["inflow"]) and np.array_equal(va["pressure"], vb["p"])
    with pytest.raises(lbm.HemeLBError):
        sim.WriteXtr(tmp_path / "c.xtr", ["velocity:"])


def test_xtr_distributions_are_those_entering_the_step(case_dir, tmp_path):
    """A record labelled t carries the distributions that entered step t."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_r8")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(9)
    entering = sim.GetFOld()
    t = sim.time_step
    sim.step(1)
    path = tmp_path / "f.xtr"
    sim.WriteXtr(path, ["distributions"])
    (label, coords, vals), = read_xtr(path)["records"]
    assert label == t
    assert np.array_equal(vals["distributions"], entering.astype(np.float32))


def test_checkpoint_round_trip(case_dir, tmp_path):
    """Records appended at two steps; restoring either by its label resumes the run
    from the float32 distributions at that label."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    a = lbm.LBM(xml, kernel=kernel, wall=wall)
    path = tmp_path / "cp.xtr"
    a.step(10)
    a.WriteXtr(path, ["distributions"])
    a.step(5)
    a.WriteXtr(path, ["distributions"])
    x = read_xtr(path)
    labels = [r[0] for r in x["records"]]
    assert labels == [10, 15]
    for label, _, vals in x["records"]:
        b = lbm.LBM(xml, kernel=kernel, wall=wall)
        b.ReadCheckpoint(path, label)
        assert b.time_step == label
        assert np.array_equal(b.GetFOld(), vals["distributions"].astype(np.float64))
    # resume from the last record and compare with the uninterrupted run
    c = lbm.LBM(xml, kernel=kernel, wall=wall)
    c.ReadCheckpoint(path)
    ref = lbm.LBM(xml, kernel=kernel, wall=wall)
    ref.step(14)
    c.step(20)
    ref.step(20)
    fc, fr = c.GetFOld(), ref.GetFOld()
    assert np.max(np.abs(fc - fr)) <= 1e-6 * np.max(np.abs(fr))


def test_checkpoint_rejects_a_missing_step_and_a_wrong_lattice(case_dir, tmp_path):
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_r8")
    a = lbm.LBM(xml, kernel=kernel, wall=wall)
    a.step(3)
    path = tmp_path / "cp.xtr"
    a.WriteXtr(path, ["distributions"])
    b = lbm.LBM(xml, kernel=kernel, wall=wall)
    with pytest.raises(lbm.HemeLBError):
        b.ReadCheckpoint(path, 7)
    xml2, _, _, kernel2, wall2, _ = make_small_case(case_dir, "pipe_bfl")
    c = lbm.LBM(xml2, kernel=kernel2, wall=wall2)
    with pytest.raises(lbm.HemeLBError) as e:
        c.ReadCheckpoint(path)
    assert e.value.code == -3


def test_selected_record_is_the_whole_record_restricted(case_dir, tmp_path):
    """A record for a plane or a sphere holds exactly the sites the selector takes,
    with the same values as the whole-lattice record at those sites."""
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(30, macro=True)
    fields = ["pressure", "velocity", "shearstress"]
    sim.WriteXtr(tmp_path / "whole.xtr", fields)
    (_, wcoords, wvals), = read_xtr(tmp_path / "whole.xtr")["records"]
    dx = units(xml, kernel)[0]
    lo, hi = wcoords.min(0), wcoords.max(0)
    mid = (lo + hi) / 2.0 * dx
    geo = lbm.Geometry(gmy)
    for sel in (lbm.selector("plane", point=mid, normal=(0, 0, 1)),
                lbm.selector("sphere", point=mid, radius=0.6 * (hi[0] - lo[0]) / 2.0 * dx),
                lbm.selector("surface")):
        path = tmp_path / f"sel{sel.type}.xtr"
        sim.WriteXtr(path, fields, geometry=sel)
        x = read_xtr(path)
        mask = geo.select(sel, dx, (0.0, 0.0, 0.0))
        assert x["nsites"] == int(mask.sum()) > 0
        (label, coords, vals), = x["records"]
        assert np.array_equal(coords, wcoords[mask])
        for f in fields:
            assert np.array_equal(vals[f], wvals[f][mask])


def test_device_selection_is_byte_identical_to_host_selection(case_dir, tmp_path):
    """Every selector type, selected and gathered on the device: the file equals,
    byte for byte, the whole-lattice file restricted to the sites the host
    selector (the reference's float arithmetic, hb_geometry_select) takes, with
    macroscopic fields, stress caches and distributions."""
    import struct as st
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(40, macro=True, stress=True)
    fields = ["pressure", "velocity", "shearstress", "vonmisesstress", "stresstensor", "traction", "distributions"]
    whole = tmp_path / "whole.xtr"
    sim.WriteXtr(whole, fields)
    w = read_xtr(whole)
    raw = open(whole, "rb").read()
    hdr = raw[:w["header_len"]]
    per_site = 4 * (3 + sum(width for _, width, _ in w["fields"]))
    body = raw[w["header_len"] + 8:]
    label = raw[w["header_len"]:w["header_len"] + 8]
    (_, wcoords, wvals), = w["records"]
    dx = units(xml, kernel)[0]
    lo, hi = wcoords.min(0), wcoords.max(0)
    mid = (lo + hi) / 2.0 * dx
    r = (hi[0] - lo[0]) / 2.0 * dx
    wall_site = wcoords[np.flatnonzero(np.abs(wvals["shearstress"][:, 0]) < 1e30)[len(wcoords) // 100]] * dx
    geo = lbm.Geometry(gmy)
    sels = [lbm.selector("whole"),
            lbm.selector("plane", point=mid, normal=(0, 0, 1)),
            lbm.selector("plane", point=mid, normal=(0, 1, 1), radius=0.5 * r),
            lbm.selector("line", point=lo * dx, point2=hi * dx),
            lbm.selector("sphere", point=mid, radius=0.6 * r),
            lbm.selector("inlet"), lbm.selector("outlet"), lbm.selector("surface"),
            lbm.selector("surfaceWithinSphere", point=mid, radius=1.3 * r),
            lbm.selector("surfacepoint", point=wall_site)]
    for k, sel in enumerate(sels):
        path = tmp_path / f"sel{k}.xtr"
        sim.WriteXtr(path, fields, geometry=sel)
        mask = geo.select(sel, dx, (0.0, 0.0, 0.0))
        assert mask.any(), k
        expect = bytearray(hdr)
        expect[44:52] = st.pack(">Q", int(mask.sum()))
        rows = [body[j * per_site:(j + 1) * per_site] for j in np.flatnonzero(mask)]
        expect += label + b"".join(rows)
        assert open(path, "rb").read() == bytes(expect), (k, sel.type)
