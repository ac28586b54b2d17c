"""Extraction geometry selectors and property-output parsing, on the host.

The selectors are restated here in numpy float32, operation by operation, from
the reference's selector classes (src/extraction/PlaneGeometrySelector.cc:54-81,
StraightLineGeometrySelector.cc:30-49, SphereGeometrySelector.cc,
SurfacePointSelector.cc:22-40, GeometrySurfaceSelector.cc, InletSelector.cc,
OutletSelector.cc), and compared with the library's masks site by site.
"""

import numpy as np
import pytest

from conftest import make_small_case
from hemepure_b200 import extraction, lbm, vessels
from oracle import case as ocase

F = np.float32


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def reference_mask(tb, kind, voxel, origin, point=(0, 0, 0), point2=(0, 0, 0), normal=(0, 0, 1), radius=0.0):
    coords = tb["coords"]
    c = (coords.astype(F).astype(np.float64) * voxel + np.asarray(origin, np.float64)).astype(F)
    P, P2 = np.asarray(point, np.float64).astype(F), np.asarray(point2, np.float64).astype(F)
    n = np.asarray(normal, np.float64).astype(F)
    if np.any(n != 0):
        n = n / np.sqrt(F(_dot(n, n)))
    r = F(radius)
    wall = tb["wall_mask"] != 0
    if kind == "whole":
        return np.ones(len(coords), bool)
    if kind == "plane":
        perp = _dot(c - P, n)
        keep = ~(np.abs(perp) > 0.5 * voxel)
        if r <= 0.0:
            return keep
        d = (c - n * perp[:, None]) - P
        return keep & (_dot(d, d) <= r * r)
    if kind == "line":
        L = P2 - P
        llen = np.sqrt(F(_dot(L, L)))
        along = _dot(np.broadcast_to(L, c.shape), c - P) / llen
        keep = ~((along < 0.0) | (along > llen))
        d = (P + (L * along[:, None]) / llen) - c
        return keep & (_dot(d, d) <= 2.0 * 0.5 * 0.5 * voxel * voxel)
    dist = np.sqrt(_dot(c - P, c - P))
    if kind == "sphere":
        return dist <= r
    if kind == "surfaceWithinSphere":
        return wall & (dist <= r)
    if kind == "surfacepoint":
        return wall & ((dist.astype(np.float64) / voxel).astype(F) <= F(np.sqrt(3.0)))
    if kind == "surface":
        return wall
    if kind == "inlet":
        return tb["site_type"] == 1
    if kind == "outlet":
        return tb["site_type"] == 2
    raise ValueError(kind)


@pytest.fixture(scope="module")
def pipe(case_dir):
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    cfg = ocase.load_case(xml, kernel)
    g = lbm.Geometry(gmy)
    return g, g.tables(), cfg.dx, [0.0, 0.0, 0.0]


def _cases(dx, coords):
    lo, hi = coords.min(0), coords.max(0)
    mid = (lo + hi) / 2.0 * dx
    r = (hi[0] - lo[0]) / 2.0 * dx
    return [
        ("whole", {}),
        ("plane", {"point": mid, "normal": (0, 0, 1)}),
        ("plane", {"point": mid, "normal": (0, 0, 1), "radius": 0.5 * r}),
        ("plane", {"point": mid, "normal": (0.3, 0.0, 1.0), "radius": 0.7 * r}),
        ("line", {"point": (mid[0], mid[1], lo[2] * dx), "point2": (mid[0], mid[1], hi[2] * dx)}),
        ("line", {"point": (lo[0] * dx, mid[1], mid[2]), "point2": (hi[0] * dx, mid[1] + 3 * dx, mid[2])}),
        ("sphere", {"point": mid, "radius": 0.8 * r}),
        ("surfaceWithinSphere", {"point": mid, "radius": 1.2 * r}),
        ("surfacepoint", {"point": (mid[0] + r, mid[1], mid[2])}),
        ("surface", {}),
        ("inlet", {}),
        ("outlet", {}),
    ]


def test_selectors_match_the_reference_float_arithmetic(pipe):
    g, tb, dx, origin = pipe
    for kind, kw in _cases(dx, tb["coords"]):
        got = g.select(lbm.selector(kind, **kw), dx, origin)
        want = reference_mask(tb, kind, dx, origin, **kw)
        assert got.sum() > 0, kind
        assert np.array_equal(got, want), (kind, int(got.sum()), int(want.sum()))


def test_property_outputs_are_read_from_the_case(tmp_path):
    v = vessels.Pipe(4, 16)
    gmy = tmp_path / "p.gmy"
    vessels.voxelise(v, str(gmy))
    xml = tmp_path / "p.xml"
    props = [{"file": "whole.xtr", "period": 10, "fields": ["pressure", "velocity"]},
             {"file": "plane.xtr", "period": 5, "geometry": {"type": "plane", "point": (1e-4, 2e-4, 3e-4),
                                                            "normal": (0, 0, 1), "radius": 5e-4},
              "fields": ["shearstress"]},
             {"file": "line.xtr", "period": 7, "geometry": {"type": "line", "point": (0, 0, 0), "point2": (0, 0, 1e-3)},
              "fields": ["distributions"]}]
    vessels.write_case_xml(str(xml), "p.gmy", v, vessels.CaseUnits(tau=0.8), 100, [vessels.PressureBC(1.001)],
                           [vessels.PressureBC(0.999)], properties=props)
    outs = extraction.property_outputs(str(xml))
    assert [o.file for o in outs] == ["whole.xtr", "plane.xtr", "line.xtr"]
    assert outs[0].geometry.type == lbm.SELECTORS["whole"] and outs[0].fields == ["pressure", "velocity"]
    p = outs[1].geometry
    assert p.type == lbm.SELECTORS["plane"] and list(p.point) == [1e-4, 2e-4, 3e-4] and p.radius == 5e-4
    assert list(outs[2].geometry.point2) == [0, 0, 1e-3]
    assert outs[1].due(10) and not outs[1].due(11) and outs[2].due(0) and outs[2].due(14)
    assert not extraction.needs_stress(outs, 10)


def test_every_output_field_type_is_accepted(tmp_path):
    """All twelve OutputField types of SimConfig::DoIOForPropertyField are read;
    an unknown type is an error, as in the reference."""
    v = vessels.Pipe(4, 16)
    gmy = tmp_path / "p.gmy"
    vessels.voxelise(v, str(gmy))
    xml = tmp_path / "p.xml"
    props = [{"file": "all.xtr", "period": 4, "fields": list(extraction.WRITABLE_FIELDS)}]
    vessels.write_case_xml(str(xml), "p.gmy", v, vessels.CaseUnits(tau=0.8), 100, [vessels.PressureBC(1.001)],
                           [vessels.PressureBC(0.999)], properties=props)
    (o,) = extraction.property_outputs(str(xml))
    assert o.fields == list(extraction.WRITABLE_FIELDS) and len(o.fields) == 12
    assert extraction.needs_stress([o], 8) and not extraction.needs_stress([o], 9)
    assert o.field_specs() == o.fields
    named = tmp_path / "named.xml"
    vessels.write_case_xml(str(named), "p.gmy", v, vessels.CaseUnits(tau=0.8), 100, [vessels.PressureBC(1.001)],
                           [vessels.PressureBC(0.999)], properties=[{"file": "n.xtr", "period": 1,
                                                                      "fields": ["velocity:v", "pressure"]}])
    (n,) = extraction.property_outputs(str(named))
    assert n.fields == ["velocity", "pressure"] and n.names == ["v", "pressure"]
    assert n.field_specs() == ["velocity:v", "pressure"]
    bad = tmp_path / "bad.xml"
    vessels.write_case_xml(str(bad), "p.gmy", v, vessels.CaseUnits(tau=0.8), 100, [vessels.PressureBC(1.001)],
                           [vessels.PressureBC(0.999)], properties=[{"file": "x.xtr", "period": 1,
                                                                      "fields": ["vorticity"]}])
    with pytest.raises(ValueError):
        extraction.property_outputs(str(bad))
