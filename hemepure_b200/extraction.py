"""Property outputs of a case file: which fields of which sites go to which .xtr
file at which steps.

Restates SimConfig::DoIOForProperties / DoIOForPropertyOutputFile and the
geometry readers (src/configuration/SimConfig.cc:409-564) and the write test
LocalPropertyOutput::ShouldWrite (src/extraction/LocalPropertyOutput.cc:205-210).
The records themselves are written by the library (`LBM.WriteXtr`).
"""

from __future__ import annotations

import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass
from typing import List

from . import lbm

# OutputField types (src/extraction/OutputField.h:17-31, SimConfig::DoIOForPropertyField,
# src/configuration/SimConfig.cc:566-632), all written by the library.
WRITABLE_FIELDS = ("pressure", "velocity", "shearstress", "vonmisesstress", "shearrate", "stresstensor", "traction",
                   "tangentialprojectiontraction", "normalprojectiontraction", "wallextension", "distributions",
                   "mpirank")
# Types read from the stress caches: the step before such a record runs with stress=True.
STRESS_FIELDS = tuple(lbm.STRESS_FIELDS)


@dataclass
class PropertyOutput:
    file: str
    period: int
    start: int
    stop: int
    geometry: lbm.Selector
    fields: List[str]
    names: List[str] = None  # header name of each field (the type when the case gives none)

    def field_specs(self) -> List[str]:
        """The fields as the library's writer takes them: "type", or "type:name"
        when the case names the field."""
        names = self.names or self.fields
        return [t if n == t else f"{t}:{n}" for t, n in zip(self.fields, names)]

    def due(self, time_step: int) -> bool:
        """LocalPropertyOutput::ShouldWrite for a record labelled `time_step`."""
        return self.start <= time_step <= self.stop and time_step % self.period == 0


def _value(el, units: str) -> str:
    if el is None:
        raise ValueError("missing element")
    if el.get("units") != units:
        raise ValueError(f"invalid units for {el.tag}: expected {units!r}, got {el.get('units')!r}")
    return el.get("value")


def _vec(el, units: str):
    s = _value(el, units).strip()
    if not (s.startswith("(") and s.endswith(")")):
        raise ValueError(f"bad vector {s!r}")
    parts = [float(p) for p in s[1:-1].split(",")]
    if len(parts) != 3:
        raise ValueError(f"bad vector {s!r}")
    return parts


def _geometry(el) -> lbm.Selector:
    kind = el.get("type")
    if kind not in lbm.SELECTORS:
        raise ValueError(f"Unrecognised property output geometry selector '{kind}'")
    if kind == "plane":
        radius_el = el.find("radius")
        radius = float(_value(radius_el, "m")) if radius_el is not None else 0.0
        return lbm.selector("plane", point=_vec(el.find("point"), "m"),
                            normal=_vec(el.find("normal"), "dimensionless"), radius=radius)
    if kind == "line":
        points = el.findall("point")
        if len(points) < 2:
            raise ValueError("a line selector needs two <point> elements")
        return lbm.selector("line", point=_vec(points[0], "m"), point2=_vec(points[1], "m"))
    if kind in ("sphere", "surfaceWithinSphere"):
        return lbm.selector(kind, point=_vec(el.find("point"), "m"), radius=float(_value(el.find("radius"), "m")))
    if kind == "surfacepoint":
        return lbm.selector(kind, point=_vec(el.find("point"), "m"))
    return lbm.selector(kind)


def property_outputs(xml_path: str) -> List[PropertyOutput]:
    """The <propertyoutput> entries of a case file, in file order."""
    root = ET.parse(xml_path).getroot()
    props = root.find("properties")
    out: List[PropertyOutput] = []
    if props is None:
        return out
    for po in props.findall("propertyoutput"):
        file = po.get("file")
        if file is None or po.get("period") is None:
            raise ValueError("a <propertyoutput> needs 'file' and 'period'")
        geom = po.find("geometry")
        if geom is None:
            raise ValueError("a <propertyoutput> needs a <geometry>")
        fields, names = [], []
        for f in po.findall("field"):
            kind = f.get("type")
            if kind not in WRITABLE_FIELDS:
                raise ValueError(f"Unrecognised field type '{kind}'")
            fields.append(kind)
            names.append(f.get("name", kind))
        out.append(PropertyOutput(file=file, period=int(po.get("period")), start=int(po.get("start", 0)),
                                  stop=int(po.get("stop", 1000000000)), geometry=_geometry(geom), fields=fields, names=names))
    return out


def needs_stress(outputs: List[PropertyOutput], label: int) -> bool:
    """Whether a record labelled `label` due now reads a stress cache."""
    return any(o.due(label) and any(f in STRESS_FIELDS for f in o.fields) for o in outputs)


def write_due(sim: "lbm.LBM", outputs: List[PropertyOutput], directory: str) -> List[str]:
    """Append a record to every output due for the step just completed; returns
    the files written.  Outputs other than distributions need the step run with
    the macroscopic caches filled, and the stress types with the stress caches."""
    label = sim.time_step - 1
    written = []
    for o in outputs:
        if o.due(label):
            path = os.path.join(directory, o.file)
            sim.WriteXtr(path, o.field_specs(), geometry=o.geometry)
            written.append(path)
    return written
