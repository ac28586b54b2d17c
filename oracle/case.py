"""Case-file reader for the CPU oracle (test infrastructure only).

An independent Python restatement of the reference's XML v3 handling and unit
conversion, kept apart from the product's C++ reader so that the two check each
other:

* `src/configuration/SimConfig.cc:84-198` (simulation section, extra warm-up steps),
  `:262-408` (iolets), `:640-655` (iolet position in lattice units, normalised normal),
  `:668-723` (initial conditions, sponge layer), `:725-754` (cosine),
  `:756-794` (file pressure, WK2), `:796-824` (WK3), `:826-854` (fileWK),
  `:856-876` (parabolic), `:878-901` (Womersley), `:937-954` (file velocity);
* `src/lb/iolets/InOutLetFile.cc:48-127` (the file pressure iolet's density table),
  `src/lb/iolets/InOutLetFileVelocity.cc:34-101` (the file velocity iolet's table);
* `src/util/UnitConverter.cc:15-118`, `src/util/UnitConverter.h:153-203`;
* `src/lb/LbmParameters.h:29-37` (tau from dt and dx), `src/constants.h`.
"""

from __future__ import annotations

import math
import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import List, Optional

CS2 = 1.0 / 3.0
MMHG_TO_PASCAL = 133.3223874
BLOOD_DENSITY = 1000.0
BLOOD_VISCOSITY = 0.004
REFERENCE_PRESSURE_MMHG = 0.0


def _vec(s: str):
    s = s.strip()
    if not (s.startswith("(") and s.endswith(")")):
        raise ValueError(f"bad vector {s!r}")
    parts = [float(p) for p in s[1:-1].split(",")]
    if len(parts) != 3:
        raise ValueError(f"bad vector {s!r}")
    return parts


def _val(el, units: str, conv=float):
    got = el.get("units")
    if got != units:
        raise ValueError(f"invalid units for {el.tag}: expected {units!r}, got {got!r}")
    return conv(el.get("value"))


class Units:
    def __init__(self, dt: float, dx: float, origin):
        self.dx, self.dt = dx, dt
        self.mass = BLOOD_DENSITY * dx * dx * dx
        self.speed = dx / dt
        self.pressure = self.mass / (dx * dt * dt)

    def pressure_to_lattice(self, p_mmhg: float) -> float:
        return CS2 + self.pressure_diff_to_lattice(p_mmhg - REFERENCE_PRESSURE_MMHG)

    def pressure_diff_to_lattice(self, dp: float) -> float:
        return dp * MMHG_TO_PASCAL / self.pressure

    def to_lattice(self, units: str, value: float) -> float:
        if units == "m":
            sf = self.dx
        elif units == "s":
            sf = self.dt
        elif units in ("rad", "dimensionless"):
            sf = 1.0
        elif units == "m/s":
            sf = self.dx / self.dt
        elif units == "mmHg":
            sf = self.mass / (self.dx * self.dt * self.dt) / MMHG_TO_PASCAL
        elif units == "mmHg/m":
            sf = self.mass / (self.dx * self.dx * self.dt * self.dt) / MMHG_TO_PASCAL
        else:
            raise ValueError(units)
        return value / sf

    def resistance(self, r: float) -> float:
        return r * ((self.dt * self.dx) / BLOOD_DENSITY)

    def capacitance(self, c: float) -> float:
        return c * (BLOOD_DENSITY / (self.dt * self.dt * self.dx))

    def area(self, a: float) -> float:
        return a / (self.dx * self.dx)


@dataclass
class IoletCfg:
    kind: str                  # a key of oracle.IOLET_KINDS
    position: List[float]
    normal: List[float]
    density_mean: float = 0.0
    density_amp: float = 0.0
    phase: float = 0.0
    period: float = 0.0
    warmup: int = 0
    radius: float = 0.0
    max_speed: float = 0.0
    rc: float = 0.0
    rp: float = 0.0
    cp: float = 0.0
    area: float = 0.0
    table: Optional[List[float]] = None   # file pressure: density per 0-indexed step;
    density_min: float = 0.0              # file velocity: peak speed per 1-based step
    pressure_gradient_amplitude: float = 0.0   # Womersley
    womersley_number: float = 0.0


@dataclass
class CaseCfg:
    gmy_path: str
    tau: float
    total_steps: int
    warmup: int
    initial_density: float
    initial_step: int
    relaxation_parameter: float
    viscosity_ratio: float
    sponge_width: float
    sponge_lifetime: int
    inlets: List[IoletCfg] = field(default_factory=list)
    outlets: List[IoletCfg] = field(default_factory=list)
    dt: float = 0.0
    dx: float = 0.0


def _read_time_value_pairs(path: str):
    """`while (file.good()) { file >> t >> v; pairs[t] = v; }`: a file whose last
    number is followed by whitespace makes one more pass, in which the stream
    reaches its end while skipping whitespace, so neither extraction runs and
    the last pair is stored again unchanged."""
    tokens = open(path).read().split()
    pairs = {}
    for k in range(0, len(tokens) - 1, 2):
        pairs[float(tokens[k])] = float(tokens[k + 1])
    return pairs


def _linear_interpolate(xs, ys, x):
    """util::NumericalFunctions::LinearInterpolate (src/util/utilityFunctions.h:96-134)."""
    i = 0
    while not (x >= xs[i] and x <= xs[i + 1]):
        i += 1
        if i + 1 >= len(xs):
            raise ValueError("interpolation beyond the file's time range")
    return ys[i] + (x - xs[i]) / (xs[i + 1] - xs[i]) * (ys[i + 1] - ys[i])


def file_density_table(path: str, total_steps: int, dt: float, u: "Units"):
    """InOutLetFile::CalculateTable (src/lb/iolets/InOutLetFile.cc:48-127): the
    lattice density at every step 0..total_steps, and the minimum density."""
    pairs = _read_time_value_pairs(path)
    times, values = [], []
    entries = sorted(pairs.items())
    p_min = p_max = entries[0][1]
    end = total_steps * dt
    for t, v in entries:
        if t > end:
            ratio = (end - times[-1]) / (t - times[-1])
            final = values[-1] + ratio * (v - values[-1])
            times.append(end)
            p_min, p_max = min(p_min, final), max(p_max, final)
            values.append(final)
            break
        p_min, p_max = min(p_min, v), max(p_max, v)
        times.append(t)
        values.append(v)
    density_min = u.pressure_to_lattice(p_min) / CS2
    period_steps = int(times[-1] / dt)
    if period_steps <= 0:
        raise ValueError("the file's time range is shorter than one step")
    table = []
    for step in range(total_steps + 1):
        point = times[0] + (float(step % period_steps) / float(total_steps)) * (times[-1] - times[0])
        table.append(u.pressure_to_lattice(_linear_interpolate(times, values, point)) / CS2)
    return table, density_min


def file_velocity_table(path: str, total_steps: int, dt: float, u: "Units"):
    """InOutLetFileVelocity::CalculateTable (src/lb/iolets/InOutLetFileVelocity.cc:34-101):
    the lattice peak speed at every step 0..total_steps, the file's (time in s,
    speed in m/s) profile clipped at the run's end and looped like the pressure
    table."""
    pairs = _read_time_value_pairs(path)
    times, values = [], []
    end = total_steps * dt
    for t, v in sorted(pairs.items()):
        if t > end:
            ratio = (end - times[-1]) / (t - times[-1])
            times.append(end)
            values.append(values[-1] + ratio * (v - values[-1]))
            break
        times.append(t)
        values.append(v)
    period_steps = int(times[-1] / dt)
    if period_steps <= 0:
        raise ValueError("the file's time range is shorter than one step")
    table = []
    for step in range(total_steps + 1):
        point = times[0] + (float(step % period_steps) / float(total_steps)) * (times[-1] - times[0])
        table.append(_linear_interpolate(times, values, point) / u.speed)
    return table


def _normalised(v):
    m2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2]
    if v == [0.0, 0.0, 0.0]:
        return v
    m = math.sqrt(m2)
    return [v[0] / m, v[1] / m, v[2] / m]


def load_case(xml_path: str, kernel: str = "LBGK") -> CaseCfg:
    root = ET.parse(xml_path).getroot()
    if root.tag != "hemelbsettings" or root.get("version") != "3":
        raise ValueError("not a version-3 hemelbsettings file")
    sim = root.find("simulation")
    steps = _val(sim.find("steps"), "lattice", int)
    dt = _val(sim.find("step_length"), "s")
    wu_el = sim.find("extra_warmup_steps")
    warmup = 0
    if wu_el is not None:
        warmup = _val(wu_el, "lattice", int)
        steps += warmup
    relax = 0.0
    if kernel in ("TRT", "TRTSL"):  # SimConfig.cc:165
        relax = _val(sim.find("relaxation_parameter"), "lattice")
    dx = _val(sim.find("voxel_size"), "m")
    origin = _vec(sim.find("origin").get("value"))
    u = Units(dt, dx, origin)
    tau = 0.5 + (dt * BLOOD_VISCOSITY / BLOOD_DENSITY) / (CS2 * dx * dx)
    gmy = root.find("geometry").find("datafile").get("path")
    gmy = os.path.join(os.path.dirname(os.path.abspath(xml_path)), gmy)

    ic = root.find("initialconditions")
    t0 = 0
    tel = ic.find("time")
    if tel is not None:
        t0 = _val(tel, "lattice", int)
    p0 = _val(ic.find("pressure").find("uniform"), "mmHg")
    rho0 = u.pressure_to_lattice(p0) / CS2
    vr = sw = 0.0
    life = 0
    if kernel in ("LBGKSL", "LBGKLESSL", "TRTSL"):  # SimConfig.cc:707
        sp = ic.find("sponge_layer")
        vr = _val(sp.find("viscosity_ratio"), "dimensionless")
        sw = u.to_lattice("m", _val(sp.find("width"), "m"))
        life = _val(sp.find("lifetime"), "lattice", int)

    def iolets(group: str) -> List[IoletCfg]:
        out = []
        for el in root.find(group).findall(group[:-1]):
            cond = el.find("condition")
            pos = _vec(el.find("position").get("value"))
            if el.find("position").get("units") != "lattice":
                raise ValueError("iolet position must be in lattice units")
            nrm = _normalised(_vec(el.find("normal").get("value")))
            typ, sub = cond.get("type"), cond.get("subtype")
            if typ == "pressure" and sub == "cosine":
                io = IoletCfg("cosine", pos, nrm)
                io.density_amp = u.pressure_diff_to_lattice(_val(cond.find("amplitude"), "mmHg")) / CS2
                io.density_mean = u.pressure_to_lattice(_val(cond.find("mean"), "mmHg")) / CS2
                io.phase = u.to_lattice("rad", _val(cond.find("phase"), "rad"))
                io.period = u.to_lattice("s", _val(cond.find("period"), "s"))
                io.warmup = warmup
            elif typ == "pressure" and sub == "WK3":
                io = IoletCfg("wk3", pos, nrm)
                io.rc = u.resistance(_val(cond.find("Rc"), "kg/m^4*s"))
                io.rp = u.resistance(_val(cond.find("Rp"), "kg/m^4*s"))
                io.cp = u.capacitance(_val(cond.find("Cp"), "m^4*s^2/kg"))
                io.radius = u.to_lattice("m", _val(cond.find("radius"), "m"))
                io.area = u.area(_val(cond.find("area"), "m^2"))
            elif typ == "pressure" and sub == "WK2":
                io = IoletCfg("wk2", pos, nrm)
                io.rp = u.resistance(_val(cond.find("R"), "kg/m^4*s"))
                io.cp = u.capacitance(_val(cond.find("C"), "m^4*s^2/kg"))
                io.radius = u.to_lattice("m", _val(cond.find("radius"), "m"))
                io.area = u.area(_val(cond.find("area"), "m^2"))
            elif typ == "pressure" and sub == "file":
                io = IoletCfg("file", pos, nrm)
                path = cond.find("path").get("value")
                path = os.path.normpath(os.path.join(os.path.dirname(os.path.abspath(xml_path)), path))
                io.table, io.density_min = file_density_table(path, steps, dt, u)
            elif typ == "pressure" and sub == "fileWK":
                # InOutLetFileWK behaves as WK2: its weights file is read only in
                # builds with HEMELB_USE_VELOCITY_WEIGHTS_FILE; its radius is unset.
                io = IoletCfg("wk2", pos, nrm)
                if cond.find("path") is None:
                    raise ValueError("fileWK condition without <path>")
                io.rp = u.resistance(_val(cond.find("R"), "kg/m^4*s"))
                io.cp = u.capacitance(_val(cond.find("C"), "m^4*s^2/kg"))
                io.area = u.area(_val(cond.find("area"), "m^2"))
            elif typ == "velocity" and sub == "file":
                io = IoletCfg("file_velocity", pos, nrm)
                path = cond.find("path").get("value")
                path = os.path.normpath(os.path.join(os.path.dirname(os.path.abspath(xml_path)), path))
                io.radius = u.to_lattice("m", _val(cond.find("radius"), "m"))
                io.table = file_velocity_table(path, steps, dt, u)
            elif typ == "velocity" and sub == "womersley":
                io = IoletCfg("womersley", pos, nrm)
                io.radius = u.to_lattice("m", _val(cond.find("radius"), "m"))
                io.pressure_gradient_amplitude = u.to_lattice(
                    "mmHg/m", _val(cond.find("pressure_gradient_amplitude"), "mmHg/m"))
                io.period = u.to_lattice("s", _val(cond.find("period"), "s"))
                io.womersley_number = u.to_lattice("dimensionless", _val(cond.find("womersley_number"), "dimensionless"))
            elif typ == "velocity" and sub == "parabolic":
                io = IoletCfg("parabolic", pos, nrm)
                io.radius = u.to_lattice("m", _val(cond.find("radius"), "m"))
                io.max_speed = u.to_lattice("m/s", _val(cond.find("maximum"), "m/s"))
                io.warmup = warmup
            else:
                raise ValueError(f"unsupported iolet condition {typ}/{sub}")
            out.append(io)
        return out

    return CaseCfg(gmy_path=gmy, tau=tau, total_steps=steps, warmup=warmup, initial_density=rho0,
                   initial_step=t0 if t0 else 1, relaxation_parameter=relax, viscosity_ratio=vr,
                   sponge_width=sw, sponge_lifetime=life, inlets=iolets("inlets"),
                   outlets=iolets("outlets"), dt=dt, dx=dx)
