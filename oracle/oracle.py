"""ctypes front-end of the CPU oracle (test infrastructure only).

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use
this module, as the checker or as the timed CPU baseline.  The product library
never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from . import case as case_mod

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhboracle.so")

KERNELS = {"LBGK": 0, "TRT": 1, "LBGKLESSL": 2, "LBGKSL": 3, "TRTSL": 4}
WALLS = {"SBB": 0, "BFL": 1, "GZS": 2}
IOLET_KINDS = {"cosine": 0, "wk3": 1, "parabolic": 2, "wk2": 3, "file": 4, "file_velocity": 5, "womersley": 6}


def build(force: bool = False) -> str:
    """Compile the oracle (plain C, -ffp-contract=off so no FMA contraction)."""
    src = os.path.join(HERE, "hb_oracle.c")
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "hb_oracle.h"))):
        return LIB_PATH
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-o", LIB_PATH + ".tmp", src, "-lz", "-lm"]
    subprocess.check_call(cmd)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


class _Iolet(C.Structure):
    _fields_ = [("kind", C.c_int), ("position", C.c_double * 3), ("normal", C.c_double * 3),
                ("density_mean", C.c_double), ("density_amp", C.c_double), ("phase", C.c_double),
                ("period", C.c_double), ("warmup", C.c_uint64), ("radius", C.c_double),
                ("max_speed", C.c_double), ("rc", C.c_double), ("rp", C.c_double), ("cp", C.c_double),
                ("area", C.c_double), ("table", C.c_void_p), ("table_len", C.c_uint64), ("density_min", C.c_double),
                ("pressure_gradient_amplitude", C.c_double), ("womersley_number", C.c_double)]


class _Params(C.Structure):
    _fields_ = [("kernel", C.c_int), ("wall", C.c_int), ("tau", C.c_double),
                ("relaxation_parameter", C.c_double), ("viscosity_ratio", C.c_double),
                ("sponge_width", C.c_double), ("sponge_lifetime", C.c_uint64),
                ("initial_density", C.c_double), ("initial_step", C.c_uint64),
                ("n_inlets", C.c_int), ("n_outlets", C.c_int),
                ("inlets", _Iolet * 16), ("outlets", _Iolet * 16)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P, I64 = C.c_void_p, C.c_int64
        L.orc_lattice_load.argtypes = [C.c_char_p, C.POINTER(P), C.c_char_p, C.c_int]
        L.orc_lattice_free.argtypes = [P]
        L.orc_site_count.argtypes = [P]
        L.orc_site_count.restype = I64
        L.orc_type_counts.argtypes = [P, P]
        L.orc_dims.argtypes = [P, P, P]
        for name in ("orc_get_coords", "orc_get_neighbours", "orc_get_wall_distance", "orc_get_wall_normal"):
            getattr(L, name).argtypes = [P, P]
        L.orc_get_sitedata.argtypes = [P, P, P, P, P]
        L.orc_sim_create.argtypes = [P, C.POINTER(_Params), C.POINTER(P), C.c_char_p, C.c_int]
        L.orc_sim_free.argtypes = [P]
        L.orc_sim_set_threads.argtypes = [P, C.c_int]
        L.orc_sim_run.argtypes = [P, I64, C.c_int]
        L.orc_sim_time_step.argtypes = [P]
        L.orc_sim_time_step.restype = C.c_uint64
        L.orc_sim_get_f.argtypes = [P, P]
        L.orc_sim_set_f.argtypes = [P, P]
        L.orc_sim_get_macro.argtypes = [P, P, P, P]
        L.orc_sim_get_stress.argtypes = [P, C.c_int, P]
        L.orc_sim_get_wk3.argtypes = [P, C.c_int, C.c_int, P]
        L.orc_sim_get_vtau.argtypes = [P, P]
        L.orc_iolet_velocity.argtypes = [C.POINTER(_Iolet), P, C.c_uint64, P]
        L.orc_bessel_j0.argtypes = [C.c_double, C.c_double, P]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Lattice:
    """The reference's classified lattice: contiguous order and integer tables."""

    def __init__(self, gmy_path: str):
        L = lib()
        h = C.c_void_p()
        err = C.create_string_buffer(256)
        rc = L.orc_lattice_load(gmy_path.encode(), C.byref(h), err, 256)
        if rc != 0:
            raise RuntimeError(f"oracle: cannot load {gmy_path}: {err.value.decode()} ({rc})")
        self._h = h
        self.n = int(L.orc_site_count(h))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_lattice_free(self._h)
            self._h = None

    def type_counts(self):
        a = np.zeros(6, np.int64)
        lib().orc_type_counts(self._h, _ptr(a))
        return a

    def coords(self):
        a = np.zeros((self.n, 3), np.int64)
        lib().orc_get_coords(self._h, _ptr(a))
        return a

    def neighbours(self):
        a = np.zeros((self.n, 19), np.int64)
        lib().orc_get_neighbours(self._h, _ptr(a))
        return a

    def sitedata(self):
        w = np.zeros(self.n, np.uint32)
        io = np.zeros(self.n, np.uint32)
        t = np.zeros(self.n, np.int32)
        i = np.zeros(self.n, np.int32)
        lib().orc_get_sitedata(self._h, _ptr(w), _ptr(io), _ptr(t), _ptr(i))
        return w, io, t, i

    def wall_distance(self):
        a = np.zeros((self.n, 18), np.float64)
        lib().orc_get_wall_distance(self._h, _ptr(a))
        return a

    def wall_normal(self):
        a = np.zeros((self.n, 3), np.float64)
        lib().orc_get_wall_normal(self._h, _ptr(a))
        return a


def make_params(cfg: case_mod.CaseCfg, kernel: str, wall: str, keep: Optional[list] = None) -> _Params:
    """The oracle's parameter block; file iolets' density tables are appended to
    `keep`, which must outlive the simulation that uses them."""
    p = _Params()
    p.kernel = KERNELS[kernel]
    p.wall = WALLS[wall]
    p.tau = cfg.tau
    p.relaxation_parameter = cfg.relaxation_parameter
    p.viscosity_ratio = cfg.viscosity_ratio
    p.sponge_width = cfg.sponge_width
    p.sponge_lifetime = cfg.sponge_lifetime
    p.initial_density = cfg.initial_density
    p.initial_step = cfg.initial_step
    for group, src in ((p.inlets, cfg.inlets), (p.outlets, cfg.outlets)):
        for k, io in enumerate(src):
            d = group[k]
            d.kind = IOLET_KINDS[io.kind]
            d.position[:] = io.position
            d.normal[:] = io.normal
            d.density_mean, d.density_amp, d.phase, d.period = io.density_mean, io.density_amp, io.phase, io.period
            d.warmup = io.warmup
            d.radius, d.max_speed = io.radius, io.max_speed
            d.rc, d.rp, d.cp, d.area = io.rc, io.rp, io.cp, io.area
            d.pressure_gradient_amplitude, d.womersley_number = io.pressure_gradient_amplitude, io.womersley_number
            if io.table is not None:
                tab = np.ascontiguousarray(io.table, dtype=np.float64)
                if keep is not None:
                    keep.append(tab)
                d.table = tab.ctypes.data
                d.table_len = len(tab)
                d.density_min = io.density_min
    p.n_inlets = len(cfg.inlets)
    p.n_outlets = len(cfg.outlets)
    return p


def iolet_params(cfg: case_mod.IoletCfg, keep: list) -> _Iolet:
    """One iolet's oracle parameter block (its table appended to `keep`)."""
    c = case_mod.CaseCfg(gmy_path="", tau=1.0, total_steps=0, warmup=0, initial_density=1.0, initial_step=1,
                         relaxation_parameter=0.0, viscosity_ratio=0.0, sponge_width=0.0, sponge_lifetime=0,
                         inlets=[cfg])
    p = make_params(c, "LBGK", "SBB", keep)
    return p.inlets[0]


def iolet_velocity(cfg: case_mod.IoletCfg, x, t: int) -> np.ndarray:
    """The oracle's InOutLetVelocity::GetVelocity (raises ValueError outside the radius)."""
    keep = []
    io = iolet_params(cfg, keep)
    xv = np.ascontiguousarray(x, np.float64)
    v = np.zeros(3, np.float64)
    rc = lib().orc_iolet_velocity(C.byref(io), _ptr(xv), int(t), _ptr(v))
    if rc != 0:
        raise ValueError(f"orc_iolet_velocity: {rc}")
    return v


def bessel_j0(z: complex) -> complex:
    """util::BesselJ0ComplexArgument (tolSq 1e-12) as the oracle restates it."""
    out = np.zeros(2, np.float64)
    lib().orc_bessel_j0(float(z.real), float(z.imag), _ptr(out))
    return complex(out[0], out[1])


class Simulation:
    """The reference's FP64 push-form time step on the CPU."""

    def __init__(self, xml_path: str, kernel: str = "LBGK", wall: str = "SBB",
                 lattice: Optional[Lattice] = None, threads: int = 0):
        self.cfg = case_mod.load_case(xml_path, kernel)
        self.lattice = lattice or Lattice(self.cfg.gmy_path)
        self.n = self.lattice.n
        self._tables = []
        params = make_params(self.cfg, kernel, wall, self._tables)
        h = C.c_void_p()
        err = C.create_string_buffer(256)
        rc = lib().orc_sim_create(self.lattice._h, C.byref(params), C.byref(h), err, 256)
        if rc != 0:
            raise RuntimeError(f"oracle: {err.value.decode()}")
        self._h = h
        lib().orc_sim_set_threads(h, threads or os.cpu_count() or 1)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_sim_free(self._h)
            self._h = None

    def run(self, steps: int, macro: bool = False) -> int:
        return int(lib().orc_sim_run(self._h, int(steps), 1 if macro else 0))

    @property
    def time_step(self) -> int:
        return int(lib().orc_sim_time_step(self._h))

    def f(self) -> np.ndarray:
        a = np.zeros((self.n, 19), np.float64)
        lib().orc_sim_get_f(self._h, _ptr(a))
        return a

    def set_f(self, f: np.ndarray) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib().orc_sim_set_f(self._h, _ptr(f))

    def macro(self):
        rho = np.zeros(self.n)
        u = np.zeros((self.n, 3))
        wss = np.zeros(self.n)
        lib().orc_sim_get_macro(self._h, _ptr(rho), _ptr(u), _ptr(wss))
        return rho, u, wss

    # Stress caches: name -> (field index, values per site), as in the library.
    STRESS = {"vonmisesstress": (0, 1), "shearrate": (1, 1), "stresstensor": (2, 6), "traction": (3, 3),
              "tangentialprojectiontraction": (4, 3), "normalprojectiontraction": (5, 3)}

    def stress(self, field: str) -> np.ndarray:
        idx, k = self.STRESS[field]
        out = np.zeros((self.n, k))
        if lib().orc_sim_get_stress(self._h, idx, _ptr(out)) != 0:
            raise RuntimeError("no macro step has filled the stress caches")
        return out

    def wk3(self, group: int, index: int):
        a = np.zeros(4)
        lib().orc_sim_get_wk3(self._h, group, index, _ptr(a))
        return a

    def vtau(self):
        a = np.zeros(self.n)
        lib().orc_sim_get_vtau(self._h, _ptr(a))
        return a
