"""Python mirror of the reference's lb::LBM interface over the C ABI (libhemeb200.so).

The reference drives one time step as RequestComms, PreSend, PreReceive,
PostReceive, EndIteration (src/lb/lb.hpp:191-346); this class keeps those names
and argument meanings.  Distributions and site arrays are in the reference's
contiguous site order.  Errors raise `HemeLBError` carrying the HB_* status,
as the reference throws hemelb::Exception; instability is reported as
`Unstable` (the reference's SimulationState::SetStability(Unstable)).
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhemeb200.so")

HB_OK = 0
HB_UNSTABLE = 1
STATUS_NAMES = {1: "HB_UNSTABLE", -1: "HB_ERR_ARG", -2: "HB_ERR_IO", -3: "HB_ERR_FORMAT", -4: "HB_ERR_CUDA",
                -5: "HB_ERR_OOM", -6: "HB_ERR_BAD_INDEX", -7: "HB_ERR_UNSUPPORTED", -8: "HB_ERR_IOLET_RADIUS",
                -9: "HB_ERR_TIMEOUT"}
KERNELS = {"LBGK": 0, "TRT": 1, "LBGKLESSL": 2, "LBGKSL": 3, "TRTSL": 4}
WALLS = {"SBB": 0, "BFL": 1, "GZS": 2}
PRECISIONS = {"fp64": 0, "fp32": 1, "fp16": 2}
IOLET_KINDS = {"cosine": 0, "wk3": 1, "parabolic": 2, "wk2": 3, "file": 4, "file_velocity": 5, "womersley": 6}
STEP_MACRO = 1
BATCH_FORMS = {"persistent": 0, "split": 1}
STEP_STRESS = 2
# Stress caches (HB_STRESS_*): name -> (index, values per site).
STRESS_FIELDS = {"vonmisesstress": (0, 1), "shearrate": (1, 1), "stresstensor": (2, 6), "traction": (3, 3),
                 "tangentialprojectiontraction": (4, 3), "normalprojectiontraction": (5, 3)}

# Every entry point include/hemeb200.h declares.
EXPORTS = [
    "hb_default_options", "hb_create_from_xml", "hb_create", "hb_destroy", "hb_last_error",
    "hb_request_comms", "hb_pre_send", "hb_pre_receive", "hb_post_receive", "hb_end_iteration",
    "hb_step", "hb_site_count", "hb_time_step", "hb_get_params", "hb_get_fs", "hb_set_fs",
    "hb_get_macro", "hb_get_stress", "hb_set_iolet_densities", "hb_get_wk3", "hb_get_tables", "hb_write_xtr", "hb_read_checkpoint",
    "hb_last_step_timing", "hb_setup_timing", "hb_device_bytes", "hb_read_case", "hb_geometry_open", "hb_geometry_site_count",
    "hb_geometry_tables", "hb_geometry_layout", "hb_geometry_layout_digest", "hb_geometry_close", "hb_profile_steps",
    "hb_set_time_step", "hb_moment_sums", "hb_moment_sums_noalloc",
    "hb_batch_bytes", "hb_batch_create", "hb_batch_destroy", "hb_batch_add_xml", "hb_batch_add", "hb_batch_remove",
    "hb_batch_run", "hb_batch_get_macro", "hb_batch_member_info", "hb_batch_set_tuning", "hb_batch_set_step_form",
    "hb_batch_stats",
    "hb_batch_prepare_xml", "hb_batch_prepare_xml_device", "hb_batch_prep_sites", "hb_batch_add_prepared", "hb_batch_prep_free",
    "hb_write_xtr_selected", "hb_geometry_select", "hb_read_case_iolet_table", "hb_iolet_velocity",
    "hb_shard_plan", "hb_create_shard_from_xml", "hb_shard_halo_sizes", "hb_shard_pack", "hb_shard_unpack",
    "hb_shard_site_ids", "hb_shard_describe", "hb_write_state", "hb_read_state",
    "hb_geometry_open_device", "hb_geometry_read_timing",
]

# Extraction geometry selectors (the <geometry type="..."> of a <propertyoutput>).
SELECTORS = {"whole": 0, "plane": 1, "line": 2, "sphere": 3, "inlet": 4, "outlet": 5, "surface": 6,
             "surfaceWithinSphere": 7, "surfacepoint": 8}


class HemeLBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Unstable(HemeLBError):
    pass


class Options(C.Structure):
    _fields_ = [("kernel", C.c_int), ("wall", C.c_int), ("precision", C.c_int), ("device", C.c_int),
                ("geometry_reader", C.c_int)]


class Iolet(C.Structure):
    _fields_ = [("kind", C.c_int), ("position", C.c_double * 3), ("normal", C.c_double * 3),
                ("density_mean", C.c_double), ("density_amp", C.c_double), ("phase", C.c_double),
                ("period", C.c_double), ("warmup", C.c_uint64), ("radius", C.c_double),
                ("max_speed", C.c_double), ("rc", C.c_double), ("rp", C.c_double), ("cp", C.c_double),
                ("area", C.c_double), ("table", C.c_void_p),
                ("table_steps", C.c_uint64), ("density_min", C.c_double),
                ("pressure_gradient_amplitude", C.c_double), ("womersley_number", C.c_double)]


class Params(C.Structure):
    _fields_ = [("tau", C.c_double), ("relaxation_parameter", C.c_double), ("viscosity_ratio", C.c_double),
                ("sponge_width", C.c_double), ("sponge_lifetime", C.c_uint64), ("initial_density", C.c_double),
                ("initial_step", C.c_uint64), ("n_inlets", C.c_int), ("n_outlets", C.c_int),
                ("inlets", Iolet * 16), ("outlets", Iolet * 16)]


class Selector(C.Structure):
    _fields_ = [("type", C.c_int), ("point", C.c_double * 3), ("point2", C.c_double * 3), ("normal", C.c_double * 3),
                ("radius", C.c_double)]


def selector(type: str = "whole", point=(0.0, 0.0, 0.0), point2=(0.0, 0.0, 0.0), normal=(0.0, 0.0, 1.0),
             radius: float = 0.0) -> Selector:
    """A geometry selector; points and radii in metres, as in the case file."""
    s = Selector()
    s.type = SELECTORS[type]
    s.point[:] = [float(v) for v in point]
    s.point2[:] = [float(v) for v in point2]
    s.normal[:] = [float(v) for v in normal]
    s.radius = float(radius)
    return s


class LatticeDesc(C.Structure):
    _fields_ = [("n_sites", C.c_int64), ("dims", C.c_int64 * 3), ("coords", C.c_void_p),
                ("wall_mask", C.c_void_p), ("iolet_mask", C.c_void_p), ("site_type", C.c_void_p),
                ("iolet_id", C.c_void_p), ("wall_distance", C.c_void_p), ("wall_normal", C.c_void_p),
                ("neighbours", C.c_void_p)]


_lib = None


def library() -> C.CDLL:
    """Load libhemeb200.so; raise if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m hemepure_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, I, I64, U32, U64 = C.c_void_p, C.c_int, C.c_int64, C.c_uint32, C.c_uint64
    L.hb_default_options.argtypes = [P]
    L.hb_default_options.restype = None
    L.hb_create_from_xml.argtypes = [C.c_char_p, P, C.POINTER(P)]
    L.hb_create.argtypes = [P, P, P, C.POINTER(P)]
    L.hb_destroy.argtypes = [P]
    L.hb_last_error.argtypes = [P, C.c_char_p, C.c_size_t]
    for name in ("hb_request_comms", "hb_pre_send", "hb_post_receive", "hb_end_iteration"):
        getattr(L, name).argtypes = [P]
    L.hb_pre_receive.argtypes = [P, U32]
    L.hb_step.argtypes = [P, I64, U32]
    L.hb_site_count.argtypes = [P, P]
    L.hb_time_step.argtypes = [P, P]
    L.hb_get_params.argtypes = [P, P]
    L.hb_get_fs.argtypes = [P, P]
    L.hb_set_fs.argtypes = [P, P]
    L.hb_get_macro.argtypes = [P, P, P, P]
    L.hb_get_stress.argtypes = [P, I, P]
    L.hb_set_iolet_densities.argtypes = [P, P, I, P, I]
    L.hb_get_wk3.argtypes = [P, I, I, P]
    L.hb_get_tables.argtypes = [P, P, P, P, P, P, P, P]
    L.hb_write_xtr.argtypes = [P, C.c_char_p, C.c_char_p, C.c_char_p]
    L.hb_write_xtr_selected.argtypes = [P, C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(Selector)]
    L.hb_geometry_select.argtypes = [P, C.POINTER(Selector), C.c_double, P, P]
    L.hb_read_case_iolet_table.argtypes = [C.c_char_p, I, I, I, P, U64]
    L.hb_iolet_velocity.argtypes = [C.POINTER(Iolet), P, U64, P]
    L.hb_read_checkpoint.argtypes = [P, C.c_char_p, U64]
    L.hb_last_step_timing.argtypes = [P, P, P]
    L.hb_setup_timing.argtypes = [P, P]
    L.hb_device_bytes.argtypes = [P, P]
    L.hb_read_case.argtypes = [C.c_char_p, I, P, C.c_char_p, C.c_size_t]
    L.hb_geometry_open.argtypes = [C.c_char_p, C.POINTER(P)]
    L.hb_geometry_open_device.argtypes = [C.c_char_p, I, C.POINTER(P)]
    L.hb_geometry_read_timing.argtypes = [P, P]
    L.hb_geometry_site_count.argtypes = [P, P, P]
    L.hb_geometry_tables.argtypes = [P] + [P] * 9
    L.hb_geometry_layout.argtypes = [P, P, I, P]
    L.hb_geometry_layout_digest.argtypes = [P, P, I, I, P]
    L.hb_geometry_close.argtypes = [P]
    L.hb_profile_steps.argtypes = [P, I64, P]
    L.hb_set_time_step.argtypes = [P, U64]
    L.hb_moment_sums.argtypes = [P, P]
    L.hb_moment_sums_noalloc.argtypes = [P, I64, I64, I64, P, P]
    L.hb_batch_bytes.argtypes = [I64, I64, I, I, P]
    L.hb_batch_create.argtypes = [I64, I64, I, I, I, C.POINTER(P)]
    L.hb_batch_destroy.argtypes = [P]
    L.hb_batch_add_xml.argtypes = [P, C.c_char_p, I, I, U64, P]
    L.hb_batch_add.argtypes = [P, P, P, I, I, U64, P]
    L.hb_batch_remove.argtypes = [P, I]
    L.hb_batch_run.argtypes = [P, I, P, I, P]
    L.hb_batch_get_macro.argtypes = [P, I, P, P, P]
    L.hb_batch_member_info.argtypes = [P, I, P, P, P]
    L.hb_batch_set_tuning.argtypes = [P, I, I]
    L.hb_batch_set_step_form.argtypes = [P, I]
    L.hb_batch_stats.argtypes = [P, P, P, P]
    L.hb_batch_prepare_xml.argtypes = [C.c_char_p, I, I, U64, C.POINTER(P)]
    L.hb_batch_prepare_xml_device.argtypes = [C.c_char_p, I, I, U64, I, C.POINTER(P)]
    L.hb_batch_prep_sites.argtypes = [P, P]
    L.hb_batch_add_prepared.argtypes = [P, P, P]
    L.hb_batch_prep_free.argtypes = [P]
    L.hb_write_state.argtypes = [P, C.c_char_p]
    L.hb_read_state.argtypes = [P, C.c_char_p]
    L.hb_shard_plan.argtypes = [C.c_char_p, I, I, P, P]
    L.hb_create_shard_from_xml.argtypes = [C.c_char_p, P, P, C.POINTER(P)]
    L.hb_shard_halo_sizes.argtypes = [P, P, P]
    L.hb_shard_pack.argtypes = [P, P, P, P]
    L.hb_shard_unpack.argtypes = [P, P, P, P]
    L.hb_shard_site_ids.argtypes = [P, P]
    L.hb_shard_describe.argtypes = [C.c_char_p, I, I, P, P, P, P, P, P, P, P]
    for name in EXPORTS:
        fn = getattr(L, name)
        if name != "hb_default_options":
            fn.restype = I
    _lib = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def check_rc(rc: int, what: str) -> None:
    """Raise HemeLBError for a failed call that takes no handle."""
    if rc != HB_OK:
        raise HemeLBError(rc, f"{what}: {last_create_error()}")


def _dptr(t) -> Optional[int]:
    """Device pointer of a torch tensor (or None)."""
    return None if t is None else int(t.data_ptr())


GEOMETRY_READERS = {"host": 0, "device": 1}


def _flags(macro: bool, stress: bool) -> int:
    return (STEP_MACRO if macro else 0) | (STEP_STRESS if (macro and stress) else 0)


def options(kernel="LBGK", wall="SBB", precision="fp64", device=0, geometry_reader="device") -> Options:
    o = Options()
    library().hb_default_options(C.byref(o))
    o.kernel = KERNELS[kernel]
    o.wall = WALLS[wall]
    o.precision = PRECISIONS[precision]
    o.device = int(device)
    o.geometry_reader = GEOMETRY_READERS[geometry_reader]
    return o


class LBM:
    """One lattice resident on one GPU: the reference's lb::LBM<D3Q19>."""

    def __init__(self, xml_path: Optional[str] = None, kernel: str = "LBGK", wall: str = "SBB",
                 precision: str = "fp64", device: int = 0, lattice: Optional[Dict[str, np.ndarray]] = None,
                 params: Optional[Params] = None, geometry_reader: str = "device", shard=None):
        """`shard` = (axis, lo, hi): only the slab lo <= coordinate < hi of the
        case's lattice, with its halo (hb_create_shard_from_xml)."""
        L = library()
        self._h = C.c_void_p()
        self._opt = options(kernel, wall, precision, device, geometry_reader)
        if shard is not None:
            from .shard import ShardSpec
            spec = ShardSpec(int(shard[0]), int(shard[1]), int(shard[2]))
            rc = L.hb_create_shard_from_xml(os.fspath(xml_path).encode(), C.byref(self._opt), C.byref(spec),
                                            C.byref(self._h))
        elif xml_path is not None:
            rc = L.hb_create_from_xml(os.fspath(xml_path).encode(), C.byref(self._opt), C.byref(self._h))
        else:
            if lattice is None or params is None:
                raise ValueError("pass an XML case file, or lattice tables and parameters")
            self._keep = {k: np.ascontiguousarray(v) for k, v in lattice.items() if v is not None}
            d = LatticeDesc()
            d.n_sites = int(self._keep["coords"].shape[0])
            d.dims[:] = [int(v) for v in lattice["dims"]]
            for name, key, dt in (("coords", "coords", np.int64), ("wall_mask", "wall_mask", np.uint32),
                                  ("iolet_mask", "iolet_mask", np.uint32), ("site_type", "site_type", np.int32),
                                  ("iolet_id", "iolet_id", np.int32), ("wall_distance", "wall_distance", np.float64),
                                  ("wall_normal", "wall_normal", np.float64), ("neighbours", "neighbours", np.int64)):
                if key in self._keep:
                    self._keep[key] = np.ascontiguousarray(self._keep[key], dtype=dt)
                    setattr(d, name, _p(self._keep[key]))
            rc = L.hb_create(C.byref(d), C.byref(params), C.byref(self._opt), C.byref(self._h))
        if rc != HB_OK:
            raise HemeLBError(rc, self._error(None))
        n = C.c_int64()
        L.hb_site_count(self._h, C.byref(n))
        self.n = int(n.value)

    # -- housekeeping -----------------------------------------------------------
    def _error(self, h) -> str:
        buf = C.create_string_buffer(1024)
        library().hb_last_error(h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc: int) -> int:
        if rc == HB_OK:
            return rc
        if rc == HB_UNSTABLE:
            raise Unstable(rc, "the simulation became unstable (some f <= 0 or NaN)")
        raise HemeLBError(rc, self._error(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            library().hb_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- lb::LBM per-step phases -------------------------------------------------------
    def RequestComms(self) -> None:
        self._check(library().hb_request_comms(self._h))

    def PreSend(self) -> None:
        self._check(library().hb_pre_send(self._h))

    def PreReceive(self, macro: bool = False, stress: bool = False) -> None:
        self._check(library().hb_pre_receive(self._h, _flags(macro, stress)))

    def PostReceive(self) -> None:
        self._check(library().hb_post_receive(self._h))

    def EndIteration(self) -> None:
        self._check(library().hb_end_iteration(self._h))

    def step(self, n: int = 1, macro: bool = False, stress: bool = False) -> None:
        """`n` full time steps (all phases); `macro` fills the caches on the last,
        `stress` (with `macro`) the stress caches too."""
        self._check(library().hb_step(self._h, int(n), _flags(macro, stress)))

    # -- state ---------------------------------------------------------------------------
    @property
    def time_step(self) -> int:
        t = C.c_uint64()
        library().hb_time_step(self._h, C.byref(t))
        return int(t.value)

    @time_step.setter
    def time_step(self, t: int) -> None:
        self._check(library().hb_set_time_step(self._h, int(t)))

    def GetLbmParams(self) -> Params:
        p = Params()
        self._check(library().hb_get_params(self._h, C.byref(p)))
        return p

    def GetFOld(self) -> np.ndarray:
        """Distributions entering the next step, [n, 19] in reference order."""
        f = np.empty((self.n, 19), np.float64)
        self._check(library().hb_get_fs(self._h, _p(f)))
        return f

    def SetFs(self, f: np.ndarray) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.shape != (self.n, 19):
            raise ValueError(f"expected shape {(self.n, 19)}")
        self._check(library().hb_set_fs(self._h, _p(f)))

    def GetPropertyCache(self):
        """(density [n], velocity [n, 3], wall-shear-stress [n]) of the last macro step."""
        rho = np.empty(self.n)
        u = np.empty((self.n, 3))
        w = np.empty(self.n)
        self._check(library().hb_get_macro(self._h, _p(rho), _p(u), _p(w)))
        return rho, u, w

    def GetStress(self, field: str) -> np.ndarray:
        """Stress cache `field` of the last stress step in lattice units, [n, k] in
        reference order: "vonmisesstress", "shearrate" (k = 1), "stresstensor" (xx, xy,
        xz, yy, yz, zz), "traction", "tangentialprojectiontraction",
        "normalprojectiontraction" (k = 3, zero off the wall)."""
        idx, k = STRESS_FIELDS[field]
        out = np.empty((self.n, k))
        self._check(library().hb_get_stress(self._h, idx, _p(out)))
        return out

    def SetIoletDensities(self, inlets=None, outlets=None) -> None:
        """Densities (lattice units) of every inlet and outlet used by the cosine and
        file pressure iolets from the next step on, in place of the case's own
        (BoundaryValues::GetBoundaryDensity supplied by the caller); no arguments
        return to the case's values."""
        if inlets is None and outlets is None:
            self._check(library().hb_set_iolet_densities(self._h, None, 0, None, 0))
            return
        i = np.ascontiguousarray(inlets, dtype=np.float64)
        o = np.ascontiguousarray(outlets, dtype=np.float64)
        self._check(library().hb_set_iolet_densities(self._h, _p(i), len(i), _p(o), len(o)))

    def moment_sums(self) -> np.ndarray:
        """(total density, total momentum x, y, z) of the current distributions, FP64."""
        a = np.empty(4)
        self._check(library().hb_moment_sums(self._h, _p(a)))
        return a

    def GetWK3(self, group: int, index: int) -> np.ndarray:
        a = np.empty(4)
        self._check(library().hb_get_wk3(self._h, int(group), int(index), _p(a)))
        return a

    def read_timing(self) -> Dict[str, float]:
        """Wall-clock milliseconds of the open's phases."""
        ms = np.zeros(5)
        library().hb_geometry_read_timing(self._g, _p(ms))
        return dict(zip(("read", "inflate", "h2d", "device", "d2h"), ms.tolist()))

    def tables(self) -> Dict[str, np.ndarray]:
        n = self.n
        out = {"neighbours": np.empty((n, 19), np.int64), "wall_mask": np.empty(n, np.uint32),
               "iolet_mask": np.empty(n, np.uint32), "site_type": np.empty(n, np.int32),
               "iolet_id": np.empty(n, np.int32), "coords": np.empty((n, 3), np.int64),
               "type_counts": np.empty(6, np.int64)}
        self._check(library().hb_get_tables(self._h, *(_p(out[k]) for k in (
            "neighbours", "wall_mask", "iolet_mask", "site_type", "iolet_id", "coords", "type_counts"))))
        return out

    def WriteXtr(self, path: str, fields: Sequence[str], offset_path: Optional[str] = None,
                 geometry: Optional[Selector] = None) -> None:
        """Append one .xtr record (LocalPropertyOutput::Write) for the whole lattice,
        or for the sites `geometry` (see `selector`) takes."""
        off = os.fspath(offset_path).encode() if offset_path else None
        if geometry is None:
            self._check(library().hb_write_xtr(self._h, os.fspath(path).encode(), ",".join(fields).encode(), off))
        else:
            self._check(library().hb_write_xtr_selected(self._h, os.fspath(path).encode(), ",".join(fields).encode(),
                                                        off, C.byref(geometry)))

    def ReadCheckpoint(self, path: str, step: int = 0) -> None:
        self._check(library().hb_read_checkpoint(self._h, os.fspath(path).encode(), int(step)))

    def setup_timing(self) -> Dict[str, float]:
        """Wall-clock ms of the construction from a case file: case, geometry
        (decode, layout, tables back), solver (uploads, initial state), total."""
        ms = np.zeros(4)
        self._check(library().hb_setup_timing(self._h, _p(ms)))
        return {"case": float(ms[0]), "geometry": float(ms[1]), "solver": float(ms[2]), "total": float(ms[3])}

    def last_step_timing(self):
        ms = C.c_double()
        n = C.c_int64()
        library().hb_last_step_timing(self._h, C.byref(ms), C.byref(n))
        return float(ms.value), int(n.value)

    def WriteState(self, path) -> None:
        """Exact FP64 restart file (hb_write_state)."""
        self._check(library().hb_write_state(self._h, os.fspath(path).encode()))

    def ReadState(self, path) -> None:
        """Restore a run from hb_write_state's file: it continues bit for bit."""
        self._check(library().hb_read_state(self._h, os.fspath(path).encode()))

    # -- sharded form -------------------------------------------------------------------
    def shard_halo_sizes(self):
        """Stored elements (send lower, send upper, receive lower, receive upper)
        and the element size in bytes."""
        c = np.zeros(4, np.int64)
        e = C.c_int()
        self._check(library().hb_shard_halo_sizes(self._h, _p(c), C.byref(e)))
        return [int(v) for v in c], int(e.value)

    def shard_pack(self, to_lower, to_upper, stream: Optional[int] = None) -> None:
        """Device tensors (or raw device pointers) of the send buffers."""
        lo = to_lower if isinstance(to_lower, (int, type(None))) else _dptr(to_lower)
        hi = to_upper if isinstance(to_upper, (int, type(None))) else _dptr(to_upper)
        self._check(library().hb_shard_pack(self._h, lo, hi, stream))

    def shard_unpack(self, from_lower, from_upper, stream: Optional[int] = None) -> None:
        lo = from_lower if isinstance(from_lower, (int, type(None))) else _dptr(from_lower)
        hi = from_upper if isinstance(from_upper, (int, type(None))) else _dptr(from_upper)
        self._check(library().hb_shard_unpack(self._h, lo, hi, stream))

    def shard_site_ids(self) -> np.ndarray:
        ids = np.zeros(self.n, np.int64)
        self._check(library().hb_shard_site_ids(self._h, _p(ids)))
        return ids

    def profile_steps(self, n: int):
        """Advance 2n steps timing the launches: (step launch ms over the first n
        steps as `step` runs them, plain-bulk kernel ms and boundary kernel ms
        over the next n steps run one kernel after the other)."""
        ms = np.zeros(3)
        self._check(library().hb_profile_steps(self._h, int(n), _p(ms)))
        return float(ms[0]), float(ms[1]), float(ms[2])

    def device_bytes(self) -> int:
        b = C.c_int64()
        library().hb_device_bytes(self._h, C.byref(b))
        return int(b.value)


def last_create_error() -> str:
    buf = C.create_string_buffer(1024)
    library().hb_last_error(None, buf, 1024)
    return buf.value.decode(errors="replace")


def read_case(xml_path: str, kernel: str = "LBGK"):
    """(Params, gmy path) as the library's case reader sees them (no GPU needed)."""
    p = Params()
    buf = C.create_string_buffer(4096)
    rc = library().hb_read_case(os.fspath(xml_path).encode(), KERNELS[kernel], C.byref(p), buf, 4096)
    if rc != HB_OK:
        raise HemeLBError(rc, last_create_error())
    return p, buf.value.decode()


def read_case_iolet_table(xml_path: str, kernel: str, outlet: bool, index: int, count: int) -> np.ndarray:
    """The first `count` entries of a file iolet's table (no GPU needed): lattice
    densities of a file pressure iolet, peak speeds of a file velocity iolet."""
    out = np.zeros(int(count), np.float64)
    rc = library().hb_read_case_iolet_table(os.fspath(xml_path).encode(), KERNELS[kernel], 1 if outlet else 0,
                                            int(index), _p(out), int(count))
    if rc != HB_OK:
        raise HemeLBError(rc, last_create_error())
    return out


def iolet_velocity(iolet: Iolet, x, t: int) -> np.ndarray:
    """InOutLetVelocity::GetVelocity of a velocity iolet (parabolic, file velocity,
    Womersley) at lattice position `x` and 1-based step `t`, as the kernels impose
    it (no GPU needed).  A point outside a parabolic or file profile's radius raises
    HB_ERR_IOLET_RADIUS, as the reference exits there."""
    xv = np.ascontiguousarray(x, np.float64)
    v = np.zeros(3, np.float64)
    rc = library().hb_iolet_velocity(C.byref(iolet), _p(xv), int(t), _p(v))
    if rc != HB_OK:
        raise HemeLBError(rc, "iolet velocity")
    return v


class Geometry:
    """Reference-order lattice tables of a `.gmy`: read by the library's host code
    (no GPU needed), or with `device` set decoded, binned and linked on that GPU
    (the blocks inflated on host threads); the tables are the same bit for bit."""

    def __init__(self, gmy_path: str, device: Optional[int] = None):
        self._g = C.c_void_p()
        if device is None:
            rc = library().hb_geometry_open(os.fspath(gmy_path).encode(), C.byref(self._g))
        else:
            rc = library().hb_geometry_open_device(os.fspath(gmy_path).encode(), int(device), C.byref(self._g))
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())
        n = C.c_int64()
        dims = np.zeros(3, np.int64)
        library().hb_geometry_site_count(self._g, C.byref(n), _p(dims))
        self.n = int(n.value)
        self.dims = dims

    def read_timing(self) -> Dict[str, float]:
        """Wall-clock milliseconds of the open's phases."""
        ms = np.zeros(5)
        library().hb_geometry_read_timing(self._g, _p(ms))
        return dict(zip(("read", "inflate", "h2d", "device", "d2h"), ms.tolist()))

    def tables(self) -> Dict[str, np.ndarray]:
        n = self.n
        out = {"neighbours": np.empty((n, 19), np.int64), "wall_mask": np.empty(n, np.uint32),
               "iolet_mask": np.empty(n, np.uint32), "site_type": np.empty(n, np.int32),
               "iolet_id": np.empty(n, np.int32), "coords": np.empty((n, 3), np.int64),
               "type_counts": np.empty(6, np.int64), "wall_distance": np.empty((n, 18)),
               "wall_normal": np.empty((n, 3))}
        rc = library().hb_geometry_tables(self._g, *(_p(out[k]) for k in (
            "neighbours", "wall_mask", "iolet_mask", "site_type", "iolet_id", "coords", "type_counts",
            "wall_distance", "wall_normal")))
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())
        out["dims"] = self.dims.copy()
        return out

    def select(self, geometry: Selector, voxel_size: float, origin=(0.0, 0.0, 0.0)) -> np.ndarray:
        """Mask (contiguous order) of the sites a geometry selector takes."""
        n = C.c_int64()
        dims = (C.c_int64 * 3)()
        library().hb_geometry_site_count(self._g, C.byref(n), dims)
        mask = np.zeros(n.value, np.uint8)
        org = np.asarray(origin, dtype=np.float64)
        rc = library().hb_geometry_select(self._g, C.byref(geometry), float(voxel_size), _p(org), _p(mask))
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())
        return mask.astype(bool)

    def layout(self, params: Params, wall: str = "SBB") -> Dict[str, int]:
        st = np.zeros(4, np.int64)
        rc = library().hb_geometry_layout(self._g, C.byref(params), WALLS[wall], _p(st))
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())
        return {"axis": int(st[0]), "runs": int(st[1]), "bulk_sites": int(st[2]), "general_sites": int(st[3])}

    def layout_digest(self, params: Params, wall: str = "SBB", device: int = -1) -> np.ndarray:
        """Digests of every array of the storage layout, built on the host
        (device < 0) or on that GPU; the two builds agree bit for bit."""
        out = np.zeros(32, np.uint64)
        rc = library().hb_geometry_layout_digest(self._g, C.byref(params), WALLS[wall], int(device), _p(out))
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())
        return out

    def close(self):
        if getattr(self, "_g", None) and self._g.value:
            library().hb_geometry_close(self._g)
            self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PreparedLattice:
    """A case parsed, its geometry read and its storage layout built on the
    host, ready for Batch.add_prepared.  Preparation needs no device and releases
    the interpreter lock, so it runs on worker threads while blocks step.  With
    `device`, the geometry is decoded and laid out on that GPU instead (same
    result; it synchronises the device)."""

    def __init__(self, xml_path: str, kernel: str = "LBGK", wall: str = "SBB", steps: int = 1000,
                 device: Optional[int] = None):
        self._h = C.c_void_p()
        if device is None:
            rc = library().hb_batch_prepare_xml(os.fspath(xml_path).encode(), KERNELS[kernel], WALLS[wall], int(steps),
                                                C.byref(self._h))
        else:
            rc = library().hb_batch_prepare_xml_device(os.fspath(xml_path).encode(), KERNELS[kernel], WALLS[wall],
                                                       int(steps), int(device), C.byref(self._h))
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())
        n = C.c_int64()
        library().hb_batch_prep_sites(self._h, C.byref(n))
        self.sites = int(n.value)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().hb_batch_prep_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many lattices resident on one GPU, stepped together (the batched form)."""

    def __init__(self, site_capacity: int, general_capacity: int, max_lattices: int = 64,
                 precision: str = "fp32", device: int = 0):
        self._b = C.c_void_p()
        rc = library().hb_batch_create(int(site_capacity), int(general_capacity), int(max_lattices),
                                       PRECISIONS[precision], int(device), C.byref(self._b))
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())
        self.max_lattices = int(max_lattices)

    @staticmethod
    def bytes_for(site_capacity: int, general_capacity: int, max_lattices: int = 64, precision: str = "fp32") -> int:
        b = C.c_int64()
        library().hb_batch_bytes(int(site_capacity), int(general_capacity), int(max_lattices), PRECISIONS[precision],
                                 C.byref(b))
        return int(b.value)

    def _check(self, rc):
        if rc != HB_OK:
            raise HemeLBError(rc, last_create_error())

    def add_xml(self, xml_path: str, kernel: str = "LBGK", wall: str = "SBB", steps: int = 1000) -> int:
        slot = C.c_int()
        self._check(library().hb_batch_add_xml(self._b, os.fspath(xml_path).encode(), KERNELS[kernel], WALLS[wall],
                                               int(steps), C.byref(slot)))
        return int(slot.value)

    def add_prepared(self, prep: "PreparedLattice") -> int:
        """Admit a prepared lattice (uploads only).  Raises HemeLBError with code
        -5 when it does not fit yet; the prepared lattice then stays usable."""
        slot = C.c_int()
        self._check(library().hb_batch_add_prepared(self._b, prep._h, C.byref(slot)))
        return int(slot.value)

    def remove(self, slot: int) -> None:
        self._check(library().hb_batch_remove(self._b, int(slot)))

    def run(self, k: int):
        """Run k steps; returns the slots that finished in this block: reached
        their step count, or went unstable (check `info`; then no fields)."""
        buf = (C.c_int * self.max_lattices)()
        n = C.c_int()
        self._check(library().hb_batch_run(self._b, int(k), buf, self.max_lattices, C.byref(n)))
        return [int(buf[i]) for i in range(n.value)]

    def macro(self, slot: int):
        n, _, _ = self.info(slot)
        rho, u, w = np.empty(n), np.empty((n, 3)), np.empty(n)
        self._check(library().hb_batch_get_macro(self._b, int(slot), _p(rho), _p(u), _p(w)))
        return rho, u, w

    def info(self, slot: int):
        n, t, st = C.c_int64(), C.c_uint64(), C.c_int()
        self._check(library().hb_batch_member_info(self._b, int(slot), C.byref(n), C.byref(t), C.byref(st)))
        return int(n.value), int(t.value), int(st.value)

    def set_tuning(self, sites_per_thread: int, block: int, form: str = "persistent") -> None:
        """Launch shape of the step: sites per thread, threads per block, and the
        form ("persistent": one kernel interleaving bulk and boundary tiles;
        "split": the same tiles as two kernels side by side)."""
        self._check(library().hb_batch_set_tuning(self._b, int(sites_per_thread), int(block)))
        self._check(library().hb_batch_set_step_form(self._b, BATCH_FORMS[form]))

    def stats(self):
        ms, act, by = C.c_double(), C.c_int64(), C.c_int64()
        library().hb_batch_stats(self._b, C.byref(ms), C.byref(act), C.byref(by))
        return float(ms.value), int(act.value), int(by.value)

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            library().hb_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
