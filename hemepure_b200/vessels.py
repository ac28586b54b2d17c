"""Synthetic vessel voxeliser: writes HemeLB `.gmy` v4 geometry and XML v3 case files.

The reference ships no generator for the benchmark geometries (its Benchmarking
`.gmy` files are absent), so this module produces seeded synthetic lattices:
straight pipes, axisymmetric cosine stenoses and symmetric Y-bifurcations.  The
same files feed the CPU oracle and the GPU solver.

File format (all XDR big-endian), as read by the reference
(`src/geometry/GeometryReader.cc:382-444,515-607,800-946`,
`src/io/formats/geometry.h:48-148`, `src/io/formats/geometry.cc:15-53`):

* preamble, 32 bytes: magic 0x686c6221, 0x676d7904, version 4, blocks x/y/z,
  block size, padding 0;
* header, 12 bytes per block in (bx*By + by)*Bz + bz order: fluid sites,
  compressed bytes, uncompressed bytes;
* one zlib stream per non-empty block; sites in (x*bs + y)*bs + z order; a solid
  site is the word 0; a fluid site is the word 1, then 26 links in the
  displacement order below (cut type, then a float distance for a wall, or an
  iolet id and a float distance for an iolet), then the wall-normal flag and,
  when set, three floats.

Link distances are the fraction of the link vector at which the segment from
the site to its neighbour leaves the fluid domain, in (0, 1].
"""

from __future__ import annotations

import math
import os
import zlib
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# Displacement order of the 26 links in a .gmy site record
# (src/io/formats/geometry.cc:16-52): x-major, then y, then z, skipping (0,0,0).
GMY_DISPLACEMENTS = np.array(
    [(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
     if (dx, dy, dz) != (0, 0, 0)], dtype=np.int64)

CUT_NONE, CUT_WALL, CUT_INLET, CUT_OUTLET = 0, 1, 2, 3

# Physical constants used by the reference's unit conversion (src/constants.h).
MMHG_TO_PASCAL = 133.3223874
BLOOD_DENSITY = 1000.0
BLOOD_VISCOSITY = 0.004
CS2 = 1.0 / 3.0


@dataclass
class Iolet:
    """A planar inlet or outlet: a disc of `radius` centred on `position`.

    `normal` points into the fluid, as in the reference's case files."""
    kind: str                 # "inlet" or "outlet"
    position: np.ndarray      # lattice units
    normal: np.ndarray        # unit vector, into the fluid
    radius: float             # lattice units


class Vessel:
    """Implicit vessel: `level(p) < 0` inside the lumen; iolet planes clip it."""

    iolets: List[Iolet]
    bbox_lo: np.ndarray
    bbox_hi: np.ndarray

    def level(self, x, y, z):
        raise NotImplementedError

    def normal(self, x, y, z):
        """Outward unit normal of the lumen surface nearest to each point."""
        raise NotImplementedError

    def wall_exit(self, p, c, t_hi):
        """Fraction t in (0, t_hi] where p + t c leaves the lumen (bisection on level)."""
        lo = np.zeros(len(p))
        hi = np.array(t_hi, dtype=np.float64)
        for _ in range(48):
            mid = 0.5 * (lo + hi)
            q = p + mid[:, None] * c
            inside = self.level(q[:, 0], q[:, 1], q[:, 2]) < 0.0
            lo = np.where(inside, mid, lo)
            hi = np.where(inside, hi, mid)
        return hi

    def inside(self, x, y, z):
        ok = self.level(x, y, z) < 0.0
        for io in self.iolets:
            ok &= ((x - io.position[0]) * io.normal[0] + (y - io.position[1]) * io.normal[1]
                   + (z - io.position[2]) * io.normal[2]) > 0.0
        return ok


class Pipe(Vessel):
    """Straight rigid pipe of `radius` along z with `length` fluid slices."""

    def __init__(self, radius: float, length: int, margin: int = 2):
        self.radius = float(radius)
        self.length = int(length)
        half = int(math.ceil(radius)) + margin
        # Axis on a half-integer so the voxelisation has the lattice's mirror symmetry.
        self.cx = self.cy = half + 0.5
        self.z0 = margin + 1
        self.bbox_lo = np.array([0, 0, 0])
        self.bbox_hi = np.array([2 * half + 1, 2 * half + 1, self.z0 + self.length + margin + 1])
        zin = self.z0 - 0.5
        zout = self.z0 + self.length - 0.5
        self.iolets = [
            Iolet("inlet", np.array([self.cx, self.cy, zin]), np.array([0.0, 0.0, 1.0]), self.radius),
            Iolet("outlet", np.array([self.cx, self.cy, zout]), np.array([0.0, 0.0, -1.0]), self.radius),
        ]

    def radius_at(self, z):
        return np.full_like(np.asarray(z, dtype=np.float64), self.radius)

    def level(self, x, y, z):
        r = self.radius_at(z)
        return (x - self.cx) ** 2 + (y - self.cy) ** 2 - r * r

    def normal(self, x, y, z):
        dx, dy = x - self.cx, y - self.cy
        n = np.stack([dx, dy, np.zeros_like(dx)], axis=1)
        return n / np.linalg.norm(n, axis=1, keepdims=True)

    def wall_exit(self, p, c, t_hi):
        # Analytic exit of a straight line from the cylinder: larger root of
        # |p_xy + t c_xy - centre|^2 = R^2.
        px, py = p[:, 0] - self.cx, p[:, 1] - self.cy
        a = c[:, 0] ** 2 + c[:, 1] ** 2
        b = 2.0 * (px * c[:, 0] + py * c[:, 1])
        cc = px * px + py * py - self.radius ** 2
        disc = np.maximum(b * b - 4.0 * a * cc, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (-b + np.sqrt(disc)) / (2.0 * a)
        return np.where(a > 0, np.minimum(t, t_hi), t_hi)


class Stenosis(Pipe):
    """Pipe of radius r0 whose radius dips to r_min at mid-length following a
    raised cosine over `span` slices (axisymmetric stenosis)."""

    def __init__(self, radius: float, length: int, r_min: float, span: float, margin: int = 2):
        super().__init__(radius, length, margin)
        self.r_min = float(r_min)
        self.span = float(span)
        self.zc = self.z0 + 0.5 * (self.length - 1)

    def radius_at(self, z):
        z = np.asarray(z, dtype=np.float64)
        s = (z - self.zc) / self.span
        dip = 0.5 * (self.radius - self.r_min) * (1.0 + np.cos(2.0 * np.pi * s))
        return np.where(np.abs(s) < 0.5, self.radius - dip, self.radius)

    def normal(self, x, y, z):
        dx, dy = x - self.cx, y - self.cy
        r = np.sqrt(dx * dx + dy * dy)
        s = (z - self.zc) / self.span
        drdz = np.where(np.abs(s) < 0.5,
                        -0.5 * (self.radius - self.r_min) * np.sin(2.0 * np.pi * s) * 2.0 * np.pi / self.span, 0.0)
        n = np.stack([dx / r, dy / r, -drdz], axis=1)
        return n / np.linalg.norm(n, axis=1, keepdims=True)

    def wall_exit(self, p, c, t_hi):
        return Vessel.wall_exit(self, p, c, t_hi)


class YBifurcation(Vessel):
    """Symmetric Y-bifurcation: a parent tube along +z splits at the junction into
    two daughters at +-angle in the x-z plane.  The lumen is the union of the
    three capsules (tube segments with rounded ends)."""

    def __init__(self, r_parent: float, l_parent: float, r_daughter: float, l_daughter: float,
                 angle_deg: float = 35.0, margin: int = 2):
        self.rp, self.lp, self.rd, self.ld = map(float, (r_parent, l_parent, r_daughter, l_daughter))
        a = math.radians(angle_deg)
        d1 = np.array([math.sin(a), 0.0, math.cos(a)])
        d2 = np.array([-math.sin(a), 0.0, math.cos(a)])
        # Extents: parent from z=0 to lp, daughters from the junction.
        half_x = self.ld * math.sin(a) + self.rd / math.cos(a) + margin + 1
        half_y = max(self.rp, self.rd) + margin + 1
        cx = math.ceil(half_x) + 0.5
        cy = math.ceil(half_y) + 0.5
        z0 = margin + 1
        self.p0 = np.array([cx, cy, z0 - 0.5])
        self.j = self.p0 + np.array([0.0, 0.0, self.lp])
        self.e1 = self.j + self.ld * d1
        self.e2 = self.j + self.ld * d2
        self.segs = [(self.p0 - np.array([0, 0, self.rp]), self.j, self.rp),
                     (self.j, self.e1 + self.rd * d1, self.rd),
                     (self.j, self.e2 + self.rd * d2, self.rd)]
        zmax = max(self.e1[2], self.e2[2]) + self.rd * math.sin(a) + margin + 2
        self.bbox_lo = np.array([0, 0, 0])
        self.bbox_hi = np.array([int(2 * cx) + 1, int(2 * cy) + 1, int(math.ceil(zmax))])
        self.iolets = [
            Iolet("inlet", self.p0.copy(), np.array([0.0, 0.0, 1.0]), self.rp),
            Iolet("outlet", self.e1.copy(), -d1, self.rd),
            Iolet("outlet", self.e2.copy(), -d2, self.rd),
        ]

    @staticmethod
    def _seg_dist(x, y, z, a, b):
        ab = b - a
        px, py, pz = x - a[0], y - a[1], z - a[2]
        t = np.clip((px * ab[0] + py * ab[1] + pz * ab[2]) / float(ab @ ab), 0.0, 1.0)
        qx, qy, qz = px - t * ab[0], py - t * ab[1], pz - t * ab[2]
        return np.sqrt(qx * qx + qy * qy + qz * qz), (qx, qy, qz)

    def level(self, x, y, z):
        out = None
        for a, b, r in self.segs:
            d, _ = self._seg_dist(x, y, z, a, b)
            v = d - r
            out = v if out is None else np.minimum(out, v)
        return out

    def normal(self, x, y, z):
        best = None
        vecs = None
        for a, b, r in self.segs:
            d, (qx, qy, qz) = self._seg_dist(x, y, z, a, b)
            v = d - r
            q = np.stack([qx, qy, qz], axis=1)
            if best is None:
                best, vecs = v, q
            else:
                sel = v < best
                best = np.where(sel, v, best)
                vecs = np.where(sel[:, None], q, vecs)
        return vecs / np.linalg.norm(vecs, axis=1, keepdims=True)


@dataclass
class GeometryInfo:
    path: str
    blocks: Tuple[int, int, int]
    block_size: int
    fluid_sites: int
    wall_sites: int
    iolet_ids: List[Tuple[str, int]] = field(default_factory=list)


def voxelise(vessel: Vessel, path: str, block_size: int = 8, chunk_blocks: int = 2048) -> GeometryInfo:
    """Write `vessel` as a `.gmy` v4 file; returns counts for cross-checks."""
    hi = vessel.bbox_hi
    nb = [int(math.ceil(float(hi[d]) / block_size)) for d in range(3)]
    dims = [nb[d] * block_size for d in range(3)]
    xs = np.arange(dims[0], dtype=np.float64)
    ys = np.arange(dims[1], dtype=np.float64)
    zs = np.arange(dims[2], dtype=np.float64)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    fluid = vessel.inside(X, Y, Z)
    # The outermost layer must stay solid so every neighbour lookup is in range.
    fluid[0, :, :] = fluid[-1, :, :] = False
    fluid[:, 0, :] = fluid[:, -1, :] = False
    fluid[:, :, 0] = fluid[:, :, -1] = False
    del X, Y, Z

    # Per-iolet id within its kind (inlets and outlets are numbered separately).
    kinds = []
    counters = {"inlet": 0, "outlet": 0}
    for io in vessel.iolets:
        kinds.append((io.kind, counters[io.kind]))
        counters[io.kind] += 1

    bs = block_size
    blocks_total = nb[0] * nb[1] * nb[2]
    # Reorder the grid into block-major, then in-block site order.
    order = fluid.reshape(nb[0], bs, nb[1], bs, nb[2], bs).transpose(0, 2, 4, 1, 3, 5).reshape(-1)
    # Global coordinates of every site in that order.
    bi = np.arange(blocks_total)
    bxs, bys, bzs = bi // (nb[1] * nb[2]), (bi // nb[2]) % nb[1], bi % nb[2]
    li = np.arange(bs ** 3)
    lx, ly, lz = li // (bs * bs), (li // bs) % bs, li % bs

    headers = np.zeros((blocks_total, 3), dtype=np.uint32)
    bodies = []
    total_fluid = 0
    total_wall = 0
    for b0 in range(0, blocks_total, chunk_blocks):
        b1 = min(blocks_total, b0 + chunk_blocks)
        nbk = b1 - b0
        fl = order[b0 * bs ** 3: b1 * bs ** 3]
        gx = (bxs[b0:b1, None] * bs + lx[None, :]).reshape(-1)
        gy = (bys[b0:b1, None] * bs + ly[None, :]).reshape(-1)
        gz = (bzs[b0:b1, None] * bs + lz[None, :]).reshape(-1)
        fidx = np.nonzero(fl)[0]
        nf = len(fidx)
        if nf == 0:
            continue  # every block of this chunk is solid: empty headers, no bodies
        # Word layout per fluid site: 1 + 26*3 + 1 + 3 = 83 slots, masked.
        words = np.zeros((nf, 83), dtype=np.uint32)
        valid = np.zeros((nf, 83), dtype=bool)
        words[:, 0] = 1
        valid[:, 0] = True
        px, py, pz = gx[fidx], gy[fidx], gz[fidx]
        is_wall = np.zeros(nf, dtype=bool)
        for k, (dx, dy, dz) in enumerate(GMY_DISPLACEMENTS):
            qx, qy, qz = px + dx, py + dy, pz + dz
            nfluid = fluid[qx, qy, qz]
            cut = ~nfluid
            base = 1 + 3 * k
            valid[:, base] = True
            ci = np.nonzero(cut)[0]
            if len(ci) == 0:
                continue
            p = np.stack([px[ci], py[ci], pz[ci]], axis=1).astype(np.float64)
            c = np.tile(np.array([dx, dy, dz], dtype=np.float64), (len(ci), 1))
            t_best = np.full(len(ci), np.inf)
            typ = np.zeros(len(ci), dtype=np.uint32)
            iid = np.zeros(len(ci), dtype=np.uint32)
            # Iolet planes crossed from the fluid side.
            for (kind, kid), io in zip(kinds, vessel.iolets):
                s0 = (p - io.position) @ io.normal
                s1 = s0 + c @ io.normal
                crosses = (s0 > 0) & (s1 <= 0)
                with np.errstate(divide="ignore", invalid="ignore"):
                    t = np.where(crosses, s0 / (s0 - s1), np.inf)
                better = t < t_best
                t_best = np.where(better, t, t_best)
                typ = np.where(better, CUT_INLET if kind == "inlet" else CUT_OUTLET, typ)
                iid = np.where(better, kid, iid)
            q = p + c
            lumen_exit = vessel.level(q[:, 0], q[:, 1], q[:, 2]) >= 0.0
            tw = np.full(len(ci), np.inf)
            if lumen_exit.any():
                sel = np.nonzero(lumen_exit)[0]
                tw[sel] = vessel.wall_exit(p[sel], c[sel], np.ones(len(sel)))
            wall_first = tw < t_best
            t_best = np.where(wall_first, tw, t_best)
            typ = np.where(wall_first, CUT_WALL, typ)
            if not np.all(np.isfinite(t_best)):
                raise RuntimeError("voxeliser: a cut link found no crossing")
            t32 = np.clip(t_best, 1e-6, 1.0).astype(np.float32)
            words[ci, base] = typ
            is_w = typ == CUT_WALL
            # wall: distance; iolet: id then distance
            words[ci, base + 1] = np.where(is_w, t32.view(np.uint32), iid)
            words[ci, base + 2] = np.where(is_w, 0, t32.view(np.uint32))
            valid[ci, base + 1] = True
            valid[ci, base + 2] = ~is_w
            is_wall[ci[is_w]] = True
        words[:, 79] = is_wall.astype(np.uint32)
        valid[:, 79] = True
        wi = np.nonzero(is_wall)[0]
        if len(wi):
            n = vessel.normal(px[wi].astype(np.float64), py[wi].astype(np.float64), pz[wi].astype(np.float64))
            n32 = n.astype(np.float32)
            words[wi, 80:83] = n32.view(np.uint32)
            valid[wi, 80:83] = True
        total_fluid += nf
        total_wall += int(is_wall.sum())
        # Assemble every block's word stream: solid sites are the single word 0.
        site_words = np.ones(len(fl), dtype=np.int64)
        site_words[fidx] = valid.sum(axis=1)
        stream = np.zeros(int(site_words.sum()), dtype=np.uint32)
        starts = np.concatenate([[0], np.cumsum(site_words)[:-1]])
        flat_words = words[valid]  # row-major: per site in order
        row_counts = valid.sum(axis=1)
        dest = np.repeat(starts[fidx], row_counts) + (np.arange(len(flat_words))
                                                        - np.repeat(np.concatenate([[0], np.cumsum(row_counts)[:-1]]), row_counts))
        stream[dest] = flat_words
        be = stream.astype(">u4").tobytes()
        block_word_ends = np.cumsum(site_words.reshape(nbk, bs ** 3).sum(axis=1))
        block_word_starts = np.concatenate([[0], block_word_ends[:-1]])
        fl_blocks = fl.reshape(nbk, bs ** 3).sum(axis=1)
        for j in range(nbk):
            nfl = int(fl_blocks[j])
            if nfl == 0:
                continue
            raw = be[4 * int(block_word_starts[j]):4 * int(block_word_ends[j])]
            comp = zlib.compress(raw, 6)
            headers[b0 + j] = (nfl, len(comp), len(raw))
            bodies.append(comp)

    with open(path, "wb") as fh:
        pre = np.array([0x686C6221, 0x676D7904, 4, nb[0], nb[1], nb[2], bs, 0], dtype=">u4")
        fh.write(pre.tobytes())
        fh.write(headers.astype(">u4").tobytes())
        for b in bodies:
            fh.write(b)
    return GeometryInfo(path=path, blocks=tuple(nb), block_size=bs, fluid_sites=total_fluid,
                        wall_sites=total_wall, iolet_ids=kinds)


# ---------------------------------------------------------------------------
# XML v3 case files
# ---------------------------------------------------------------------------

@dataclass
class CaseUnits:
    """Physical scales chosen so that the derived relaxation time hits `tau`.

    The reference derives tau = 0.5 + dt*(mu/rho)/(cs^2 dx^2)
    (`src/lb/LbmParameters.h:29-37`)."""
    tau: float
    voxel: float = 1e-4

    @property
    def dt(self) -> float:
        return (self.tau - 0.5) * CS2 * self.voxel * self.voxel / (BLOOD_VISCOSITY / BLOOD_DENSITY)

    @property
    def lattice_pressure(self) -> float:
        mass = BLOOD_DENSITY * self.voxel ** 3
        return mass / (self.voxel * self.dt * self.dt)

    def density_to_mmHg(self, rho: float) -> float:
        # inverse of ConvertPressureToLatticeUnits(p)/Cs2 (src/util/UnitConverter.cc:26-40)
        return (rho - 1.0) * CS2 * self.lattice_pressure / MMHG_TO_PASCAL

    def density_amp_to_mmHg(self, amp: float) -> float:
        return amp * CS2 * self.lattice_pressure / MMHG_TO_PASCAL

    def speed_to_phys(self, u: float) -> float:
        return u * self.voxel / self.dt


def _vec(v: Sequence[float]) -> str:
    return "(" + ",".join(repr(float(a)) for a in v) + ")"


@dataclass
class PressureBC:
    mean_rho: float
    amp_rho: float = 0.0
    period_steps: float = 1.0e9
    phase: float = 0.0


@dataclass
class VelocityBC:
    u_max: float                       # lattice units
    radius: Optional[float] = None     # lattice units; default: the iolet's radius


@dataclass
class WK3BC:
    r_c: float      # lattice units
    r_p: float
    c_p: float
    area: float     # lattice units
    radius: Optional[float] = None


@dataclass
class WK2BC:
    r: float        # lattice units
    c: float
    area: float     # lattice units
    radius: Optional[float] = None


@dataclass
class FilePressureBC:
    path: str       # (time in s, pressure in mmHg) pairs, one per line; relative to the case file


@dataclass
class FileWKBC:
    """InOutLetFileWK: a two-element Windkessel with a weights-file path."""
    path: str
    r: float        # lattice units
    c: float
    area: float     # lattice units


@dataclass
class FileVelocityBC:
    """InOutLetFileVelocity: the parabolic profile with a peak speed read from a
    file of (time in s, speed in m/s) pairs; relative to the case file."""
    path: str
    radius: Optional[float] = None     # lattice units; default: the iolet's radius


@dataclass
class WomersleyBC:
    """InOutLetWomersleyVelocity, in lattice units: pressure-gradient amplitude,
    period in steps, Womersley number."""
    pressure_gradient: float
    period_steps: float
    womersley_number: float
    radius: Optional[float] = None


def write_case_xml(path: str, gmy_name: str, vessel: Vessel, units: CaseUnits, steps: int,
                   inlet_bcs: Sequence, outlet_bcs: Sequence, warmup: int = 0,
                   relaxation_parameter: Optional[float] = None, sponge: Optional[dict] = None,
                   properties: Optional[List[dict]] = None, initial_rho: float = 1.0) -> None:
    """Write a HemeLB XML v3 case (`src/configuration/SimConfig.cc:84-121`)."""
    L = []
    L.append('<?xml version="1.0"?>')
    L.append('<hemelbsettings version="3">')
    L.append('  <simulation>')
    L.append(f'    <step_length units="s" value="{units.dt!r}"/>')
    L.append(f'    <steps units="lattice" value="{int(steps)}"/>')
    if warmup:
        L.append(f'    <extra_warmup_steps units="lattice" value="{int(warmup)}"/>')
    L.append('    <stresstype value="1"/>')
    if relaxation_parameter is not None:
        L.append(f'    <relaxation_parameter units="lattice" value="{float(relaxation_parameter)!r}"/>')
    L.append(f'    <voxel_size units="m" value="{units.voxel!r}"/>')
    L.append('    <origin units="m" value="(0.0,0.0,0.0)"/>')
    L.append('  </simulation>')
    L.append('  <geometry>')
    L.append(f'    <datafile path="{gmy_name}"/>')
    L.append('  </geometry>')
    L.append('  <initialconditions>')
    L.append('    <pressure>')
    L.append(f'      <uniform units="mmHg" value="{units.density_to_mmHg(initial_rho)!r}"/>')
    L.append('    </pressure>')
    if sponge is not None:
        L.append('    <sponge_layer>')
        L.append(f'      <viscosity_ratio units="dimensionless" value="{float(sponge["viscosity_ratio"])!r}"/>')
        L.append(f'      <width units="m" value="{float(sponge["width"]) * units.voxel!r}"/>')
        L.append(f'      <lifetime units="lattice" value="{int(sponge["lifetime"])}"/>')
        L.append('    </sponge_layer>')
    L.append('  </initialconditions>')
    for group, bcs in (("inlets", inlet_bcs), ("outlets", outlet_bcs)):
        kind = group[:-1]
        L.append(f'  <{group}>')
        ios = [io for io in vessel.iolets if io.kind == kind]
        if len(ios) != len(bcs):
            raise ValueError(f"{group}: {len(ios)} iolets but {len(bcs)} conditions")
        for io, bc in zip(ios, bcs):
            L.append(f'    <{kind}>')
            if isinstance(bc, PressureBC):
                L.append('      <condition subtype="cosine" type="pressure">')
                L.append(f'        <amplitude units="mmHg" value="{units.density_amp_to_mmHg(bc.amp_rho)!r}"/>')
                L.append(f'        <mean units="mmHg" value="{units.density_to_mmHg(bc.mean_rho)!r}"/>')
                L.append(f'        <phase units="rad" value="{float(bc.phase)!r}"/>')
                L.append(f'        <period units="s" value="{float(bc.period_steps) * units.dt!r}"/>')
                L.append('      </condition>')
            elif isinstance(bc, VelocityBC):
                r = io.radius if bc.radius is None else bc.radius
                L.append('      <condition subtype="parabolic" type="velocity">')
                L.append(f'        <radius units="m" value="{float(r) * units.voxel!r}"/>')
                L.append(f'        <maximum units="m/s" value="{units.speed_to_phys(bc.u_max)!r}"/>')
                L.append('      </condition>')
            elif isinstance(bc, WK3BC):
                r = io.radius if bc.radius is None else bc.radius
                res = (units.dt * units.voxel) / BLOOD_DENSITY
                cap = BLOOD_DENSITY / (units.dt * units.dt * units.voxel)
                L.append('      <condition subtype="WK3" type="pressure">')
                L.append(f'        <Rc units="kg/m^4*s" value="{bc.r_c / res!r}"/>')
                L.append(f'        <Rp units="kg/m^4*s" value="{bc.r_p / res!r}"/>')
                L.append(f'        <Cp units="m^4*s^2/kg" value="{bc.c_p / cap!r}"/>')
                L.append(f'        <radius units="m" value="{float(r) * units.voxel!r}"/>')
                L.append(f'        <area units="m^2" value="{bc.area * units.voxel * units.voxel!r}"/>')
                L.append('      </condition>')
            elif isinstance(bc, WK2BC):
                r = io.radius if bc.radius is None else bc.radius
                res = (units.dt * units.voxel) / BLOOD_DENSITY
                cap = BLOOD_DENSITY / (units.dt * units.dt * units.voxel)
                L.append('      <condition subtype="WK2" type="pressure">')
                L.append(f'        <R units="kg/m^4*s" value="{bc.r / res!r}"/>')
                L.append(f'        <C units="m^4*s^2/kg" value="{bc.c / cap!r}"/>')
                L.append(f'        <radius units="m" value="{float(r) * units.voxel!r}"/>')
                L.append(f'        <area units="m^2" value="{bc.area * units.voxel * units.voxel!r}"/>')
                L.append('      </condition>')
            elif isinstance(bc, FilePressureBC):
                L.append('      <condition subtype="file" type="pressure">')
                L.append(f'        <path value="{bc.path}"/>')
                L.append('      </condition>')
            elif isinstance(bc, FileWKBC):
                res = (units.dt * units.voxel) / BLOOD_DENSITY
                cap = BLOOD_DENSITY / (units.dt * units.dt * units.voxel)
                L.append('      <condition subtype="fileWK" type="pressure">')
                L.append(f'        <path value="{bc.path}"/>')
                L.append(f'        <R units="kg/m^4*s" value="{bc.r / res!r}"/>')
                L.append(f'        <C units="m^4*s^2/kg" value="{bc.c / cap!r}"/>')
                L.append(f'        <area units="m^2" value="{bc.area * units.voxel * units.voxel!r}"/>')
                L.append('      </condition>')
            elif isinstance(bc, FileVelocityBC):
                r = io.radius if bc.radius is None else bc.radius
                L.append('      <condition subtype="file" type="velocity">')
                L.append(f'        <path value="{bc.path}"/>')
                L.append(f'        <radius units="m" value="{float(r) * units.voxel!r}"/>')
                L.append('      </condition>')
            elif isinstance(bc, WomersleyBC):
                r = io.radius if bc.radius is None else bc.radius
                # mmHg/m -> lattice: divide by mass / (dx^2 dt^2) / mmHg_to_Pa.
                grad_unit = BLOOD_DENSITY * units.voxel ** 3 / (units.voxel ** 2 * units.dt ** 2) / MMHG_TO_PASCAL
                L.append('      <condition subtype="womersley" type="velocity">')
                L.append(f'        <pressure_gradient_amplitude units="mmHg/m" value="{bc.pressure_gradient * grad_unit!r}"/>')
                L.append(f'        <period units="s" value="{float(bc.period_steps) * units.dt!r}"/>')
                L.append(f'        <womersley_number units="dimensionless" value="{float(bc.womersley_number)!r}"/>')
                L.append(f'        <radius units="m" value="{float(r) * units.voxel!r}"/>')
                L.append('      </condition>')
            else:
                raise TypeError(bc)
            L.append(f'      <normal units="dimensionless" value="{_vec(io.normal)}"/>')
            L.append(f'      <position units="lattice" value="{_vec(io.position)}"/>')
            L.append(f'    </{kind}>')
        L.append(f'  </{group}>')
    if properties:
        L.append('  <properties>')
        for po in properties:
            L.append(f'    <propertyoutput file="{po["file"]}" period="{int(po["period"])}">')
            geo = po.get("geometry", "whole")
            if isinstance(geo, str):
                L.append(f'      <geometry type="{geo}" />')
            else:  # {"type": ..., "point": (m), "point2": (m), "normal": ..., "radius": m}
                L.append(f'      <geometry type="{geo["type"]}">')
                for key in ("point", "point2"):
                    if key in geo:
                        L.append(f'        <point units="m" value="{_vec(geo[key])}"/>')
                if "normal" in geo:
                    L.append(f'        <normal units="dimensionless" value="{_vec(geo["normal"])}"/>')
                if "radius" in geo:
                    L.append(f'        <radius units="m" value="{float(geo["radius"])!r}"/>')
                L.append('      </geometry>')
            for fld in po["fields"]:
                # "type" or "type:name"
                kind, _, name = fld.partition(":")
                L.append(f'      <field type="{kind}" name="{name}" />' if name else f'      <field type="{kind}" />')
            L.append('    </propertyoutput>')
        L.append('  </properties>')
    L.append('</hemelbsettings>')
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


# ---------------------------------------------------------------------------
# The workloads: five named vessel configurations
# ---------------------------------------------------------------------------

def make_case(name: str, out_dir: str, steps: Optional[int] = None, scale: float = 1.0,
              seed: int = 1234, tau: Optional[float] = None, inflow_scale: float = 1.0) -> Tuple[str, str, GeometryInfo]:
    """Write one of the named workloads into `out_dir`; returns (xml, gmy, info).

    `scale` < 1 shrinks radii and lengths (for fast parity tests) while keeping
    the physics choices (kernel, walls, iolets).  `tau` replaces the workload's
    relaxation time (the bifurcation's tau+) and `inflow_scale` multiplies the
    stenosis's inlet speeds: variants of a workload that stay stable for its
    full step count where the stated parameters do not."""
    os.makedirs(out_dir, exist_ok=True)
    rng = np.random.default_rng(seed)
    gmy = os.path.join(out_dir, f"{name}.gmy")
    xml = os.path.join(out_dir, f"{name}.xml")

    def sc(v, lo=3):
        return max(lo, int(round(v * scale)))

    if name == "pipe_r8":
        # Straight rigid pipe, LBGK tau=0.8, bounce-back walls, Nash pressure
        # inlet rho=1.001 / outlet rho=0.999, 2000 steps.
        v = Pipe(sc(8), sc(64, 4))
        u = CaseUnits(tau=0.8)
        write_case_xml(xml, os.path.basename(gmy), v, u, steps or 2000,
                       [PressureBC(1.001)], [PressureBC(0.999)])
    elif name == "pipe_r40":
        # Large straight pipe, LBGK tau=0.55, BFL walls, parabolic inlet u=0.02
        # ramped over 1000 steps, Nash outlet rho=1, 5000 steps.
        v = Pipe(sc(40), sc(800, 8))
        u = CaseUnits(tau=0.55)
        write_case_xml(xml, os.path.basename(gmy), v, u, steps or 4000,
                       [VelocityBC(0.02)], [PressureBC(1.0)], warmup=1000)
    elif name == "pipe_r40_short":
        # The large pipe's cross-section and physics over 200 slices (1,004,800
        # sites): the case the kernel profiles capture.
        v = Pipe(sc(40), sc(200, 8))
        u = CaseUnits(tau=0.55)
        write_case_xml(xml, os.path.basename(gmy), v, u, steps or 4000,
                       [VelocityBC(0.02)], [PressureBC(1.0)], warmup=1000)
    elif name == "bifurcation":
        # Y-bifurcation, TRT (magic 3/16, tau+=0.52), GZS walls, cosine pressure
        # inlet (mean 1, amplitude 1e-3, period 4000), two WK3 outlets.
        v = YBifurcation(sc(32), sc(400, 8), sc(25), sc(400, 8), 35.0)
        u = CaseUnits(tau=tau or 0.52)
        # Windkessel sizing.  The reference integrates the absolute lattice pressure
        # (InOutLetWK3.cc:72-91), so the total resistance must carry the outlet at
        # p = cs^2 rho with rho ~ 1 for the Poiseuille flow the branches admit; the
        # characteristic resistance is the lattice wave impedance cs/A (a larger one
        # makes the one-step-lagged flow feedback unstable); C gives R_p C ~ 2000 steps.
        mu = (u.tau - 0.5) / 3.0
        r_par = 8.0 * mu * v.lp / (math.pi * v.rp ** 4)
        r_dau = 8.0 * mu * v.ld / (math.pi * v.rd ** 4)
        q_out = CS2 * 5e-4 / (2.0 * r_par + r_dau)
        area = math.pi * v.rd ** 2
        outs = []
        for _ in range(2):
            r_tot = CS2 / q_out * float(rng.uniform(0.8, 1.2))
            rc = math.sqrt(CS2) / area
            rp = r_tot - rc
            outs.append(WK3BC(r_c=rc, r_p=rp, c_p=2000.0 / rp, area=area))
        write_case_xml(xml, os.path.basename(gmy), v, u, steps or 8000,
                       [PressureBC(1.0, 1e-3, 4000.0)], outs, relaxation_parameter=3.0 / 16.0)
    elif name == "stenosis":
        # Stenosed artery, LBGK+LES with outlet sponge, pulsatile parabolic inlet:
        # peak 0.05 (1 + 0.5 sin(2 pi t / 10^4)) lattice units from t = 0, as the
        # reference's InOutLetFileVelocity (a parabolic profile whose peak speed
        # is read from a file of time/speed pairs, one every 50 steps here).
        v = Stenosis(sc(48), sc(1200, 8), sc(24), max(4.0, 96 * scale))
        u = CaseUnits(tau=tau or 0.502)
        n_steps = steps or 20000
        table = os.path.join(out_dir, "stenosis_inflow.txt")
        with open(table, "w") as fh:
            for k in range(0, n_steps + 101, 50):
                peak = inflow_scale * 0.05 * (1.0 + 0.5 * math.sin(2.0 * math.pi * k / 10000.0))
                fh.write(f"{k * u.dt!r} {u.speed_to_phys(peak)!r}\n")
        write_case_xml(xml, os.path.basename(gmy), v, u, n_steps,
                       [FileVelocityBC(os.path.basename(table))], [PressureBC(1.0)],
                       sponge={"viscosity_ratio": 10.0, "width": max(4.0, 60 * scale),
                               "lifetime": 2 * (steps or 20000)})
    else:
        raise ValueError(name)
    info = voxelise(v, gmy)
    return xml, gmy, info
