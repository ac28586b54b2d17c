"""One lattice spread over several GPUs: a slab per process, halo exchange per step.

HemePure runs one lattice on many MPI ranks: each rank owns the sites of its
part of the decomposition (src/geometry/decomposition/BasicDecomposition.cc,
OptimisedDecomposition.cc) and, every step, sends the post-collision values of
the links that cross into a neighbour's part and copies the received ones into
place (geometry::LatticeData::SendAndReceive / CopyReceived,
src/geometry/LatticeData.cc:665-689).

Here the cut is a set of planes across one lattice axis (slabs with balanced
site counts, `plan`).  Each process owns one slab on its own GPU
(`hb_create_shard_from_xml`) and keeps the plane of sites just beyond each cut
as halo sites.  After each step it packs, on the device, the post-collision
values that the neighbouring slabs pull across the cut (`hb_shard_pack`),
exchanges them with the two neighbours (point-to-point over torch.distributed:
NCCL between GPUs, gloo on the CPU), and unpacks what it received into its halo
sites before the next step (`hb_shard_unpack`).  Every site's arithmetic is the
one-GPU arithmetic, so the sharded run equals the single-lattice run bit for bit.

Restrictions (rejected at creation): a GZS wall link whose extrapolation
neighbour is a halo site (the virtual node re-gathers the neighbour's
pre-collision values, which live in the other slab), and a Windkessel iolet
whose coupling sites or centre site span two slabs.
"""

from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import lbm as _lbm


class ShardSpec(C.Structure):
    _fields_ = [("axis", C.c_int), ("lo", C.c_int64), ("hi", C.c_int64)]


def plan(xml_path: str, n_shards: int, kernel: str = "LBGK", axis: int = -1) -> Tuple[int, List[int]]:
    """Slab bounds with balanced site counts: shard k owns the sites whose
    coordinate along `axis` lies in [bounds[k], bounds[k+1])."""
    L = _lbm.library()
    ax = C.c_int(axis)
    bounds = np.zeros(n_shards + 1, np.int64)
    rc = L.hb_shard_plan(xml_path.encode(), _lbm.KERNELS[kernel], int(n_shards), C.byref(ax),
                         bounds.ctypes.data_as(C.c_void_p))
    _lbm.check_rc(rc, "hb_shard_plan")
    return int(ax.value), [int(b) for b in bounds]


def describe(xml_path: str, kernel: str, wall: str, axis: int, lo: int, hi: int) -> dict:
    """The shard's sites and exchange lists, computed on the host without a GPU:
    `owned` and `halo` global site ids (the reference's contiguous order), and
    for each of send_lower, send_upper, recv_lower, recv_upper an (m, 2) array of
    (global site id, direction) in exchange order."""
    L = _lbm.library()
    spec = ShardSpec(axis, lo, hi)
    counts = np.zeros(6, np.int64)
    rc = L.hb_shard_describe(xml_path.encode(), _lbm.KERNELS[kernel], _lbm.WALLS[wall], C.byref(spec),
                             counts.ctypes.data_as(C.c_void_p), None, None, None, None, None, None)
    _lbm.check_rc(rc, "hb_shard_describe")
    owned = np.zeros(counts[0], np.int64)
    halo = np.zeros(counts[1], np.int64)
    lists = [np.zeros((int(c), 2), np.int64) for c in counts[2:]]
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = L.hb_shard_describe(xml_path.encode(), _lbm.KERNELS[kernel], _lbm.WALLS[wall], C.byref(spec),
                             ptr(counts), ptr(owned), ptr(halo), *[ptr(a) for a in lists])
    _lbm.check_rc(rc, "hb_shard_describe")
    return {"owned": owned, "halo": halo, "send_lower": lists[0], "send_upper": lists[1],
            "recv_lower": lists[2], "recv_upper": lists[3]}


class Exchange:
    """The per-step halo exchange of one shard with its two neighbours over
    torch.distributed.  Buffers are torch tensors on the shard's device (CUDA
    for NCCL, CPU for gloo); `pack` fills the send buffers, `unpack` consumes
    the receive buffers.  Every rank posts the same operations in the same order:
    lower neighbour first, then upper."""

    DTYPES = {8: "float64", 4: "float32", 2: "int16"}  # the storage element, moved as raw bits

    def __init__(self, sizes: Sequence[int], rank: int, world: int, device, dist, group=None, elem_bytes: int = 8):
        import torch
        self.rank, self.world, self.dist, self.group = rank, world, dist, group
        dt = getattr(torch, self.DTYPES[int(elem_bytes)])
        mk = lambda k: torch.empty(max(1, int(k)), dtype=dt, device=device)  # noqa: E731
        self.sizes = [int(k) for k in sizes]
        self.send_lower, self.send_upper, self.recv_lower, self.recv_upper = (mk(k) for k in self.sizes)

    def run(self) -> None:
        d = self.dist
        ops = []
        if self.rank > 0:
            ops.append(d.P2POp(d.isend, self.send_lower[:self.sizes[0]], self.rank - 1, self.group))
            ops.append(d.P2POp(d.irecv, self.recv_lower[:self.sizes[2]], self.rank - 1, self.group))
        if self.rank < self.world - 1:
            ops.append(d.P2POp(d.isend, self.send_upper[:self.sizes[1]], self.rank + 1, self.group))
            ops.append(d.P2POp(d.irecv, self.recv_upper[:self.sizes[3]], self.rank + 1, self.group))
        if ops:
            for req in d.batch_isend_irecv(ops):
                req.wait()


class ShardedLBM:
    """This process's slab of a lattice on its GPU, stepped in lockstep with the
    other ranks of the process group (launched one process per GPU)."""

    def __init__(self, xml_path: str, kernel: str = "LBGK", wall: str = "SBB", precision: str = "fp64",
                 device: Optional[int] = None, group=None, axis: int = -1):
        import torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.axis, self.bounds = plan(xml_path, self.world, kernel, axis)
        dev = torch.cuda.current_device() if device is None else device
        self.lbm = _lbm.LBM(xml_path, kernel=kernel, wall=wall, precision=precision, device=dev,
                            shard=(self.axis, self.bounds[self.rank], self.bounds[self.rank + 1]))
        sizes, elem = self.lbm.shard_halo_sizes()
        self.exchange = Exchange(sizes, self.rank, self.world, torch.device("cuda", dev), dist, group, elem)
        # Neighbours must agree on what crosses each cut.
        mine = torch.tensor(sizes, dtype=torch.int64, device=torch.device("cuda", dev))
        every = [torch.zeros_like(mine) for _ in range(self.world)]
        dist.all_gather(every, mine, group=group)
        for r in range(self.world - 1):
            lower, upper = every[r].tolist(), every[r + 1].tolist()
            if lower[1] != upper[2] or upper[0] != lower[3]:
                raise RuntimeError(f"shards {r} and {r + 1} disagree on the values crossing their cut")

    def step(self, n: int = 1, macro: bool = False) -> None:
        """`n` time steps, each followed by the halo exchange.  The stability of
        all shards is reduced after every step, so that every rank raises
        together (none is left waiting in the next exchange)."""
        import torch
        stream = torch.cuda.current_stream().cuda_stream
        ex = self.exchange
        flag = torch.zeros(1, dtype=torch.int32, device=ex.send_lower.device)
        for k in range(n):
            unstable = 0
            try:
                self.lbm.step(1, macro=macro and k == n - 1)
            except _lbm.Unstable:
                unstable = 1
            self.lbm.shard_pack(ex.send_lower, ex.send_upper, stream)
            ex.run()
            self.lbm.shard_unpack(ex.recv_lower, ex.recv_upper, stream)
            flag.fill_(unstable)
            self.dist.all_reduce(flag, op=self.dist.ReduceOp.MAX, group=self.group)
            if int(flag.item()):
                raise _lbm.Unstable(_lbm.HB_UNSTABLE, "the simulation became unstable on some shard")

    def site_ids(self) -> np.ndarray:
        return self.lbm.shard_site_ids()
