"""The sharded form's host logic on the CPU: slab plan, halo lists, and the
exchange over torch.distributed (gloo, two and three ranks).

The values exchanged are checked against the oracle run on the whole lattice:
the value a shard sends for (site y, direction i) is y's post-collision f*_i,
which the single-lattice step pushes into the neighbour y + c_i, so it equals
the oracle's pre-collision f_i at y + c_i after the step.  Each rank packs those
values in its send-list order, the ranks exchange them with the same Exchange
class the GPU path uses, and each rank checks that what lands in its halo for
(y, i) is the value the owned site y + c_i pulls in the single-lattice run.
"""

import os

import numpy as np
import pytest

from conftest import make_small_case
from hemepure_b200 import shard, vessels
from oracle import oracle as O

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])


def _plans(xml, kernel, wall, n):
    axis, bounds = shard.plan(xml, n, kernel)
    return axis, bounds, [shard.describe(xml, kernel, wall, axis, bounds[k], bounds[k + 1]) for k in range(n)]


@pytest.mark.parametrize("key,n", [("pipe_r8", 2), ("pipe_r8", 3), ("pipe_bfl", 4)])
def test_plan_partitions_the_lattice(case_dir, key, n):
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    axis, bounds, d = _plans(xml, kernel, wall, n)
    owned = np.concatenate([x["owned"] for x in d])
    assert np.array_equal(np.sort(owned), np.arange(info.fluid_sites))
    sizes = [len(x["owned"]) for x in d]
    assert max(sizes) - min(sizes) <= 0.1 * info.fluid_sites / n + 2 * max(1, info.fluid_sites // 64)
    coords = O.Lattice(gmy).coords()
    for k, x in enumerate(d):
        c = coords[x["owned"], axis]
        assert c.min() >= bounds[k] and c.max() < bounds[k + 1]
        h = coords[x["halo"], axis]
        assert set(np.unique(h)) <= {bounds[k] - 1, bounds[k + 1]}
    # Neighbours agree on what crosses each cut, in the same order.
    for k in range(n - 1):
        assert np.array_equal(d[k]["send_upper"], d[k + 1]["recv_lower"])
        assert np.array_equal(d[k + 1]["send_lower"], d[k]["recv_upper"])
        assert len(d[k]["send_upper"]) > 0
    assert len(d[0]["recv_lower"]) == 0 and len(d[-1]["send_upper"]) == 0


def test_crossing_links_are_the_cut_links(case_dir):
    """Every pair sent across a cut is a link of a site next to the cut whose
    direction crosses it, and lands on a fluid site of the other slab."""
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_r8")
    axis, bounds, d = _plans(xml, kernel, wall, 2)
    lat = O.Lattice(gmy)
    coords, nbr = lat.coords(), lat.neighbours().reshape(-1)
    c_ax = [CX, CY, CZ][axis]
    for gid, dirn in d[0]["send_upper"]:
        assert coords[gid, axis] == bounds[1] - 1 and c_ax[dirn] == 1
        t = nbr[gid * 19 + dirn]
        assert t < info.fluid_sites * 19 and coords[t // 19, axis] == bounds[1]


def _exchange_worker(rank, world, port, xml, kernel, wall, steps, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        axis, bounds = shard.plan(xml, world, kernel)
        me = shard.describe(xml, kernel, wall, axis, bounds[rank], bounds[rank + 1])
        orc = O.Simulation(xml, kernel, wall, threads=1)
        orc.run(steps)
        f_next = orc.f()
        nbr = orc.lattice.neighbours().reshape(-1)

        def pushed(pairs):  # f*_i(y) of each (y, i): the oracle's f_i at y + c_i after the step
            tgt = nbr[pairs[:, 0] * 19 + pairs[:, 1]] // 19
            return f_next[tgt, pairs[:, 1]]

        sizes = [len(me["send_lower"]), len(me["send_upper"]), len(me["recv_lower"]), len(me["recv_upper"])]
        ex = shard.Exchange(sizes, rank, world, torch.device("cpu"), dist)
        if sizes[0]:
            ex.send_lower[:sizes[0]] = torch.from_numpy(pushed(me["send_lower"]))
        if sizes[1]:
            ex.send_upper[:sizes[1]] = torch.from_numpy(pushed(me["send_upper"]))
        ex.run()
        ok = True
        if sizes[2]:
            ok &= np.array_equal(ex.recv_lower[:sizes[2]].numpy(), pushed(me["recv_lower"]))
        if sizes[3]:
            ok &= np.array_equal(ex.recv_upper[:sizes[3]].numpy(), pushed(me["recv_upper"]))
        with open(os.path.join(out_dir, f"rank{rank}"), "w") as fh:
            fh.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_exchange_delivers_the_single_lattice_values(case_dir, tmp_path, world):
    import socket

    import torch.multiprocessing as mp
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_r8")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_exchange_worker, args=(world, port, xml, kernel, wall, 7, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        assert (tmp_path / f"rank{r}").read_text() == "ok"


def test_windkessel_iolet_across_a_cut_is_rejected(tmp_path):
    """A Windkessel outlet whose sites straddle a cut would need its flow sum
    across shards: the shard is refused, not silently wrong."""
    from hemepure_b200 import lbm
    v = vessels.Pipe(4, 16)
    vessels.voxelise(v, str(tmp_path / "p.gmy"))
    units = vessels.CaseUnits(tau=0.8)
    xml = tmp_path / "case.xml"
    vessels.write_case_xml(str(xml), "p.gmy", v, units, 10, [vessels.PressureBC(1.001)],
                           [vessels.WK3BC(r_c=1.0, r_p=10.0, c_p=100.0, area=np.pi * 16)])
    coords = O.Lattice(str(tmp_path / "p.gmy")).coords()
    mid = int(np.median(coords[:, 0]))
    with pytest.raises(lbm.HemeLBError, match="Windkessel"):
        shard.describe(str(xml), "LBGK", "SBB", 0, 0, mid)  # a cut along the pipe splits the outlet's sites
    shard.describe(str(xml), "LBGK", "SBB", 2, 0, int(coords[:, 2].max()) - 2)  # across the pipe: allowed
