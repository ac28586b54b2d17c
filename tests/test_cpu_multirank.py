"""The N > 1 path of the benchmark on CPU: two ranks over gloo (127.0.0.1).

bench.py runs one replica per rank (the plain form does not shard a lattice);
its only collectives are the max over ranks of the device timings.  Here two
processes reduce different timings and must agree on the slowest, and the
whole-job figure must count both replicas' work over that time.  The
reference arm must leave ranks other than 0 without work or output.
"""

import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(values[rank], dist, "cpu")
        out[rank] = (ms, bench.replica_mlups(world, 1000, 10, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    port = _free_port()
    values = [2.0, 5.0]
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, values, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms, mlups = res[0]
    assert ms == 5.0
    assert mlups == pytest.approx(2 * 1000 * 10 / 5e-3 / 1e6)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_reference_arm_on_a_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
