"""The sharded form on one GPU: every shard of a lattice as its own handle in one
process, stepped in turn, with the halo buffers exchanged by device copies
between the steps (no shard waits on another inside a kernel).  The assembled
result must equal the single-lattice run bit for bit: the FP64 shards against
the oracle, the FP32 shards against the single-lattice FP32 run."""

import numpy as np
import pytest

from conftest import gpu_available, make_small_case

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _run_shards(xml, kernel, wall, precision, n, steps):
    import torch

    from hemepure_b200 import lbm, shard
    axis, b = shard.plan(xml, n, kernel)
    parts = [lbm.LBM(xml, kernel=kernel, wall=wall, precision=precision, shard=(axis, b[k], b[k + 1]))
             for k in range(n)]
    dt = {8: torch.float64, 4: torch.float32, 2: torch.int16}
    bufs = []
    for p in parts:
        sizes, elem = p.shard_halo_sizes()
        bufs.append([torch.zeros(max(1, m), dtype=dt[elem], device="cuda") for m in sizes] + [sizes])
    for k in range(n - 1):  # neighbours agree on each cut
        assert bufs[k][4][1] == bufs[k + 1][4][2] and bufs[k + 1][4][0] == bufs[k][4][3]
    stream = torch.cuda.current_stream().cuda_stream
    for t in range(steps):
        for p in parts:
            p.step(1, macro=t == steps - 1)
        for p, (slo, shi, rlo, rhi, sizes) in zip(parts, bufs):
            p.shard_pack(slo, shi, stream)
        for k in range(n):
            sizes = bufs[k][4]
            if k > 0:
                bufs[k][2][:sizes[2]].copy_(bufs[k - 1][1][:sizes[2]])
            if k < n - 1:
                bufs[k][3][:sizes[3]].copy_(bufs[k + 1][0][:sizes[3]])
        for p, (slo, shi, rlo, rhi, sizes) in zip(parts, bufs):
            p.shard_unpack(rlo, rhi, stream)
    torch.cuda.synchronize()
    total = sum(p.n for p in parts)
    f = np.full((total, 19), np.nan)
    rho, u, wss = np.full(total, np.nan), np.full((total, 3), np.nan), np.full(total, np.nan)
    for p in parts:
        ids = p.shard_site_ids()
        f[ids] = p.GetFOld()
        r, v, w = p.GetPropertyCache()
        rho[ids], u[ids], wss[ids] = r, v, w
    sizes = [p.n for p in parts]
    for p in parts:
        p.close()
    return f, rho, u, wss, sizes


@pytest.mark.parametrize("key,n", [("pipe_r8", 2), ("pipe_r8", 3), ("pipe_bfl", 2), ("stenosis", 3)])
def test_fp64_shards_equal_the_oracle(case_dir, key, n):
    from oracle import oracle as O
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, key)
    steps = min(steps, 400)
    f, rho, u, wss, sizes = _run_shards(xml, kernel, wall, "fp64", n, steps)
    assert sum(sizes) == info.fluid_sites and min(sizes) > 0
    orc = O.Simulation(xml, kernel, wall)
    assert orc.run(steps, macro=True) == 0
    assert np.array_equal(f, orc.f())
    r_o, u_o, w_o = orc.macro()
    assert np.array_equal(rho, r_o) and np.array_equal(u, u_o) and np.array_equal(wss, w_o)
    assert np.max(np.abs(u_o)) > 0


def test_fp32_shards_equal_the_single_lattice(case_dir):
    from hemepure_b200 import lbm
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_bfl")
    steps = 300
    f, rho, u, wss, sizes = _run_shards(xml, kernel, wall, "fp32", 3, steps)
    one = lbm.LBM(xml, kernel=kernel, wall=wall, precision="fp32")
    one.step(steps, macro=True)
    assert np.array_equal(f, one.GetFOld())
    r1, u1, w1 = one.GetPropertyCache()
    assert np.array_equal(rho, r1) and np.array_equal(u, u1) and np.array_equal(wss, w1)


def test_a_shard_steps_one_step_per_call(case_dir):
    from hemepure_b200 import lbm, shard
    xml, gmy, info, kernel, wall, steps = make_small_case(case_dir, "pipe_r8")
    axis, b = shard.plan(xml, 2, kernel)
    p = lbm.LBM(xml, kernel=kernel, wall=wall, shard=(axis, b[0], b[1]))
    with pytest.raises(lbm.HemeLBError):
        p.step(2)
    p.close()
