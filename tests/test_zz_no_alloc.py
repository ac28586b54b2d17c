"""hb_moment_sums_noalloc: the conserved-sum reduction without any device allocation.

It serves callers whose device memory is already committed (their own pool or a
fixed HBM budget) and who cannot let the library call cudaMalloc; it works on
buffers they own and keeps its scratch in a fixed array inside the library.
This file is collected last so that a run stopping at the first failure has
already run every other test."""

import ctypes as C

import numpy as np
import pytest

from conftest import make_small_case
from hemepure_b200 import lbm

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point(case_dir):
    import torch
    xml, gmy, info, kernel, wall, _ = make_small_case(case_dir, "pipe_bfl")
    sim = lbm.LBM(xml, kernel=kernel, wall=wall)
    sim.step(30)
    ref = sim.moment_sums()                      # hb_moment_sums: allocates its scratch
    f = np.ascontiguousarray(sim.GetFOld())     # [n, 19] AoS, reference order
    dev_f = torch.from_numpy(f).to("cuda")
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    L = lbm.library()
    free_after = []
    for call in range(2):                        # two calls in a row share the scratch
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.hb_moment_sums_noalloc(C.c_void_p(dev_f.data_ptr()), 1, 19, sim.n, C.c_void_p(out.data_ptr()),
                                      C.c_void_p(stream))
        assert rc == 0, lbm.last_create_error()
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        got = out.cpu().numpy()
        assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0]), (call, got, ref)
        assert np.max(np.abs(got[1:] - ref[1:])) <= 1e-12 * abs(ref[0]), (call, got, ref)
    # After the first call (which may load the library's module), calls take no device memory.
    assert free_after[1] == free_after[0], free_after


def test_noalloc_at_its_site_limit():
    """Exactly 16,777,216 sites (8192 scratch slots): distribution i of site s is
    v[s + i], so the sums are those of a sliding window, computed here with torch."""
    import torch
    n = 16_777_216
    g = torch.Generator(device="cuda").manual_seed(7)
    v = torch.rand(n + 19, dtype=torch.float64, device="cuda", generator=g) + 0.5
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    L = lbm.library()
    torch.cuda.synchronize()
    rc = L.hb_moment_sums_noalloc(C.c_void_p(v.data_ptr()), 1, 1, n, C.c_void_p(out.data_ptr()),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lbm.last_create_error()
    torch.cuda.synchronize()
    win = v.as_strided((n, 19), (1, 1))
    cx = torch.tensor([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0], dtype=torch.float64, device="cuda")
    cy = torch.tensor([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1], dtype=torch.float64, device="cuda")
    cz = torch.tensor([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1], dtype=torch.float64, device="cuda")
    ref = torch.stack([win.sum(), (win * cx).sum(), (win * cy).sum(), (win * cz).sum()]).cpu().numpy()
    got = out.cpu().numpy()
    assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0]), (got, ref)
    assert np.max(np.abs(got[1:] - ref[1:])) <= 1e-10 * abs(ref[0]), (got, ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = lbm.library()
    rc = L.hb_moment_sums_noalloc(C.c_void_p(16), 1, 19, 16_777_217, C.c_void_p(16), None)
    assert rc == -1
    assert "exceed" in lbm.last_create_error()
