"""Continuous-batching server: requests arrive while others run, are admitted
as capacity frees up, and each result equals the same request solved alone."""

import numpy as np
import pytest

from hemepure_b200 import lbm, serving

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def requests(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("req"))
    return serving.generate_requests(10, d, seed=11, radius=(4.0, 8.0), length_radii=(6.0, 12.0),
                                     steps=(150, 400), workers=1)


def test_server_completes_a_stream_and_matches_solo_runs(requests):
    serving.poisson_arrivals(requests, rate_per_s=200.0, seed=3)
    # A budget that holds only part of the stream at once, so admission waits for retirements.
    total = sum(r.sites for r in requests)
    budget = lbm.Batch.bytes_for(int(total * 0.5), int(total * 0.5), 256)
    srv = serving.Server(budget, block_steps=50)
    srv.run(requests, keep_results=True)
    rep = srv.report()
    print("serving report", rep)
    assert rep["requests"] == len(requests) and rep["failed"] == 0
    assert rep["p99_latency_s"] >= rep["p50_latency_s"] > 0
    # overlap: some request was admitted while another was still running
    spans = sorted((r.admitted, r.finished) for r in srv.completed)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    for r in srv.completed[:3]:
        b = lbm.Batch(r.sites * 2 + 1024, r.sites * 2 + 1024, 4)
        slot = b.add_xml(r.xml, r.kernel, r.wall, r.steps)
        done = []
        while not done:
            done = b.run(50)
        solo = b.macro(slot)
        for a, m in zip(solo, r.result):
            assert np.array_equal(a, m), r.rid


def test_autotuner_picks_a_measured_configuration(requests):
    t = serving.autotune(requests[:3], tolerance=1e-4, block_steps=32)
    assert t.precision == "fp32"
    assert t.sites_per_thread in (1, 2) and t.block in (128, 256)
    assert t.mlups == max(t.table.values()) > 0
