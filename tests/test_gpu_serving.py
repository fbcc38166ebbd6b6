"""Serving on the GPU: results alone and in the mix are identical; a short
Poisson run completes every request."""
import numpy as np
import pytest

from pyheartsim_b200 import serving

pytestmark = pytest.mark.gpu


def _small_requests():
    # the first request runs ~4000 steps, long enough that the later two arrive
    # (2 and 4 ms after it) while it is on the GPU
    reqs = [serving.Request(0, 0.0, 20_000, 200.0, 0, 11_000),
            serving.Request(1, 0.0, 30_000, 20.0, 1, 12_000),
            serving.Request(2, 0.0, 25_000, 25.0, 0, 13_000)]
    return reqs


@pytest.mark.parametrize("async_download", [False, True])
def test_result_alone_equals_result_in_the_mix(async_download, cuda_device):
    alone = {}
    for r in _small_requests():
        srv = serving.Server(hbm_budget_bytes=8 << 30, steps_per_launch=40)
        done, _ = srv.run([r], keep_history=True)
        srv.close()
        alone[r.rid] = done[0].history
    # all three together, the later ones admitted while the first is running
    mix = _small_requests()
    mix[1].arrival_s = 0.002
    mix[2].arrival_s = 0.004
    # built on the device this time: the same instances, so the same results
    srv = serving.Server(hbm_budget_bytes=8 << 30, steps_per_launch=40, rebalance_every=2, device_build=True,
                         async_download=async_download)
    done, totals = srv.run(mix, keep_history=True)
    srv.close()
    assert len(done) == 3
    # the requests really shared the GPU: each later request was admitted
    # before the first one retired
    by_id = {r.rid: r for r in done}
    assert by_id[1].admit_s < by_id[0].done_s and by_id[2].admit_s < by_id[0].done_s
    assert by_id[0].admit_s <= by_id[1].admit_s
    for r in done:
        assert r.status == 0
        assert r.history.shape == alone[r.rid].shape
        np.testing.assert_array_equal(r.history, alone[r.rid])   # bit-identical


def test_short_poisson_run_completes(cuda_device):
    reqs = serving.poisson_requests(6, rate_per_s=20.0, n_min=20_000, n_max=60_000, dur_ms=(20.0, 60.0), seed=7)
    srv = serving.Server(hbm_budget_bytes=8 << 30, steps_per_launch=50)
    done, totals = srv.run(reqs)
    srv.close()
    s = serving.summarize(done, totals, reqs)
    assert s["requests"] == 6 and s["failed"] == 0
    assert s["p99_latency_s"] >= s["p50_latency_s"] > 0
