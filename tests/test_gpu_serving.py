"""The serving loop on the GPU: requests batched with others (continuous
batching over two workers / streams) return exactly what they return alone,
and what the plain FP64 kernel returns; the HBM budget bounds what is
admitted at once."""
import numpy as np
import pytest
import torch

from setsm_b200 import serving

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes(gpu_ctx):
    dev = torch.device("cuda", 0)
    return [serving.make_resident_scene(gpu_ctx, sid, 1024, 3, dev, seed=40 + sid)
            for sid in range(2)]


def stream(scenes, n=24, seed=5):
    return serving.poisson_requests(n, 400.0, scenes, seed=seed, grid_min=12, grid_max=96,
                                    levels=(0, 1), templates=(11, 15))


def test_mixed_batches_equal_requests_alone(gpu_ctx, scenes):
    reqs = stream(scenes)
    srv = serving.Server(scenes, max_batch=6, n_workers=2)
    rep = srv.run(reqs, realtime=False)
    assert rep["requests"] == len(reqs)
    assert rep["mean_batch"] > 1.5
    assert rep["p99_ms"] >= rep["p50_ms"] > 0
    dev = torch.device("cuda", 0)
    by_sid = {rs.sid: rs for rs in scenes}
    for r in reqs:
        alone, acc, _ = serving.run_alone(gpu_ctx, r, by_sid[r.sid], dev)
        assert r.accessable == acc
        assert r.nccresult.tobytes() == alone.tobytes(), r.rid
    # and the plain FP64 kernel gives the same results
    for r in reqs[:4]:
        plain, acc, _ = serving.run_alone(gpu_ctx, r, by_sid[r.sid], dev, kernel="plain")
        assert r.accessable == acc
        assert r.nccresult.tobytes() == plain.tobytes(), r.rid


def test_budget_bounds_admission(gpu_ctx, scenes):
    reqs = stream(scenes, n=12, seed=9)
    biggest = max(serving.request_bytes(r) for r in reqs)
    srv = serving.Server(scenes, hbm_budget=biggest, max_batch=4, n_workers=2)
    rep = srv.run(reqs, realtime=True)
    assert rep["requests"] == len(reqs)
    assert srv.max_in_use <= biggest
