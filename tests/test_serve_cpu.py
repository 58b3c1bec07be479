"""Host logic of the serving benchmark (no GPU)."""
import numpy as np
import pytest

from appearance_b200 import serve


def test_job_list_is_seeded_and_follows_the_mix():
    a = serve.serving_jobs(4000, 200.0, 4, seed=3)
    b = serve.serving_jobs(4000, 200.0, 4, seed=3)
    assert a == b
    arr = np.array([j["arrival"] for j in a])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert np.mean(np.diff(arr)) == pytest.approx(1 / 200.0, rel=0.08)
    res = [(j["width"], j["height"]) for j in a]
    for r, p in zip(serve.RESOLUTIONS, serve.RES_PROBS):
        assert res.count(r) / len(res) == pytest.approx(p, abs=0.03)
    assert {j["spp"] for j in a} == set(serve.SPPS)
    assert {j["scene"] for j in a} == {0, 1, 2, 3}
    assert all(j["depth"] == 8 for j in a)


def test_summary_percentiles():
    jobs = [dict(width=10, height=10, spp=1)] * 5
    res = [dict(total_ms=t, queued_ms=0.0, gpu_ms=1.0) for t in (5.0, 1.0, 3.0, 2.0, 4.0)]
    s = serve.summarise(jobs, res, 2.0)
    assert s["p50_ms"] == 3.0 and s["p99_ms"] == 5.0
    assert s["msamples_per_s"] == pytest.approx(500 / 2.0 / 1e6)


def test_server_creation_fails_cleanly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(serve.RendererError):
        serve.RenderServer(hbm_budget=1e9)
