"""CPU: the serving workload's request stream and the latency statistics (no device work)."""
import numpy as np
import pytest

from volprim_b200.serving import make_trace, percentile, schedule_spec


def test_trace_distribution():
    tr = make_trace(1, 4000, rate=50.0, n_scenes=4)
    gaps = np.diff([0.0] + [r.arrival for r in tr])
    assert abs(gaps.mean() - 1 / 50.0) < 0.1 / 50.0          # exponential with mean 1/rate
    assert abs(np.median(gaps) - np.log(2) / 50.0) < 0.15 / 50.0
    res = [r.config.image_width for r in tr]
    assert all(r.config.image_width == r.config.image_height for r in tr)
    for v in (64, 128, 256, 512):
        assert abs(res.count(v) / len(tr) - 0.25) < 0.03
    spp = [r.config.num_samples_per_pixel for r in tr]
    for v in (1, 4, 16, 64):
        assert abs(spp.count(v) / len(tr) - 0.25) < 0.03
    sc = [r.scene_id for r in tr]
    assert set(sc) == {0, 1, 2, 3}
    for r in tr[:200]:
        eye = np.array(r.camera.eye)
        assert abs(np.linalg.norm(eye) - 3.5) < 1e-5
        assert tuple(r.camera.lookat) == (0.0, 0.0, 0.0)
    # E[paths] = E[res^2] E[spp] = 87,040 x 21.25
    mean_paths = np.mean([r.paths for r in tr])
    assert abs(mean_paths / (87040 * 21.25) - 1) < 0.1
    assert [r.config.seed for r in tr[:5]] == [0, 1, 2, 3, 4]


def test_trace_is_seeded():
    a = make_trace(7, 50, 10.0, 4)
    b = make_trace(7, 50, 10.0, 4)
    assert [(r.arrival, r.scene_id, r.camera.eye, r.paths) for r in a] == \
           [(r.arrival, r.scene_id, r.camera.eye, r.paths) for r in b]


def test_percentile_nearest_rank():
    v = list(range(1, 101))
    assert percentile(v, 50) == 50
    assert percentile(v, 99) == 99
    assert percentile(v, 100) == 100
    assert percentile([3.0], 99) == 3.0


def test_schedule_spec():
    assert schedule_spec("fifo") == ("fifo", 0.0)
    assert schedule_spec("srpt") == ("srpt", 0.0)
    assert schedule_spec("srpt/0.25") == ("srpt", 0.25)
    for bad in ("lifo", "fair/1", "srpt/-1", "srpt/x"):
        with pytest.raises(ValueError):
            schedule_spec(bad)
