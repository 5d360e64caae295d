"""Host-side logic of the serving driver (no GPU): the request stream and the
latency summary it prints."""
import pytest

from vfb_b200 import serve, synth


class _R:
    def __init__(self, status):
        self.status = status


def test_percentile_nearest_rank():
    xs = [5.0, 1.0, 3.0, 2.0, 4.0]
    assert serve.percentile(xs, 0) == 1.0
    assert serve.percentile(xs, 50) == 3.0
    assert serve.percentile(xs, 100) == 5.0
    assert serve.percentile([], 50) is None


def test_summary_counts_statuses_and_splits_classes():
    res = [_R(0), _R(0), _R(2), None, _R(3)]
    lat = [0.001, 0.002, 0.5, 0.004, 0.003]
    large = [False, False, True, False, False]
    out = serve.summarize(10.0, res, lat, 1.0, 4, large)
    assert out["status"] == {"found": 2, "limit": 1, "missing": 1, "oom": 1}
    assert out["requests"] == 5 and out["solves_per_s"] == 5.0
    assert out["large"]["requests"] == 1 and out["large"]["p50_ms"] == pytest.approx(500.0)
    assert out["mixed"]["requests"] == 4 and out["mixed"]["p99_ms"] == pytest.approx(4.0)
    assert "large" not in serve.summarize(10.0, res, lat, 1.0, 4)


def test_request_stream_is_seeded_and_poisson_ordered():
    a = synth.config_serving(seed=4, count=200, rate=50.0, large_frac=0.05)
    b = synth.config_serving(seed=4, count=200, rate=50.0, large_frac=0.05)
    assert [t for t, _ in a] == [t for t, _ in b]
    assert [i.name for _, i in a] == [i.name for _, i in b]
    times = [t for t, _ in a]
    assert times == sorted(times) and times[0] > 0
    # the mean gap is about 1 / rate
    assert 0.5 / 50.0 < times[-1] / len(times) < 2.0 / 50.0
    assert any(i.name == "large" for _, i in a)
    # a slower rate replays the same requests further apart
    c = synth.config_serving(seed=4, count=200, rate=25.0, large_frac=0.05)
    assert [i.name for _, i in c] == [i.name for _, i in a]
    assert c[-1][0] > a[-1][0]
