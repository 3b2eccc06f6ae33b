"""The serving tuner's choice among its trials (host logic, no GPU)."""
from anchorwave_b200 import autotune


def _t(slots, batch, seconds, p99):
    return {"slots": slots, "max_batch": batch, "seconds": seconds, "p99_ms": p99, "p50_ms": 0.0,
            "requests_per_s": 3000 / seconds}


def test_lowest_p99_among_the_fast_trials():
    trials = [_t(2, 1024, 4.6, 1899.0), _t(2, 2048, 4.4, 2100.0), _t(4, 1024, 4.3, 1410.0),
              _t(4, 2048, 6.0, 900.0)]
    # 4 x 2048 has the lowest p99 but finished 40% behind the fastest trial
    assert autotune.pick_serving(trials) == (4, 1024)


def test_ties_go_to_the_faster_trial():
    trials = [_t(2, 1024, 4.5, 1500.0), _t(4, 1024, 4.2, 1500.0)]
    assert autotune.pick_serving(trials) == (4, 1024)


def test_slack_bounds_the_candidates():
    trials = [_t(2, 1024, 4.0, 2000.0), _t(2, 2048, 4.5, 1000.0)]
    assert autotune.pick_serving(trials, slack=0.10) == (2, 1024)
    assert autotune.pick_serving(trials, slack=0.15) == (2, 2048)


def test_grid_is_the_whole_trace_candidates():
    assert set(autotune.SERVE_SLOTS) == {2} and set(autotune.SERVE_BATCH) == {1024, 2048}
