"""The serving driver's arrival process (host logic, no GPU): a seeded
compound Poisson process whose offered rate is the requested one."""
import numpy as np

from kspir_b200.serving import poisson_schedule


def test_schedule_is_seeded_sorted_and_in_range():
    a = poisson_schedule(2000.0, 2.0, seed=7, max_group=128)
    assert a == poisson_schedule(2000.0, 2.0, seed=7, max_group=128)
    assert a != poisson_schedule(2000.0, 2.0, seed=8, max_group=128)
    times = [t for t, _ in a]
    sizes = [g for _, g in a]
    assert times == sorted(times)
    assert all(0.0 < t < 2.0 for t in times)
    assert all(1 <= g <= 128 for g in sizes)


def test_schedule_offers_the_requested_rate():
    for rate, max_group in [(5000.0, 128), (100.0, 1), (800.0, 8)]:
        duration = 4000.0 * (1 + max_group) / 2 / rate   # ~4000 groups
        a = poisson_schedule(rate, duration, seed=11, max_group=max_group)
        offered = sum(g for _, g in a) / duration
        assert abs(offered / rate - 1) < 0.06, (rate, max_group, offered)
        if max_group == 1:
            assert all(g == 1 for _, g in a)
        # exponential gaps: their coefficient of variation is about 1
        gaps = np.diff([0.0] + [t for t, _ in a])
        assert 0.9 < gaps.std() / gaps.mean() < 1.1


def test_schedule_empty_when_duration_is_shorter_than_any_gap():
    assert poisson_schedule(1e-6, 1.0, seed=3) == []
