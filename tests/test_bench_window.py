"""The benchmark's timing window and cell-sort accounting (host logic)."""
import bench


def mean_age(first, K, I):
    """Mean steps since the last sort over the window's steps."""
    return sum((first + k) % I for k in range(K)) / K


def test_short_window_is_centred_in_the_sort_interval():
    for warmup in (0, 3, 5, 79, 80, 81, 200):
        for K, I in ((20, 80), (10, 40), (79, 80), (1, 80), (21, 80)):
            first = bench.window_start(warmup, K, I)
            assert warmup <= first < warmup + I
            assert abs(mean_age(first, K, I) - (I - 1) / 2) <= 0.5
            assert bench.sorts_in(first, K, I) <= 1


def test_long_window_starts_at_a_sort():
    for warmup in (0, 5, 80, 123):
        for K, I in ((80, 80), (160, 80), (120, 40)):
            first = bench.window_start(warmup, K, I)
            assert first >= warmup and first % I == 0
            assert bench.sorts_in(first, K, I) == K // I
            assert mean_age(first, K, I) == (I - 1) / 2


def test_no_sort_interval_keeps_the_warmup():
    assert bench.window_start(5, 20, 0) == 5


def test_amortised_sort_share():
    # a window without a sort is charged K / interval sorts; one with exactly
    # K / interval sorts is left as it ran
    assert bench.amortised_ms(10.0, 20, 30, 80, 0.5) == 10.0 + 0.25 * 0.5
    assert bench.amortised_ms(10.0, 80, 80, 80, 0.5) == 10.0
    assert bench.amortised_ms(10.0, 20, 30, 0, 0.5) == 10.0
