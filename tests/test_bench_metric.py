"""The metric's own arithmetic in bench.py, on the host: k, the outer
iteration after which the pressure drop stays within 1e-5 of the converged
value (time-to-converge is the device time of exactly k iterations)."""
import numpy as np

import bench


def test_first_stable_iter_monotone_approach():
    star = 1.4e6
    k = np.arange(1, 101)
    dp = star * (1.0 + 1e-2 * 0.8 ** k)
    # |dp_k - star| / star = 1e-2 0.8^k <= 1e-5  <=>  k >= log(1e-3) / log(0.8) = 30.96
    assert bench.first_stable_iter(dp, star) == 31
    assert np.all(np.abs(dp[30:] - star) <= 1e-5 * star) and abs(dp[29] - star) > 1e-5 * star


def test_first_stable_iter_counts_the_last_excursion():
    star = -250.0                       # the tolerance is relative to |dP*|
    dp = np.full(60, star)
    dp[10] = star * (1 + 2e-5)          # early excursion
    dp[41] = star * (1 - 3e-5)          # a later one resets the count
    assert bench.first_stable_iter(dp, star) == 43
    assert bench.first_stable_iter(dp, star, tol=5e-5) == 1


def test_first_stable_iter_edges():
    star = 85.8
    assert bench.first_stable_iter(np.full(5, star), star) == 1
    dp = np.full(5, star)
    dp[-1] = 2 * star                   # not settled within the history: one past its end
    assert bench.first_stable_iter(dp, star) == 6
