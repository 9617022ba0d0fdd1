"""Host logic of the serving loop (no device)."""
import math

import numpy as np

from qmcbeaver_b200.serving import blocked_error, make_jobs, state_footprint
from qmcbeaver_b200.system import make_system


def test_blocked_error():
    rng = np.random.default_rng(0)
    x = rng.normal(0.0, 1.0, 4000)
    e = blocked_error(x)
    assert 0.5 / math.sqrt(4000) < e < 2.0 / math.sqrt(4000)
    assert blocked_error([1.0, 2.0]) == math.inf


def test_footprint_grows_with_size():
    a = state_footprint(make_system("vmc_water_10e"), 1000)
    b = state_footprint(make_system("dmc_6nuc_30e"), 1000)
    assert 0 < a < b
    # 30 electrons: 3232 doubles per walker block, two blocks per walker
    assert b == 2 * 1000 * 3232 * 8


def test_poisson_arrivals_and_sizes():
    jobs = make_jobs(8, rate=10.0, seed=2, electrons=(4, 12), walkers=(256, 300))
    t = [j.arrival for j in jobs]
    assert all(b > a for a, b in zip(t, t[1:]))
    for j in jobs:
        assert 4 <= j.system.n_electrons <= 12 and j.system.n_electrons % 2 == 0
        assert j.system.n_basis == 4 * j.system.n_electrons
        assert 256 <= j.walkers <= 300
