"""Asynchronous step batches (qmcb_run_steps_async / qmcb_steps_collect):
two batches in flight on one handle follow exactly the chain of the same
steps run synchronously, and are collected in order."""
import numpy as np
import pytest

from qmcbeaver_b200.api import QMCB200Functions, QMCBError
from qmcbeaver_b200.desc import QMCB_IMPORTANCE_SAMPLING, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


def test_two_batches_in_flight_match_synchronous_steps():
    s = make_system("vmc_water_10e", seed=1)
    W, N = 512, s.n_electrons
    p = run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.05, seed=8,
                   rel_cutoff=0.0)
    a, b = QMCB200Functions(s, W, p), QMCB200Functions(s, W, p)
    R = s.initial_positions(W, seed=2)
    a.init_walkers(R)
    b.init_walkers(R)
    sync = [a.run_steps(k * N, N) for k in range(6)]
    got = []
    b.run_steps_async(0, N)
    for k in range(1, 6):
        b.run_steps_async(k * N, N)
        with pytest.raises(QMCBError, match="two batches"):
            b.run_steps_async(99 * N, N)
        with pytest.raises(QMCBError, match="collect"):
            b.run_steps(99 * N, N)
        got.append(b.steps_collect())
    got.append(b.steps_collect())
    with pytest.raises(QMCBError, match="no batch"):
        b.steps_collect()
    for x, y in zip(sync, got):
        assert x.n_moves == y.n_moves
        assert x.sum_weight_energy == pytest.approx(y.sum_weight_energy, rel=1e-12)
    assert np.array_equal(a.get_walkers()["R"], b.get_walkers()["R"])
