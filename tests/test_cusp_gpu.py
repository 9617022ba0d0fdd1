"""Cusp replacement on the device: per-call parity with the oracle (pinned
to the reference with the replacement on), with electrons inside the
replacement radii; one and several determinants; the mixed-precision path
and the Markov chain with the replacement on."""
import dataclasses

import numpy as np
import pytest

from helpers import PARITY_RTOL, compare, cond_bounds, place_near_nuclei, slater_conditions
from qmcbeaver_b200.api import QMCB200Functions
from qmcbeaver_b200.desc import QMCB_IMPORTANCE_SAMPLING, QMCB_PREC_MIXED, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


def _cusp(workload, seed=3):
    return dataclasses.replace(make_system(workload, seed=seed), replace_cusps=True)


def _sequence(s, W, sweeps, seed, qf=2, dt=0.01):
    from oracle.evaluators import OracleEvaluator
    orc = OracleEvaluator(s, qf_mod=qf, dt=dt)
    f = QMCB200Functions(s, W, qf_modification=qf, dt=dt)
    ws = orc.new_walkers(W)
    slots = np.arange(W)
    rng = np.random.default_rng(seed)
    R = s.initial_positions(W, seed=seed)
    place_near_nuclei(R, s, rng)
    N = s.n_electrons
    slope, limit = cond_bounds(s)
    good = np.ones(W, bool)
    worst = np.zeros(W)
    for i in range(-1, sweeps * N):
        e = -1 if i < 0 else i % N
        if e >= 0:
            if i % 3 == 0:
                R[:, e] = s.coords[rng.integers(s.n_nuclei, size=W)] + 0.03 * rng.standard_normal((W, 3))
            else:
                R[:, e] += 0.15 * rng.standard_normal((W, 3))
        orc.evaluate(ws, R, e)
        ref = orc.results(ws)
        worst = np.maximum(worst, slater_conditions(orc, ws, s))
        good &= worst < limit
        out = f.evaluate(slots, R, e)
        kap = orc.kappa(ws)
        compare(out, ref, PARITY_RTOL, f"{s.name} call {i} whichE={e}", mask=good, kappa=kap)
        if (~good).any():
            tol = max(PARITY_RTOL, slope * float(worst[~good].max()))
            compare(out, ref, tol, f"{s.name} call {i} whichE={e} (cond {worst[~good].max():.1e})", mask=~good,
                    kappa=kap)
    f.close()


@pytest.mark.parametrize("workload,W", [("vmc_water_10e", 32), ("dmc_6nuc_30e", 32), ("vmc_multidet_12e", 16),
                                        ("vmc_cambridge2_16e", 16)])
def test_cusp_replacement_matches_oracle(workload, W):
    _sequence(_cusp(workload), W, 2, seed=7)


def test_cusp_mixed_precision_close_to_fp64():
    s = _cusp("dmc_6nuc_30e")
    W = 128
    a = QMCB200Functions(s, W, run_params(qf_modification=2, dt=0.01))
    b = QMCB200Functions(s, W, run_params(qf_modification=2, dt=0.01, precision=QMCB_PREC_MIXED))
    R = s.initial_positions(W, seed=4)
    place_near_nuclei(R, s, np.random.default_rng(4))
    sl = np.arange(W)
    x, y = a.evaluate(sl, R, -1), b.evaluate(sl, R, -1)
    ok = (x["status"] == 0) & (y["status"] == 0)
    err = np.abs(x["e_local"] - y["e_local"])[ok]
    assert np.median(err) < 1e-2, np.median(err)


def test_cusp_chain_consistent_with_full_evaluation():
    s = _cusp("dmc_6nuc_30e", seed=2)
    W = 1024
    p = run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01,
                   refresh_interval=0, seed=9, rel_cutoff=0.0)
    f = QMCB200Functions(s, W, p)
    f.init_walkers(s.initial_positions(W, seed=3))
    N = s.n_electrons
    for k in range(10):
        st = f.run_steps(k * N, N)
        assert np.isfinite(st.sum_weight_energy / st.sum_weight)
    w = f.get_walkers()
    fresh = QMCB200Functions(s, W, qf_modification=2, dt=0.01).evaluate(np.arange(W), w["R"], -1)
    ok = fresh["status"] == 0
    for k in ("e_local", "log_abs_psi"):
        err = np.abs(w[k][ok] - fresh[k][ok]) / np.maximum(np.abs(fresh[k][ok]), 1.0)
        assert np.max(err) < 1e-8, (k, np.max(err))
