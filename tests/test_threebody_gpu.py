"""Three-body Jastrow on the device (tb_term / tb_move_lane / tb_full_lane):
per-call parity with the oracle (pinned to the reference on its own inputs),
alone and combined with cusp replacement and several determinants; the
incremental move against fresh evaluations; the Markov chain."""
import dataclasses

import numpy as np
import pytest

from helpers import PARITY_RTOL, compare, cond_bounds, place_near_nuclei, slater_conditions
from qmcbeaver_b200.api import QMCB200Functions
from qmcbeaver_b200.desc import QMCB_IMPORTANCE_SAMPLING, QMCB_PREC_MIXED, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
from qmcbeaver_b200.system import make_random_molecule, make_system, with_determinants, with_three_body

pytestmark = pytest.mark.gpu


def _sequence(s, W, sweeps, seed, qf=2, dt=0.01):
    from oracle.evaluators import OracleEvaluator
    orc = OracleEvaluator(s, qf_mod=qf, dt=dt)
    f = QMCB200Functions(s, W, qf_modification=qf, dt=dt)
    ws = orc.new_walkers(W)
    slots = np.arange(W)
    rng = np.random.default_rng(seed)
    R = s.initial_positions(W, seed=seed, sigma=0.7)
    place_near_nuclei(R, s, rng)
    N = s.n_electrons
    slope, limit = cond_bounds(s)
    good = np.ones(W, bool)
    worst = np.zeros(W)
    for i in range(-1, sweeps * N):
        e = -1 if i < 0 else i % N
        if e >= 0:
            R[:, e] += 0.2 * rng.standard_normal((W, 3))
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


def test_three_body_matches_oracle():
    _sequence(make_system("vmc_threebody_16e", seed=3), 32, 2, seed=7)


@pytest.mark.parametrize("ne,nn,nb,cusp,nd,seed", [(2, 1, 6, False, 1, 1), (10, 3, 30, True, 1, 2),
                                                   (12, 3, 36, True, 6, 3), (30, 6, 120, False, 1, 4)])
def test_three_body_combinations_match_oracle(ne, nn, nb, cusp, nd, seed):
    # one electron per spin, with cusp replacement, with several
    # determinants, and the 30-electron benchmark molecule
    s = with_three_body(make_random_molecule(ne, nn, nb, 5.0, (1, 6, 7, 8), seed=seed), seed=seed,
                        separate_kinds=seed % 2 == 0)
    s = dataclasses.replace(s, replace_cusps=cusp)
    if nd > 1:
        s = with_determinants(s, nd, 3, seed=seed)
    _sequence(s, 8, 1, seed=seed)


def test_three_body_moves_consistent_with_full_evaluation():
    s = make_system("vmc_threebody_16e", seed=4)
    W = 256
    f = QMCB200Functions(s, 2 * W, qf_modification=2, dt=0.01)
    R = s.initial_positions(W, seed=8, sigma=0.7)
    a = np.arange(W)
    f.evaluate(a, R, -1)
    rng = np.random.default_rng(4)
    for m in range(5 * s.n_electrons):
        e = m % s.n_electrons
        R[:, e] += 0.15 * rng.standard_normal((W, 3))
        last = f.evaluate(a, R, e)
    fresh = f.evaluate(a + W, R, -1)
    ok = (last["status"] == 0) & (fresh["status"] == 0)
    assert ok.mean() > 0.9
    for k in ("e_local", "log_abs_psi"):
        err = np.abs(last[k][ok] - fresh[k][ok]) / np.maximum(np.abs(fresh[k][ok]), 1.0)
        assert np.max(err) < 1e-8, (k, np.max(err))


def test_three_body_chain_runs_in_both_precisions():
    s = make_system("vmc_threebody_16e", seed=2)
    N = s.n_electrons
    for prec in (0, QMCB_PREC_MIXED):
        p = run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01,
                       refresh_interval=50, seed=3, rel_cutoff=0.0, precision=prec)
        f = QMCB200Functions(s, 1024, p)
        f.init_walkers(s.initial_positions(1024, seed=3, sigma=0.7))
        for k in range(8):
            st = f.run_steps(k * N, N)
            assert np.isfinite(st.sum_weight_energy / st.sum_weight)
            assert 0.0 < st.sum_accept / st.n_moves <= 1.0
        f.close()
