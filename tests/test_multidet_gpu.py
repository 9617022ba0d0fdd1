"""Several determinants on the device (k_full_md / k_move_md): call-for-call
parity with the oracle (which is pinned to the reference on the same
expansions and on the reference's own multi-determinant inputs), the
consistency of the double-buffered determinant blocks after many updates,
walker copies, the Markov chain, and the FP64-only rule."""
import numpy as np
import pytest

from helpers import PARITY_RTOL, compare, cond_bounds, slater_conditions
from qmcbeaver_b200.api import QMCB200Functions, QMCBError
from qmcbeaver_b200.desc import (QMCB_DMC, QMCB_ECUT_BDJM_PUSH88, QMCB_IMPORTANCE_SAMPLING, QMCB_PREC_MIXED,
                                 QMCB_QF_UMRIGAR93_UNEQUAL, run_params)
from qmcbeaver_b200.system import make_random_molecule, make_system, with_cambridge2, with_determinants

pytestmark = pytest.mark.gpu


def _sequence(s, W, qf, dt, sweeps, sigma, seed, rejects=True):
    """Full evaluation, then single-electron updates of every electron (a
    share of them put back, the reference's rejection path) on the device
    and in the oracle; every call compared."""
    from oracle.evaluators import OracleEvaluator
    orc = OracleEvaluator(s, qf_mod=qf, dt=dt)
    f = QMCB200Functions(s, 2 * W, qf_modification=qf, dt=dt)
    ws = orc.new_walkers(W)
    slots = np.arange(W) + W // 2
    rng = np.random.default_rng(seed)
    R = s.initial_positions(W, seed=seed)
    N = s.n_electrons
    good = np.ones(W, bool)
    worst = np.zeros(W)
    slope, limit = cond_bounds(s)
    prev = None
    for i in range(-1, sweeps * N):
        e = -1 if i < 0 else i % N
        if e >= 0:
            if rejects and i % 5 == 4 and prev is not None:
                pe, pr = prev
                R[:, pe] = pr
                e = pe
                prev = None
            else:
                prev = (e, R[:, e].copy())
                R[:, e] += sigma * rng.standard_normal((W, 3))
        orc.evaluate(ws, R, e)
        ref = orc.results(ws)
        worst = np.maximum(worst, slater_conditions(orc, ws, s))
        good &= worst < limit
        out = f.evaluate(slots, R, e)
        # lap / E_L: the determinant-weighted sum amplifies the rounding of
        # each determinant's ratios by its condition number kappa
        kap = orc.kappa(ws)
        compare(out, ref, PARITY_RTOL, f"{s.name} call {i} whichE={e}", mask=good, kappa=kap)
        if (~good).any():
            tol = max(PARITY_RTOL, slope * float(worst[~good].max()))
            compare(out, ref, tol, f"{s.name} call {i} whichE={e} (cond {worst[~good].max():.1e})", mask=~good,
                    kappa=kap)
    f.close()
    return good.mean()


def test_multidet_matches_oracle():
    s = make_system("vmc_multidet_12e", seed=3)
    assert s.n_det == 12
    _sequence(s, 32, 2, 0.01, 3, 0.1, seed=11)


@pytest.mark.parametrize("ne,nn,nb,nd,nv,seed", [(4, 1, 12, 5, 2, 1), (10, 3, 30, 9, 3, 2), (40, 5, 120, 20, 6, 3)])
def test_multidet_shapes_match_oracle(ne, nn, nb, nd, nv, seed):
    # tiny spins, Cambridge2 with several determinants, and 20 determinants
    # of 20 x 20 per spin
    s = make_random_molecule(ne, nn, nb, 5.0, (1, 6, 7, 8), seed=seed)
    if seed == 2:
        s = with_cambridge2(s, seed=5)
    s = with_determinants(s, nd, nv, seed=seed)
    _sequence(s, 8, 2, 0.02, 1, 0.15, seed=seed)


def test_multidet_updates_consistent_with_full_evaluation():
    # many single-electron updates through the double-buffered determinant
    # blocks, accepted and rejected, equal a fresh full evaluation
    s = make_system("vmc_multidet_12e", seed=4)
    W = 256
    f = QMCB200Functions(s, 2 * W, qf_modification=2, dt=0.01)
    R = s.initial_positions(W, seed=8)
    a = np.arange(W)
    f.evaluate(a, R, -1)
    rng = np.random.default_rng(4)
    for m in range(6 * s.n_electrons):
        e = m % s.n_electrons
        R[:, e] += 0.15 * rng.standard_normal((W, 3))
        last = f.evaluate(a, R, e)
    fresh = f.evaluate(a + W, R, -1)
    ok = (last["status"] == 0) & (fresh["status"] == 0)
    assert ok.mean() > 0.9
    for k in ("e_local", "log_abs_psi"):
        err = np.abs(last[k][ok] - fresh[k][ok]) / np.maximum(np.abs(fresh[k][ok]), 1.0)
        assert np.max(err) < 1e-8, (k, np.max(err))
    np.testing.assert_array_equal(last["sign"][ok], fresh["sign"][ok])
    g = np.max(np.abs(last["grad"][ok] - fresh["grad"][ok]) / np.maximum(np.abs(fresh["grad"][ok]), 1.0))
    assert g < 1e-7


def test_multidet_copy_slot_clones_state():
    s = make_system("vmc_multidet_12e", seed=1)
    f = QMCB200Functions(s, 8)
    R = s.initial_positions(2, seed=2)
    f.evaluate([0, 1], R, -1)
    R1 = R.copy()
    R1[:, 2] += 0.1
    f.evaluate([0, 1], R1, 2)  # flips the alpha determinant block
    f.copy_slot(0, 5)
    R2 = R1.copy()
    R2[:, 8] += 0.1
    a = f.evaluate([0], R2[:1], 8)
    b = f.evaluate([5], R2[:1], 8)
    for k in ("log_abs_psi", "e_local", "grad"):
        np.testing.assert_array_equal(a[k], b[k])


def test_multidet_is_fp64_only():
    s = make_system("vmc_multidet_12e", seed=1)
    f = QMCB200Functions(s, 4)
    with pytest.raises(QMCBError, match="FP64"):
        f.set_params(run_params(precision=QMCB_PREC_MIXED))


def test_multidet_vmc_and_dmc_chains():
    # the device chain runs (VMC moves, refreshes, then DMC branching with
    # walker copies), energies stay finite, the population stays controlled
    # and the stored states equal fresh evaluations at the end
    s = make_system("vmc_multidet_12e", seed=2)
    W = 512
    N = s.n_electrons
    common = dict(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01,
                  refresh_interval=50, seed=5, rel_cutoff=0.0, energy_cutoff=QMCB_ECUT_BDJM_PUSH88)
    f = QMCB200Functions(s, 4 * W, run_params(**common))
    f.init_walkers(s.initial_positions(W, seed=3))
    vmc = []
    for k in range(20):
        st = f.run_steps(k * N, N)
        vmc.append(st.sum_weight_energy / st.sum_weight)
        assert 0.0 < st.sum_accept / st.n_moves < 1.0
    e0 = float(np.mean(vmc[5:]))
    assert np.isfinite(e0)
    # DMC from the equilibrated walkers, E_T = the VMC energy
    f.set_params(run_params(run_type=QMCB_DMC, energy_trial=e0, energy_estimated=e0, energy_original=e0,
                            population_control=100.0, reweight_start_step=0, **common))
    energies = []
    for k in range(20, 40):
        st = f.run_steps(k * N, N)
        assert st.n_moves > 0
        energies.append(st.sum_weight_energy / st.sum_weight)
    assert np.all(np.isfinite(energies))
    n = f.num_walkers()
    assert W // 8 < n < 8 * W
    w = f.get_walkers()
    assert np.all(np.isfinite(w["e_local"])) and np.all(np.isfinite(w["log_abs_psi"]))
    fresh = QMCB200Functions(s, n, qf_modification=2, dt=0.01).evaluate(np.arange(n), w["R"], -1)
    ok = fresh["status"] == 0
    err = np.abs(w["log_abs_psi"][ok] - fresh["log_abs_psi"][ok]) / np.maximum(np.abs(fresh["log_abs_psi"][ok]), 1.0)
    assert np.max(err) < 1e-8
