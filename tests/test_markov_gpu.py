"""The device Markov chain (qmcb_run_steps) against the oracle-driven chain:
same algorithm, different random streams, so energies must agree within the
combined statistical error; and DMC branching against a restatement of
QMCRun::nonunitWeightBranching with the same device random draws."""
import numpy as np
import pytest

from philox import uniform4
from qmcbeaver_b200.api import QMCB200Functions
from qmcbeaver_b200.desc import QMCB_DMC, QMCB_IMPORTANCE_SAMPLING, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


def oracle_vmc(s, W, sweeps, dt, seed, warm):
    """Single-electron Metropolis with the oracle (QMCWalker, no importance
    sampling): R' = R + sqrt(dt) g, p = |psi'/psi|^2; observables p E' + q E
    on the steps that move electron 0."""
    from oracle.evaluators import OracleEvaluator
    orc = OracleEvaluator(s, qf_mod=0, dt=dt)
    rng = np.random.default_rng(seed)
    N = s.n_electrons
    R = s.initial_positions(W, seed=seed)
    cur = orc.new_walkers(W)
    trial = orc.new_walkers(W)
    orc.evaluate(cur, R, -1)
    for t, c in zip(trial, cur):
        orc.copy(t, c)
    res = orc.results(cur)
    E, lp = res["e_local"].copy(), res["log_abs_psi"].copy()
    samples = []
    for step in range(sweeps * N):
        e = step % N
        Rt = R.copy()
        Rt[:, e] += np.sqrt(dt) * rng.standard_normal((W, 3))
        orc.evaluate(trial, Rt, e)
        r = orc.results(trial)
        p = np.minimum(1.0, np.exp(2 * (r["log_abs_psi"] - lp)))
        p[r["singular"] != 0] = 0.0
        acc = p > rng.random(W)
        if e == 0 and step >= warm * N:
            samples.append(np.mean(p * r["e_local"] + (1 - p) * E))
        for i in range(W):
            if acc[i]:
                orc.copy(cur[i], trial[i])
            else:
                orc.copy(trial[i], cur[i])
        R[acc] = Rt[acc]
        E[acc] = r["e_local"][acc]
        lp[acc] = r["log_abs_psi"][acc]
    return np.array(samples)


def block_stats(x, nblocks=20):
    b = np.array_split(np.asarray(x), nblocks)
    m = np.array([bb.mean() for bb in b])
    return m.mean(), m.std(ddof=1) / np.sqrt(len(m))


def test_vmc_energy_agrees_with_oracle_chain():
    s = make_system("vmc_water_10e", seed=1)
    W, sweeps, warm, dt = 100, 220, 20, 0.09
    ref = oracle_vmc(s, W, sweeps, dt, seed=7, warm=warm)
    f = QMCB200Functions(s, W, run_params(dt=dt, seed=99, rel_cutoff=0.0))
    f.init_walkers(s.initial_positions(W, seed=7))
    N = s.n_electrons
    f.run_steps(1, warm * N)
    gpu = []
    acc = 0.0
    for k in range(sweeps - warm):
        st = f.run_steps(1 + (warm + k) * N, N)
        gpu.append(st.sum_weight_energy / st.sum_weight)
        acc += st.sum_accept / st.n_moves
    m1, e1 = block_stats(ref)
    m2, e2 = block_stats(gpu)
    z = abs(m1 - m2) / np.hypot(e1, e2)
    assert z < 2.0, (m1, e1, m2, e2)
    assert 0.2 < acc / (sweeps - warm) < 0.99


def branch_restatement(w, thr, fuse, seed, step):
    """QMCRun::nonunitWeightBranching (QMcBeaver/src/QMCRun.cpp:740-814): one
    pass over the live list in which a walker above the threshold splits
    (copy appended in list order), one below 0.01 dies and ones below the
    fusion threshold fuse in pairs; the fusion draws are the device's, keyed
    by the list position of a pair's first member."""
    w = list(w)
    keep = [True] * len(w)
    adds = []
    pend = None
    for i in range(len(w)):
        if w[i] > thr:
            w[i] = w[i] / 2
            adds.append(i)
        elif w[i] < 0.01:
            keep[i] = False
        elif w[i] < fuse:
            if pend is None:
                pend = i
            else:
                w1, w2 = w[pend], w[i]
                w3 = w1 + w2
                if uniform4(seed, pend, step, 7)[0] < w1 / w3:
                    w[pend] = w3
                    keep[i] = False
                else:
                    w[i] = w3
                    keep[pend] = False
                pend = None
    return [w[i] for i in range(len(w)) if keep[i]] + [w[i] for i in adds]


def test_branching_matches_reference_rule():
    s = make_system("vmc_water_10e", seed=1)
    W = 3000
    f = QMCB200Functions(s, 2 * W, run_params(run_type=QMCB_DMC, seed=4242, limit_branching=0))
    f.init_walkers(s.initial_positions(W, seed=1))
    rng = np.random.default_rng(3)
    w = np.exp(rng.normal(0.0, 1.2, W))
    w[rng.random(W) < 0.05] = 0.005
    f.set_walker_weights(w)
    n = f.branch(step=77)
    expect = branch_restatement(w, 2.0, 0.45, 4242, 77)
    got = f.get_walkers()["weight"]
    assert n == len(expect)
    np.testing.assert_allclose(got, expect, rtol=0, atol=0)
    assert abs(got.sum() - sum(expect)) < 1e-9
    # a second pass on the reordered list (deaths and appended copies), with a
    # fusion threshold above half the branching threshold: fused survivors
    # whose summed weight exceeds the branching threshold must not split
    w2 = np.exp(rng.normal(0.0, 0.8, n))
    w2[rng.random(n) < 0.3] = 1.3
    w2[rng.random(n) < 0.05] = 0.005
    f.set_params(run_params(run_type=QMCB_DMC, seed=4242, limit_branching=0, branching_threshold=2.0,
                            fusion_threshold=1.5))
    f.set_walker_weights(w2)
    n2 = f.branch(step=78)
    expect2 = branch_restatement(w2, 2.0, 1.5, 4242, 78)
    got2 = f.get_walkers()["weight"]
    assert n2 == len(expect2)
    np.testing.assert_allclose(got2, expect2, rtol=0, atol=0)
    assert np.sum(np.array(expect2) > 2.0) > 0  # fused survivors above the threshold stay whole


def test_branching_copies_walker_state():
    s = make_system("vmc_water_10e", seed=1)
    W = 40
    f = QMCB200Functions(s, 2 * W, run_params(run_type=QMCB_DMC, limit_branching=0))
    f.init_walkers(s.initial_positions(W, seed=2))
    w = np.ones(W)
    w[3] = 3.0
    f.set_walker_weights(w)
    before = f.get_walkers()
    n = f.branch(step=1)
    after = f.get_walkers()
    assert n == W + 1
    np.testing.assert_array_equal(after["R"][-1], before["R"][3])
    assert after["weight"][3] == after["weight"][-1] == 1.5
    assert after["e_local"][-1] == before["e_local"][3]


def test_dmc_population_stays_controlled():
    s = make_system("dmc_6nuc_30e", seed=1)
    W = 2048
    N = s.n_electrons
    eq = 5 * N

    def params(e0, start):
        return run_params(run_type=QMCB_DMC, sampling=QMCB_IMPORTANCE_SAMPLING,
                          qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, energy_modification=1, dt=0.01,
                          refresh_interval=50, reweight_start_step=start, energy_trial=e0, energy_estimated=e0,
                          energy_original=e0, seed=5, energy_cutoff=2, population_control=100.0)

    f = QMCB200Functions(s, 4 * W, params(-1.0, eq))
    f.init_walkers(s.initial_positions(W, seed=3))
    st = f.run_steps(0, eq)
    assert st.n_walkers == W  # weights held at 1 while equilibrating
    wk = f.get_walkers()
    e0 = float(np.mean(wk["e_local"]))
    f.set_params(params(e0, 0))
    f.init_walkers(wk["R"])
    st = f.run_steps(0, 10 * N)
    assert st.n_moves > 0.5 * 10 * N * W
    assert 0.7 * W < st.n_walkers < 1.5 * W
    assert np.isfinite(st.sum_weight_energy / st.sum_weight)
    assert st.n_singular < 0.01 * st.n_moves


def _deletion_pair(s, W, e0, equil_steps, rel_cutoff, w0, step):
    """One DMC step that reweights (electron 0 moves) with and without the
    reference's deletion rules, splitting and fusion switched off so the only
    deaths are deleted walkers; returns both walker lists (same draws)."""
    out = []
    for deletion in (0, 1):
        p = run_params(run_type=QMCB_DMC, sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL,
                       dt=0.01, energy_modification=1, energy_cutoff=2, energy_trial=e0, energy_estimated=e0,
                       energy_original=e0, reweight_start_step=0, branching_threshold=1e300, fusion_threshold=0.0,
                       limit_branching=0, rel_cutoff=rel_cutoff, seed=5, walker_deletion=deletion,
                       equilibration_steps=equil_steps)
        f = QMCB200Functions(s, W, p)
        f.init_walkers(s.initial_positions(W, seed=4))
        f.set_walker_weights(w0)
        st = f.run_steps(step, 1)
        out.append(f.get_walkers())
        f.close()
    return out


@pytest.mark.parametrize("phase", ["production", "equilibration"])
def test_walker_deletion_rules(phase):
    """QMCWalker::reweight_walker's deletions (QMcBeaver/src/QMCWalker.cpp:
    1196-1365): the walkers that survive with the rules on are exactly those
    of the rules-off run that no rule deletes, with identical weights."""
    s = make_system("dmc_6nuc_30e", seed=1)
    W, N = 2000, s.n_electrons
    f = QMCB200Functions(s, W, run_params(qf_modification=2, dt=0.01))
    f.init_walkers(s.initial_positions(W, seed=4))
    e0 = float(np.median(f.get_walkers()["e_local"]))
    f.close()
    rng = np.random.default_rng(8)
    w0 = np.exp(rng.normal(0.0, 0.3, W))
    heavy = rng.random(W) < 0.01
    light = rng.random(W) < 0.02
    w0[heavy] = 60.0   # above 50 (production) and 2 x 2.0 (equilibration)
    w0[light] = 0.05   # below 0.1 (equilibration only)
    step = 10 * N      # moves electron 0: reweights
    equil = step + 1000 if phase == "equilibration" else 0
    off, on = _deletion_pair(s, W, e0, equil, 0.3, w0, step)
    assert len(off["weight"]) == W  # nothing dies without the rules (all weights >= 0.05)
    rel = np.abs((off["e_local"] - e0) / e0)
    dW = off["weight"] / w0
    if phase == "production":
        # dW^(age+1) stays far below 15 at dt 0.01 with the energy cutoff
        keep = (off["weight"] <= 50.0) & (rel <= 0.3)
        assert dW.max() < 2.0
    else:
        # (the heavy-walker rule, weight above twice the branching threshold,
        # is off here with splitting)
        keep = (off["weight"] >= 0.1) & (dW <= 1.5) & (dW >= 0.5) & (rel <= 0.3)
    assert 0 < keep.sum() < W
    np.testing.assert_array_equal(on["weight"], off["weight"][keep])
    np.testing.assert_array_equal(on["R"], off["R"][keep])
