"""The device Umrigar93 move (sampling umrigar93_importance_sampling) step
by step against the oracle: the device's own random draws (Philox,
restated in tests/philox.py) give the proposal, the oracle (oracle/umrigar.py,
pinned to the reference's QMCWalker) the Green's functions and psi, and so
the acceptance of every walker; then the VMC energy it samples against the
plain Metropolis chain's."""
import numpy as np
import pytest

from philox import umrigar_uniforms
from qmcbeaver_b200.api import QMCB200Functions
from qmcbeaver_b200.desc import (QMCB_NO_IMPORTANCE_SAMPLING, QMCB_QF_NONE, QMCB_QF_UMRIGAR93_UNEQUAL,
                                 QMCB_UMRIGAR93_IMPORTANCE_SAMPLING, run_params)
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


def _near_nuclei(s, R, rng):
    # every third walker has one electron of each spin 0.05 bohr from a nucleus,
    # where the exponential branch of the move dominates
    for w in range(0, len(R), 3):
        for e in (0, s.n_alpha):
            R[w, e] = s.coords[int(rng.integers(s.n_nuclei))] + 0.05 * rng.standard_normal(3)
    return R


@pytest.mark.parametrize("workload,qf,dt", [("vmc_water_10e", QMCB_QF_NONE, 0.09),
                                            ("dmc_6nuc_30e", QMCB_QF_UMRIGAR93_UNEQUAL, 0.01),
                                            ("vmc_multidet_12e", QMCB_QF_UMRIGAR93_UNEQUAL, 0.03)])
def test_moves_replay_against_oracle(workload, qf, dt):
    from oracle import umrigar as U
    from oracle.evaluators import OracleEvaluator
    s = make_system(workload, seed=1)
    W, seed = 96, 4242
    C, Z = np.asarray(s.coords), np.asarray(s.Z, float)
    rng = np.random.default_rng(3)
    R = _near_nuclei(s, s.initial_positions(W, seed=8), rng)
    f = QMCB200Functions(s, W, run_params(sampling=QMCB_UMRIGAR93_IMPORTANCE_SAMPLING, qf_modification=qf, dt=dt,
                                          seed=seed, rel_cutoff=0.0))
    f.init_walkers(R)
    orc = OracleEvaluator(s, qf_mod=qf, dt=dt)
    ws = orc.new_walkers(W)
    N = s.n_electrons
    n_checked = n_acc = n_slater = 0
    steps = list(range(1, 1 + N)) + [N + 1, N + s.n_alpha + 1]
    for step in steps:
        e = step % N
        before = f.get_walkers(W)
        R0 = before["R"]
        orc.evaluate(ws, R0, -1)
        r0 = orc.results(ws)
        Rt = R0.copy()
        u = [umrigar_uniforms(seed, w, step) for w in range(W)]
        for w in range(W):
            F = U.frame(C, Z, R0[w, e], r0["mod_grad"][w, e], dt)
            Rt[w, e] = U.propose(F, u[w], dt)[0]
            n_slater += u[w][0] >= F[3]
        orc.evaluate(ws, Rt, -1)
        rt = orc.results(ws)
        f.run_steps(step, 1)
        R1 = f.get_walkers(W)["R"]
        for w in range(W):
            lf = U.log_forward(C, Z, R0[w], r0["mod_grad"][w], e, Rt[w, e], dt)
            lr = U.log_reverse(C, Z, Rt[w], rt["mod_grad"][w], e, R0[w, e], dt)
            lp = 2 * (rt["log_abs_psi"][w] - r0["log_abs_psi"][w]) + lr - lf
            p = 0.0 if (rt["singular"][w] or np.isnan(lp)) else float(np.exp(min(lp, 0.0)))
            if abs(p - u[w][6]) < 1e-5:
                continue  # too close to call at the evaluators' rounding
            acc = p > u[w][6]
            n_checked += 1
            n_acc += acc
            want = Rt[w] if acc else R0[w]
            # the proposal carries the drift, whose device and oracle values
            # agree to ~1e-10 relative away from nodes and less near them
            # (the Slater matrices' condition): 1e-8 of the displacement
            tol = 1e-8 * max(1.0, float(np.abs(Rt[w, e] - R0[w, e]).max()))
            assert np.allclose(R1[w], want, rtol=0, atol=tol), (step, w, acc, p, u[w][6])
    assert n_checked > 0.95 * W * len(steps)
    assert 0.1 * n_checked < n_acc < n_checked
    assert n_slater > 0


def test_vmc_energy_agrees_with_plain_metropolis():
    """Same wavefunction, two samplers: the VMC energies agree within their
    statistical errors (detailed balance of the Umrigar93 move)."""
    s = make_system("vmc_water_10e", seed=1)
    W, warm, sweeps = 2048, 40, 240
    N = s.n_electrons

    def chain(sampling, dt, seed):
        f = QMCB200Functions(s, W, run_params(sampling=sampling, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL,
                                              dt=dt, seed=seed, rel_cutoff=0.0))
        f.init_walkers(s.initial_positions(W, seed=seed))
        f.run_steps(1, warm * N)
        e, acc = [], 0.0
        for k in range(sweeps - warm):
            st = f.run_steps(1 + (warm + k) * N, N)
            e.append(st.sum_weight_energy / st.sum_weight)
            acc += st.sum_accept / st.n_moves
        return np.array(e), acc / (sweeps - warm)

    def stats(x, nb=20):
        m = np.array([b.mean() for b in np.array_split(x, nb)])
        return m.mean(), m.std(ddof=1) / np.sqrt(nb)

    e1, a1 = chain(QMCB_UMRIGAR93_IMPORTANCE_SAMPLING, 0.09, 11)
    e2, a2 = chain(QMCB_NO_IMPORTANCE_SAMPLING, 0.09, 12)
    (m1, s1), (m2, s2) = stats(e1), stats(e2)
    # two device samplers against each other on the random-orbital water
    # system, whose local energies are heavy-tailed (block errors of 15-45
    # Ha on means near 1e3 Ha): the blocked errors are loose estimates, so
    # the gate is 4 combined errors (the gates against the reference program
    # and the oracle chain, in test_energy_gpu / test_markov_gpu, are 2)
    assert abs(m1 - m2) < 4.0 * np.hypot(s1, s2), (m1, s1, m2, s2)
    # the importance-sampled move is accepted more often than the blind one
    assert a1 > a2 and 0.3 < a1 < 1.0, (a1, a2)
