"""Systems whose spins hold more than 16 electrons keep the moved spin's
inverse in HBM (two copies: the move reads one, writes the other, and
acceptance flips which is current) instead of staging it in shared memory.
Per-call parity of that path with the oracle, the Markov chain through
accept and reject, and the same arithmetic as the staged path."""
import numpy as np
import pytest

from helpers import PARITY_RTOL, compare, cond_bounds, slater_conditions
from qmcbeaver_b200.api import QMCB200Functions
from qmcbeaver_b200.desc import QMCB_IMPORTANCE_SAMPLING, QMCB_PREC_MIXED, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
from qmcbeaver_b200.system import make_random_molecule

pytestmark = pytest.mark.gpu


def _sequence(s, W, calls, seed, qf=2, dt=0.01):
    from oracle.evaluators import OracleEvaluator
    orc = OracleEvaluator(s, qf_mod=qf, dt=dt)
    f = QMCB200Functions(s, W, qf_modification=qf, dt=dt)
    ws = orc.new_walkers(W)
    slots = np.arange(W)
    rng = np.random.default_rng(seed)
    R = s.initial_positions(W, seed=seed, sigma=0.7)
    N = s.n_electrons
    slope, limit = cond_bounds(s)
    good = np.ones(W, bool)
    worst = np.zeros(W)
    for i in range(-1, calls):
        # both spins, wrapping around each spin's electrons more than once
        e = -1 if i < 0 else (i * 7) % N
        if e >= 0:
            R[:, e] += 0.2 * rng.standard_normal((W, 3))
        orc.evaluate(ws, R, e)
        ref = orc.results(ws)
        worst = np.maximum(worst, slater_conditions(orc, ws, s))
        good &= worst < limit
        out = f.evaluate(slots, R, e)
        # E_L = -lap/2 + V cancels terms of many electrons: its rounding
        # scales with (|lap|/2 + |V|) / |E_L| (applied to lap and E_L)
        amp = (np.abs(ref["lap"]) / 2 + np.abs(ref["potential"])) / np.maximum(np.abs(ref["e_local"]), 1.0)
        compare(out, ref, PARITY_RTOL, f"{s.name} call {i} whichE={e}", mask=good, kappa=amp)
        if (~good).any():
            tol = max(PARITY_RTOL, slope * float(worst[~good].max()))
            compare(out, ref, tol, f"{s.name} call {i} whichE={e} (cond {worst[~good].max():.1e})", mask=~good,
                    kappa=amp)
    f.close()


@pytest.mark.parametrize("ne,nn,nb,seed", [(52, 8, 160, 1), (100, 20, 400, 2)])
def test_large_spins_match_oracle(ne, nn, nb, seed):
    s = make_random_molecule(ne, nn, nb, 9.0 + ne / 25, (1, 6, 7, 8), seed=seed)
    assert s.n_alpha > 16
    _sequence(s, 8, 2 * ne + 3, seed=seed + 10)


def test_large_chain_matches_fresh_evaluations():
    """After Metropolis steps (accepted moves flip the current inverse copy,
    rejected ones leave it), the stored state equals a fresh full evaluation
    at the walkers' positions."""
    s = make_random_molecule(60, 10, 180, 10.0, (1, 6, 7, 8), seed=4)
    W, N = 256, s.n_electrons
    f = QMCB200Functions(s, W, run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL,
                                          dt=0.01, seed=9, rel_cutoff=0.0))
    f.init_walkers(s.initial_positions(W, seed=3))
    st = f.run_steps(1, 3 * N + 5)
    acc = st.sum_accept / st.n_moves
    assert 0.2 < acc < 0.999
    wk = f.get_walkers()
    g = QMCB200Functions(s, W, qf_modification=2, dt=0.01)
    fresh = g.evaluate(np.arange(W), wk["R"], -1)
    # a single-electron move after the chain uses the stored (current) inverse
    e = 11
    R2 = wk["R"].copy()
    R2[:, e] += 0.05
    a = f.evaluate(np.arange(W), R2, e)
    b = g.evaluate(np.arange(W), R2, -1)
    ok = fresh["status"] == 0
    assert ok.mean() > 0.9
    rel = lambda x, y: np.abs(x - y) / np.maximum(np.abs(y), 1.0)
    assert np.max(rel(wk["e_local"][ok], fresh["e_local"][ok])) < 1e-7
    assert np.max(np.abs(a["log_abs_psi"][ok] - b["log_abs_psi"][ok])) < 1e-8
    assert np.max(rel(a["e_local"][ok], b["e_local"][ok])) < 1e-7


def test_large_mixed_precision_runs():
    s = make_random_molecule(60, 10, 180, 10.0, (1, 6, 7, 8), seed=4)
    W = 128
    f64 = QMCB200Functions(s, W, qf_modification=2, dt=0.01)
    f32 = QMCB200Functions(s, W, run_params(precision=QMCB_PREC_MIXED, qf_modification=2, dt=0.01))
    R = s.initial_positions(W, seed=5)
    a, b = f64.evaluate(np.arange(W), R, -1), f32.evaluate(np.arange(W), R, -1)
    rng = np.random.default_rng(1)
    for e in (0, 31, 45):
        R[:, e] += 0.1 * rng.standard_normal((W, 3))
        a, b = f64.evaluate(np.arange(W), R, e), f32.evaluate(np.arange(W), R, e)
    ok = (a["status"] == 0) & (b["status"] == 0)
    assert np.median(np.abs(a["log_abs_psi"][ok] - b["log_abs_psi"][ok])) < 1e-3


def test_inverse_layouts_compute_the_same_numbers(monkeypatch):
    """The HBM-resident and the staged inverse give identical results (the
    same element formulas); the layout threshold moved by the environment."""
    s = make_random_molecule(52, 8, 160, 11.0, (1, 6, 7, 8), seed=1)
    W = 64
    outs = []
    for staged_max in ("16", "64"):
        monkeypatch.setenv("QMCB_STAGED_INVERSE_MAX", staged_max)
        f = QMCB200Functions(s, W, run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=2, dt=0.01, seed=4,
                                              rel_cutoff=0.0))
        f.init_walkers(s.initial_positions(W, seed=6))
        f.run_steps(1, 2 * s.n_electrons + 7)
        outs.append((f.get_walkers(), f.state_bytes()))
        f.close()
    (a, bytes_hbm), (b, bytes_staged) = outs
    assert bytes_hbm > bytes_staged  # two inverse copies per spin
    for k in ("R", "e_local", "log_abs_psi", "weight"):
        assert np.array_equal(a[k], b[k]), k
