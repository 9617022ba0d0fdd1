"""The Umrigar93 importance-sampling move (umrigar93_importance_sampling)
restated in the oracle (oracle/umrigar.py) against moves made by the
reference's own QMCWalker (tests/golden/moves/*.npz, written by
tests/golden/make_moves.py), and the restated proposal against the
moments of the density it must sample."""
import glob
import math
import os

import numpy as np
import pytest

from helpers import GOLDEN_DIR
from oracle import umrigar as U
from oracle.evaluators import OracleEvaluator
from qmcbeaver_b200.system import system_from_arrays

MOVE_CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "moves", "*.npz")))


def load_moves(name):
    d = np.load(os.path.join(GOLDEN_DIR, "moves", name + ".npz"))
    return system_from_arrays({k[4:]: d[k] for k in d.files if k.startswith("sys_")}), d


def test_move_goldens_present():
    assert {"umrigar93_water", "umrigar93_dmc30"} <= set(MOVE_CASES)


@pytest.mark.parametrize("case", MOVE_CASES)
def test_green_functions_match_reference(case):
    s, d = load_moves(case)
    tau = float(d["dt"])
    C, Z = np.asarray(s.coords), np.asarray(s.Z, float)
    n_slater = 0
    for m in range(len(d["R0"])):
        e = int(d["whichE"][m])
        R0, R1 = d["R0"][m], d["R1"][m]
        # only electron e moved
        assert np.array_equal(np.delete(R0, e, 0), np.delete(R1, e, 0))
        f = U.log_forward(C, Z, R0, d["mg0"][m], e, R1[e], tau)
        r = U.log_reverse(C, Z, R1, d["mg1"][m], e, R0[e], tau)
        # the reference sums the two terms of each electron's density as
        # QMCDoubles k a^b exp(c) (QMcBeaver/src/QMCDouble.cpp:403-560), which
        # rounds differently from a log-sum-exp: up to ~1e-8 in the log
        for got, want in ((f, d["gf"][m][0]), (r, d["gf"][m][1])):
            assert abs(got - want) <= 1e-7 + 1e-12 * abs(want), (m, got, want)
        n_slater += U.frame(C, Z, R0[e], d["mg0"][m][e], tau)[4] > 0.5
    # both branches of the move appear among the recorded moves
    assert 0 < n_slater < len(d["R0"])


@pytest.mark.parametrize("case", MOVE_CASES)
def test_oracle_drift_matches_reference_walkers(case):
    """The modified drift the move uses, at the old and the new positions."""
    s, d = load_moves(case)
    orc = OracleEvaluator(s, qf_mod=int(d["qf_mod"]), dt=float(d["dt"]))
    ws = orc.new_walkers(len(d["R0"]))
    for R, mg in ((d["R0"], d["mg0"]), (d["R1"], d["mg1"])):
        orc.evaluate(ws, R, -1)
        got = orc.results(ws)["mod_grad"]
        scale = np.maximum(np.abs(mg).max(axis=(1, 2), keepdims=True), 1.0)
        assert np.max(np.abs(got - mg) / scale) < 1e-10


@pytest.mark.parametrize("z,d,vz,vr", [(8.0, 0.4, -3.0, 1.0), (1.0, 0.9, 0.5, 2.0), (6.0, 0.05, -6.0, 0.3)])
def test_proposal_samples_the_transition_density(z, d, vz, vr):
    """E[y] = P_g c + P_s A and E|y - A|^2 = P_g (|c - A|^2 + 3 tau) + P_s 3 / zeta^2
    for the Gaussian / exponential mixture the move draws from."""
    tau = 0.09
    C = np.array([[0.3, -0.2, 0.1], [5.0, 5.0, 5.0]])
    x = C[0] + d * np.array([0.0, 0.6, 0.8])
    v = vz * np.array([0.0, 0.6, 0.8]) + vr * np.array([1.0, 0.0, 0.0])
    F = U.frame(C, [z, 1.0], x, v, tau)
    A, c, zeta, pg, ps = F
    rng = np.random.default_rng(5)
    n = 60000
    ys = np.array([U.propose(F, 1.0 - rng.random(8), tau)[0] for _ in range(n)])
    mean = pg * c + ps * A
    r2 = pg * (float((c - A) @ (c - A)) + 3 * tau) + ps * 3.0 / zeta ** 2
    se = np.sqrt(np.maximum(ys.var(axis=0), 1e-30) / n)
    assert np.all(np.abs(ys.mean(axis=0) - mean) < 5 * se + 1e-12)
    q = ((ys - A) ** 2).sum(axis=1)
    assert abs(q.mean() - r2) < 5 * q.std() / math.sqrt(n)
