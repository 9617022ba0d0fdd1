"""The BF16 tensor-core orbital rows (QMCB_PREC_BF16_TC: BF16 operands,
FP32 accumulation; QMCB_PREC_BF16X3_TC: the split-precision variant, each
value split as hi + lo in BF16 and hi.hi + hi.lo + lo.hi accumulated in FP32)
against a CPU restatement of the same arithmetic.

The restatement rounds the FP64 basis values and MO coefficients exactly as
the kernels do (to 8 significant bits, round to nearest by Veltkamp's split,
flushed below 2^-126) and sums the BF16 products in FP64 (every product of
two BF16 values is exact in FP64); the tensor cores accumulate the same
products in FP32, so every row element must agree within the FP32
accumulation bound (terms x 2^-22 x the sum of the terms' magnitudes, twice
the worst case of truncating accumulation).  Then the chains of these modes
run, and their local energies are compared with the FP64 path on identical
configurations: the split-precision rows are closer to FP64 than the BF16
rows by orders of magnitude."""
import numpy as np
import pytest

from oracle.precision_study import basis_eval
from qmcbeaver_b200.api import QMCB200Functions
from qmcbeaver_b200.desc import (QMCB_IMPORTANCE_SAMPLING, QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC, QMCB_PREC_FP64,
                                 run_params)
from qmcbeaver_b200.system import make_random_molecule, make_system

pytestmark = pytest.mark.gpu


def bf16_round(x):
    """x rounded to 8 significant bits as the kernels round it."""
    x = np.asarray(x, np.float64)
    c = x * 35184372088833.0  # 2^45 + 1
    h = c - (c - x)
    h[np.abs(h) < 2.0 ** -126] = 0.0
    return h


def emulated_rows(chi, C, x3):
    """rows [5][P][n] from basis rows chi [5][P][K] and coefficients C [n][K];
    returns the products' sum in FP64 and the sum of their magnitudes."""
    Ch = bf16_round(C)
    Cl = bf16_round(C - Ch)
    out, mag = [], []
    for X in chi:
        Xh = bf16_round(X)
        Xl = bf16_round(X - Xh)
        r = Xh @ Ch.T
        m = np.abs(Xh) @ np.abs(Ch.T)
        if x3:
            r = r + Xh @ Cl.T + Xl @ Ch.T
            m = m + np.abs(Xh) @ np.abs(Cl.T) + np.abs(Xl) @ np.abs(Ch.T)
        out.append(r)
        mag.append(m)
    return np.stack(out, 1), np.stack(mag, 1)  # [P][5][n]


@pytest.mark.parametrize("prec", [QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC])
@pytest.mark.parametrize("wl", ["dmc_6nuc_30e", "random_80e"])
def test_bf16_rows_equal_restatement(wl, prec):
    # 30 electrons / 120 functions (the last 16-function K step half full);
    # 40 electrons per spin / 170 functions (two orbital tiles, the second
    # with 8 orbitals); 60 walkers (the last 25-walker tile partly empty)
    if wl == "random_80e":
        s = make_random_molecule(80, 8, 170, 6.0, (1, 6, 7, 8), seed=5)
    else:
        s = make_system(wl, seed=2)
    W, N = 60, s.n_electrons
    f = QMCB200Functions(s, W, qf_modification=2, dt=0.01, precision=prec)
    R = s.initial_positions(W, seed=3)
    sl = np.arange(W)
    f.evaluate(sl, R, -1)
    rng = np.random.default_rng(11)
    terms = (3 if prec == QMCB_PREC_BF16X3_TC else 1) * s.n_basis
    for e in (0, s.n_alpha - 1, s.n_alpha, N - 1):
        R[:, e] += 0.2 * rng.standard_normal((W, 3))
        f.evaluate_moved(sl, R[:, e], e)
        got = f.get_rows(W)
        C = s.mo_alpha() if e < s.n_alpha else s.mo_beta()
        chi = basis_eval(s, R[:, e])
        ref, mag = emulated_rows(chi, C, prec == QMCB_PREC_BF16X3_TC)
        assert got.shape == ref.shape
        tol = (terms + 16) * 2.0 ** -22 * mag + 1e-300
        err = np.abs(got - ref) / tol
        assert np.all(err <= 1.0), (wl, prec, e, float(err.max()))
    f.close()


def _el_after_moves(s, prec, W, seed=4):
    f = QMCB200Functions(s, W, qf_modification=2, dt=0.01, precision=prec)
    R = s.initial_positions(W, seed=seed)
    sl = np.arange(W)
    f.evaluate(sl, R, -1)
    rng = np.random.default_rng(seed)
    els = []
    for m in range(s.n_electrons):
        R[:, m] += 0.1 * rng.standard_normal((W, 3))
        out = f.evaluate_moved(sl, R[:, m], m)
        els.append(out["e_local"].copy())
    f.close()
    return np.array(els)


def test_bf16_local_energy_error_ordering():
    """Identical configurations, one sweep of single-electron moves: the
    split-precision rows' local energies are far closer to FP64 than the
    BF16 rows' (median over walker-moves), and both stay finite."""
    s = make_system("dmc_6nuc_30e", seed=2)
    W = 200
    ref = _el_after_moves(s, QMCB_PREC_FP64, W)
    bf = _el_after_moves(s, QMCB_PREC_BF16_TC, W)
    x3 = _el_after_moves(s, QMCB_PREC_BF16X3_TC, W)
    ok = np.isfinite(ref)
    d_bf = np.abs(bf - ref)[ok]
    d_x3 = np.abs(x3 - ref)[ok]
    assert np.isfinite(d_bf).all() and np.isfinite(d_x3).all()
    print(f"median |dE_L|: bf16 {np.median(d_bf):.2e}  bf16x3 {np.median(d_x3):.2e} Ha")
    assert np.median(d_x3) < 1e-2 * np.median(d_bf)


@pytest.mark.parametrize("prec", [QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC])
def test_bf16_chain_runs(prec):
    s = make_system("dmc_6nuc_30e", seed=2)
    W = 1000
    p = run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=2, dt=0.01, seed=7, rel_cutoff=0.0,
                   precision=prec)
    f = QMCB200Functions(s, W, p)
    f.init_walkers(s.initial_positions(W, seed=7))
    st = f.run_steps(0, 2 * s.n_electrons)
    wk = f.get_walkers()
    f.close()
    assert st.n_moves == 2 * s.n_electrons * W
    assert 0.3 < st.sum_accept / st.n_moves <= 1.0
    assert np.isfinite(wk["R"]).all()
