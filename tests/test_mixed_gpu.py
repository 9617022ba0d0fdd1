"""Mixed-precision path (FP32 basis, orbital rows and Sherman-Morrison
update; FP64 determinant ratio, ratio sums, LU refresh, energies): same
evaluate sequence as the FP64 path, local-energy error stated per system."""
import numpy as np
import pytest

from qmcbeaver_b200.api import QMCB200Functions, QMCBError
from qmcbeaver_b200.desc import QMCB_PREC_FP64, QMCB_PREC_MIXED, run_params
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


def el_errors(wl, W, sigma, sweeps=2):
    s = make_system(wl, seed=1)
    f64 = QMCB200Functions(s, W, run_params(precision=QMCB_PREC_FP64, qf_modification=2, dt=0.01))
    f32 = QMCB200Functions(s, W, run_params(precision=QMCB_PREC_MIXED, qf_modification=2, dt=0.01))
    R = s.initial_positions(W, seed=4)
    rng = np.random.default_rng(1)
    sl = np.arange(W)
    f64.evaluate(sl, R, -1)
    f32.evaluate(sl, R, -1)
    errs = []
    for m in range(sweeps * s.n_electrons):
        e = m % s.n_electrons
        R[:, e] += sigma * rng.standard_normal((W, 3))
        a = f64.evaluate(sl, R, e)
        b = f32.evaluate(sl, R, e)
        ok = (a["status"] == 0) & (b["status"] == 0)
        errs.append(np.abs(a["e_local"] - b["e_local"])[ok])
    return np.concatenate(errs)


@pytest.mark.parametrize("wl,W,sigma,median_tol", [("vmc_water_10e", 128, 0.3, 1e-3), ("dmc_6nuc_30e", 128, 0.1, 1e-2)])
def test_mixed_local_energy_error(wl, W, sigma, median_tol):
    e = el_errors(wl, W, sigma)
    print(f"{wl}: |E_L(mixed) - E_L(FP64)| median {np.median(e):.2e} p99 {np.percentile(e, 99):.2e} max {e.max():.2e} Ha")
    assert np.median(e) < median_tol


def test_precision_switch_requires_reinit():
    s = make_system("vmc_water_10e", seed=1)
    f = QMCB200Functions(s, 4, run_params(precision=QMCB_PREC_FP64))
    R = s.initial_positions(4, seed=1)
    f.evaluate(np.arange(4), R, -1)
    f.set_params(run_params(precision=QMCB_PREC_MIXED))
    with pytest.raises(QMCBError, match="another precision"):
        f.evaluate(np.arange(4), R, 1)
    f.evaluate(np.arange(4), R, -1)
    f.evaluate(np.arange(4), R, 1)


def test_mixed_chain_runs():
    s = make_system("dmc_6nuc_30e", seed=1)
    W = 1024
    f = QMCB200Functions(s, 2 * W, run_params(precision=QMCB_PREC_MIXED, dt=0.01, qf_modification=2, sampling=1,
                                              refresh_interval=50))
    f.init_walkers(s.initial_positions(W, seed=2))
    st = f.run_steps(0, 90)
    assert st.n_moves == 90 * W
    assert 0.5 < st.sum_accept / st.n_moves < 1.0
