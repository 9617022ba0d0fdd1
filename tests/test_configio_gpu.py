"""print_configs from the device: the records of qmcb_run_step_configs, as
written by configio.run_with_configs, against the oracle at the recorded
positions; and a run that writes configurations follows the same Markov
chain as one that does not."""
import numpy as np
import pytest

from qmcbeaver_b200.api import QMCB200Functions
from qmcbeaver_b200.configio import read_configs, run_with_configs
from qmcbeaver_b200.desc import (QMCB_DMC, QMCB_IMPORTANCE_SAMPLING, QMCB_QF_UMRIGAR93_UNEQUAL,
                                 QMCB_UMRIGAR93_IMPORTANCE_SAMPLING, run_params)
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload,run_type,sampling", [
    ("dmc_6nuc_30e", QMCB_DMC, QMCB_IMPORTANCE_SAMPLING),
    ("vmc_multidet_12e", 0, QMCB_UMRIGAR93_IMPORTANCE_SAMPLING)])
def test_device_configs_match_oracle(tmp_path, workload, run_type, sampling):
    from oracle.evaluators import OracleEvaluator
    s = make_system(workload, seed=1)
    N, W, dt = s.n_electrons, 64, 0.01
    params = run_params(run_type=run_type, sampling=sampling, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=dt,
                        seed=5, rel_cutoff=0.0, energy_trial=-40.0, energy_estimated=-40.0)
    R0 = s.initial_positions(W, seed=2)
    f = QMCB200Functions(s, W, params)
    f.init_walkers(R0)
    path = str(tmp_path / "run.cfgs")
    first, n, freq = 1, 3 * N, N // 2
    tot = run_with_configs(f, path, first, n, frequency=freq)
    dump_steps = [k for k in range(first, first + n) if k % freq == 0]
    recs = read_configs(path, N)
    assert tot["records"] == len(recs) and len(recs) >= 2 * W * len(dump_steps) // 2
    t, o = recs[0::2], recs[1::2]
    assert np.allclose(t["weight"] + o["weight"], 1.0, rtol=0, atol=1e-15)
    assert np.all((t["weight"] >= 0) & (t["weight"] <= 1))
    assert all(np.count_nonzero(np.any(a != b, axis=1)) == 1 for a, b in zip(t["R"], o["R"]))
    orc = OracleEvaluator(s, qf_mod=QMCB_QF_UMRIGAR93_UNEQUAL, dt=dt)
    ws = orc.new_walkers(len(recs))
    orc.evaluate(ws, np.ascontiguousarray(recs["R"]), -1)
    res = orc.results(ws)
    ok = res["singular"] == 0
    assert ok.mean() > 0.9
    rel = lambda a, b: np.abs(a - b) / np.maximum(np.abs(b), 1.0)
    # the device carries these incrementally over up to 3N single-electron
    # updates: 1e-8 (laplacian) and 1e-9 relative
    assert np.max(rel(recs["D1"][ok], res["D_xx"][ok])) < 1e-8
    assert np.max(rel(recs["D2"][ok], orc.slater_grad(ws)[ok])) < 1e-9
    assert np.max(rel(recs["lnJ"][ok], res["U"][ok])) < 1e-10
    assert np.max(rel(recs["PE"][ok], res["potential"][ok])) < 1e-10
    # writing configurations does not change the chain
    g = QMCB200Functions(s, W, params)
    g.init_walkers(R0)
    g.run_steps(first, n)
    a, b = f.get_walkers(), g.get_walkers()
    assert np.array_equal(a["R"], b["R"]) and np.array_equal(a["weight"], b["weight"])
