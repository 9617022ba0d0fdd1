"""The library inside the reference program: oracle/_ref/QMcBeaver_b200.x is
the unmodified QMcBeaver driver (QMCRun, QMCWalker, its random numbers,
branching and statistics) whose QMCFunctions come from libqmcb200
(oracle/dropin_functions.cpp, selected with QMCB_DROPIN=1).  On the same
input and seed it must reproduce the stock program's energy: the same random
draws and evaluator values equal to ~1e-10 give the same Markov chain."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STOCK = os.path.join(ROOT, "oracle", "_ref", "QMcBeaver.x")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "QMcBeaver_b200.x")
_ENERGY = re.compile(r"-+ Energy -+\s*\n\s*([-0-9.eE+]+)\s*\+/-\s*([0-9.eE+-]+)")


def _run(exe, ckmf, dropin):
    env = dict(os.environ)
    env.pop("QMCB_DROPIN", None)
    if dropin:
        env["QMCB_DROPIN"] = "1"
    d = os.path.dirname(ckmf)
    p = subprocess.run([exe, os.path.basename(ckmf)], cwd=d, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    m = _ENERGY.search(p.stdout)
    assert m, "no energy in the output"
    return float(m.group(1)), float(m.group(2)), p.stdout + p.stderr


@pytest.mark.skipif(not (os.path.exists(STOCK) and os.path.exists(DROPIN)), reason="reference build absent")
@pytest.mark.parametrize("case", ["vmc_water_10e", "dmc_6nuc_30e"])
def test_dropin_reproduces_reference_program(case):
    from oracle import refrun
    s = make_system(case, seed=1)
    # VMC with the reference's default sampling on the water-like system;
    # DMC (drift-diffusion moves, Umrigar93 energy modification, nonunit
    # branching) on the 30-electron one; all-electron moves, 20 walkers
    flags = dict(refrun.RUN_FLAGS["dmc"]) if case.startswith("dmc") else {
        "run_type": "variational", "sampling_method": "umrigar93_importance_sampling",
        "QF_modification_type": "umrigar93_unequalelectrons"}
    flags.update({"dt": 0.01, "number_of_walkers": 20, "max_time_steps": 300, "equilibration_steps": 50,
                  "one_e_per_iter": 0, "walkers_per_pass": 20, "iseed": -7,
                  "energy": -55.0 if case.startswith("dmc") else -75.0, "output_interval": 10 ** 6})
    res = {}
    for dropin, exe in ((False, STOCK), (True, DROPIN)):
        d = tempfile.mkdtemp(prefix="qmcdropin_")
        path = os.path.join(d, "run.ckmf")
        s.to_ckmf(path, flags)
        res[dropin] = _run(exe, path, dropin)
    (e0, s0, _), (e1, s1, log1) = res[False], res[True]
    assert "QMCB200Functions: evaluate through" in log1  # the library did the evaluations
    assert np.isfinite(e1) and s1 > 0
    print(f"{case}: stock {e0} +/- {s0}, drop-in {e1} +/- {s1}")
    # same chain: the printed energies agree far inside the statistical error
    assert abs(e1 - e0) <= 1e-3 * s0 + 1e-9 * abs(e0), (e0, s0, e1, s1)
