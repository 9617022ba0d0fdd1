"""Electron-nucleus cusp replacement (replace_electron_nucleus_cusps): the
library's fit against the reference's own fitted records, bit for bit; the
matching conditions of the fitted functions; and the oracle against the
reference call for call with the replacement on and electrons placed inside
the replacement radii."""
import dataclasses
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle.evaluators import REFERENCE_TREE, reference_available
from qmcbeaver_b200.api import fit_cusps
from qmcbeaver_b200.system import make_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_INPUTS = REFERENCE_TREE
HAVE_REF = reference_available() and os.path.isdir(REF_INPUTS)

_SYSTEM = r"""
import sys, dataclasses, numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {root!r} + "/tests")
from qmcbeaver_b200.ckmf import read_ckmf
from qmcbeaver_b200.system import make_system
from oracle.evaluators import OracleEvaluator, ReferenceEvaluator
src = {src!r}
if src.startswith("workload:"):
    s = dataclasses.replace(make_system(src[9:], seed=2), replace_cusps=True)
    text = None
else:
    s = read_ckmf(src).to_system(replace_cusps=True, three_body=False)
    text = open(src).read()
ref = ReferenceEvaluator(s, qf_mod=2, dt=0.01, ckmf_text=text)
"""

_FIT = _SYSTEM + r"""
from qmcbeaver_b200.api import fit_cusps
mine = fit_cusps(s)
worst, fitted = 0.0, 0
for beta in (0, 1):
    if (s.n_beta if beta else s.n_alpha) == 0:
        continue
    r = ref.cusp_params(beta)
    fitted += int((r[..., 0] > 0).sum())
    worst = max(worst, float(np.max(np.abs(r - mine[beta]))))
print("RESULT", worst, fitted)
"""

_EVAL = _SYSTEM + r"""
from helpers import place_near_nuclei
orc = OracleEvaluator(s, qf_mod=2, dt=0.01)
W = 4
rng = np.random.default_rng(3)
R = s.initial_positions(W, seed=5)
place_near_nuclei(R, s, rng)
wr, wo = ref.new_walkers(W), orc.new_walkers(W)
worst = 0.0
for step in range(-1, min(3 * s.n_electrons, 60)):
    e = -1 if step < 0 else step % s.n_electrons
    if e >= 0:
        if step % 3 == 0:
            a = int(rng.integers(s.n_nuclei))
            R[:, e] = s.coords[a] + 0.03 * rng.standard_normal((W, 3))
        else:
            R[:, e] += 0.2 * rng.standard_normal((W, 3))
    ref.evaluate(wr, R, e); orc.evaluate(wo, R, e)
    a, b = ref.results(wr), orc.results(wo)
    assert np.array_equal(a["sign"], b["sign"]) and not a["singular"].any()
    for k in ("e_local", "lap", "potential", "log_abs_psi", "grad", "mod_grad"):
        d = np.abs(a[k] - b[k]) / np.maximum(np.abs(a[k]), 1.0)
        worst = max(worst, float(d.max()))
print("RESULT", worst, 0)
"""

_CASES = ["test/oepi.ckmf", "test/he.ckmf", "examples/h2o.ckmf", "examples/ne0.ckmf", "test/det.ckmf",
          "examples/Kr2-MSV-441.ckmf", "test/hmx.ckmf", "workload:vmc_water_10e", "workload:dmc_6nuc_30e",
          "workload:vmc_multidet_12e"]


def _run(code):
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("RESULT")][0].split()
    return float(line[1]), int(line[2])


def _src(case):
    return case if case.startswith("workload:") else os.path.join(REF_INPUTS, case)


@pytest.mark.skipif(not HAVE_REF, reason="reference tree / build not present")
@pytest.mark.parametrize("case", _CASES)
def test_fit_equals_reference_fit(case):
    worst, fitted = _run(_FIT.format(root=ROOT, src=_src(case)))
    assert fitted > 0
    assert worst == 0.0, worst


# HMX and Kr2 are left out of the call-for-call check: the reference's
# one-electron path needs every listed orbital occupied (HMX) and its Kr2
# walkers are singular to working precision (see test_ckmf.py)
@pytest.mark.skipif(not HAVE_REF, reason="reference tree / build not present")
@pytest.mark.parametrize("case", [c for c in _CASES if "hmx" not in c and "Kr2" not in c])
def test_oracle_matches_reference_with_cusp_replacement(case):
    worst, _ = _run(_EVAL.format(root=ROOT, src=_src(case)))
    assert worst < 1e-11, worst


def _orig_s(co, ex, r):
    """The s part of one orbital at one nucleus and its first two radial derivatives."""
    t = co * np.exp(-ex * r * r)
    return t.sum(), (-2 * ex * r * t).sum(), (2 * ex * (2 * ex * r * r - 1) * t).sum()


@pytest.mark.parametrize("workload", ["vmc_water_10e", "dmc_6nuc_30e", "mixed_20nuc_100e"])
def test_fitted_functions_match_the_orbital_at_rc(workload):
    # C + sgn0 exp(alpha(r)) meets the s part with value, first and second
    # derivative at rc (the matching conditions x1..x3 of
    # QMCElectronNucleusCuspParameters::fitReplacementOrbital)
    s = dataclasses.replace(make_system(workload, seed=1), replace_cusps=True)
    recs, _ = fit_cusps(s)
    mo = s.mo_alpha()
    checked = 0
    k0 = 0
    for i, fs in enumerate(s.basis):
        sfun = [(k0 + j, f) for j, f in enumerate(fs) if f.powers == (0, 0, 0)]
        k0 += len(fs)
        for o in range(mo.shape[0]):
            rc, sg, C, *al = recs[i, o]
            if rc <= 0:
                continue
            co = np.concatenate([f.coefficients * mo[o, k] for k, f in sfun])
            ex = np.concatenate([f.exponents for _, f in sfun])
            v, d1, d2 = _orig_s(co, ex, rc)
            p = np.polynomial.Polynomial(al)
            e = sg * np.exp(p(rc))
            dp, d2p = p.deriv()(rc), p.deriv(2)(rc)
            np.testing.assert_allclose(C + e, v, rtol=1e-9, atol=1e-12)
            np.testing.assert_allclose(e * dp, d1, rtol=1e-7, atol=1e-10)
            np.testing.assert_allclose(e * (d2p + dp * dp), d2, rtol=1e-6, atol=1e-9)
            checked += 1
    assert checked > 0


def test_cusp_flag_round_trips_through_ckmf(tmp_path):
    from qmcbeaver_b200.ckmf import read_ckmf
    s = dataclasses.replace(make_system("vmc_water_10e", seed=1), replace_cusps=True)
    s.to_ckmf(str(tmp_path / "c.ckmf"))
    assert read_ckmf(str(tmp_path / "c.ckmf")).to_system().replace_cusps
    s2 = dataclasses.replace(s, replace_cusps=False)
    s2.to_ckmf(str(tmp_path / "d.ckmf"))
    assert not read_ckmf(str(tmp_path / "d.ckmf")).to_system().replace_cusps
