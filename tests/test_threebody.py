"""Cambridge three-body Jastrow: the coefficient tables (dependency matrix of
the input parameters) against the reference's own, the constraints, the
ckmf writer / reader, and the oracle against the reference call for call
on the reference's inputs and on synthetic systems."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle.evaluators import REFERENCE_TREE, reference_available
from qmcbeaver_b200.ckmf import read_ckmf
from qmcbeaver_b200.system import make_system
from qmcbeaver_b200.threebody import ThreeBody, constraint_matrix, dependency_matrix, file_order, random_three_body

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_INPUTS = REFERENCE_TREE
HAVE_REF = reference_available() and os.path.isdir(REF_INPUTS)


@pytest.mark.parametrize("nen,nee", [(3, 3), (4, 4), (5, 5), (4, 3), (3, 5)])
def test_file_order_covers_every_coefficient_once(nen, nee):
    fo = file_order(nen, nee)
    assert sorted(fo) == list(range(nen * nen * nee))


@pytest.mark.parametrize("nen,nee,C,rep", [(3, 3, 3, (True, True)), (4, 4, 3, (True, True)), (4, 4, 2, (False, False)),
                                           (5, 5, 3, (True, False)), (4, 3, 3, (False, False))])
def test_dependencies_impose_the_constraints(nen, nee, C, rep):
    rng = np.random.default_rng(nen * 10 + nee)
    if nen != nee and all(rep):
        pytest.skip("the elimination path needs NeN == Nee")
    tb = random_three_body(rng, nen, nee, C, 0.3, 1.0, *rep)
    A = constraint_matrix(nen, nee, C, *rep)
    assert np.max(np.abs(A @ tb.coeffs)) < 1e-10 * max(1.0, np.abs(tb.coeffs).max())
    # a consistent input is its own image: writing the coefficients out and
    # reading them back gives them again
    back = ThreeBody.from_input(tb.input_parameters(), nen, nee, C, 0.3, *rep)
    np.testing.assert_allclose(back.coeffs, tb.coeffs, rtol=1e-12, atol=1e-13)
    P, free = dependency_matrix(nen, nee, C, *rep)
    assert np.allclose(P[free][:, free], np.eye(free.sum()))


def test_three_body_term_derivatives():
    # gradients and laplacian of the direct formulas against finite differences
    rng = np.random.default_rng(5)
    tb = random_three_body(rng, 4, 4, 3, 0.3, 1.0)
    r1, r2 = np.array([0.4, -0.3, 0.8]), np.array([-0.6, 0.5, 0.2])
    U, g1, g2, lap = tb.evaluate(r1, r2)
    h = 1e-5
    fd1, fd2, fl = np.zeros(3), np.zeros(3), 0.0
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        up1, dn1 = tb.evaluate(r1 + e, r2)[0], tb.evaluate(r1 - e, r2)[0]
        up2, dn2 = tb.evaluate(r1, r2 + e)[0], tb.evaluate(r1, r2 - e)[0]
        fd1[k], fd2[k] = (up1 - dn1) / (2 * h), (up2 - dn2) / (2 * h)
        fl += (up1 - 2 * U + dn1 + up2 - 2 * U + dn2) / h ** 2
    np.testing.assert_allclose(g1, fd1, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(g2, fd2, rtol=1e-6, atol=1e-9)
    assert lap == pytest.approx(fl, rel=1e-4, abs=1e-6)
    assert tb.evaluate(r1 * 20, r2)[0] == 0.0   # outside the cutoff


def test_three_body_round_trips_through_ckmf(tmp_path):
    s = make_system("vmc_threebody_16e", seed=1)
    assert s.three_body
    s.to_ckmf(str(tmp_path / "t.ckmf"))
    t = read_ckmf(str(tmp_path / "t.ckmf")).to_system()
    for l, fs in s.three_body.items():
        for a, b in zip(fs, t.three_body[l]):
            assert (a.nen, a.nee, a.C, a.cutoff) == (b.nen, b.nee, b.C, b.cutoff)
            np.testing.assert_allclose(b.coeffs, a.coeffs, rtol=1e-12, atol=1e-14)
    assert not read_ckmf(str(tmp_path / "t.ckmf")).to_system(three_body=False).three_body


_COEF = r"""
import sys, ctypes as C, numpy as np
sys.path.insert(0, {root!r})
from qmcbeaver_b200.ckmf import read_ckmf
from oracle.evaluators import ReferenceEvaluator
path = {path!r}
s = read_ckmf(path).to_system(replace_cusps=False)
ref = ReferenceEvaluator(s, qf_mod=2, dt=0.01, ckmf_text=open(path).read())
L = ref.lib
L.ref_three_body.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int]
buf = np.zeros(4096)
worst, n = 0.0, 0
for j, lab in enumerate(dict.fromkeys(s.labels)):
    mine = s.three_body.get(lab, (None, None, None))
    for kind in range(3):
        k = L.ref_three_body(kind, j, buf.ctypes.data_as(C.c_void_p), 4096)
        if k <= 0:
            assert mine[kind] is None
            continue
        m = mine[kind]
        assert (m.nen, m.nee, m.C, m.cutoff) == (int(buf[0]), int(buf[1]), int(buf[2]), buf[3])
        rc = buf[5:k]
        worst = max(worst, float(np.max(np.abs(rc - m.coeffs)) / max(np.abs(rc).max(), 1e-300)))
        n += 1
print("RESULT", worst, n)
"""

_EVAL = r"""
import sys, numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {root!r} + "/tests")
from qmcbeaver_b200.ckmf import read_ckmf
from qmcbeaver_b200.system import make_system
from oracle.evaluators import OracleEvaluator, ReferenceEvaluator
from helpers import place_near_nuclei
src = {src!r}
if src.startswith("workload:"):
    s = make_system(src[9:], seed=2)
    text = None
else:
    s = read_ckmf(src).to_system()
    text = open(src).read()
assert s.three_body
ref = ReferenceEvaluator(s, qf_mod=2, dt=0.01, ckmf_text=text)
orc = OracleEvaluator(s, qf_mod=2, dt=0.01)
W = 4
rng = np.random.default_rng(3)
R = s.initial_positions(W, seed=5, sigma=0.7)
place_near_nuclei(R, s, rng)
wr, wo = ref.new_walkers(W), orc.new_walkers(W)
worst = 0.0
for step in range(-1, min(3 * s.n_electrons, 60)):
    e = -1 if step < 0 else step % s.n_electrons
    if e >= 0:
        R[:, e] += 0.2 * rng.standard_normal((W, 3))
    ref.evaluate(wr, R, e); orc.evaluate(wo, R, e)
    a, b = ref.results(wr), orc.results(wo)
    assert np.array_equal(a["sign"], b["sign"]) and not a["singular"].any()
    for k in ("e_local", "lap", "potential", "log_abs_psi", "grad", "mod_grad"):
        d = np.abs(a[k] - b[k]) / np.maximum(np.abs(a[k]), 1.0)
        worst = max(worst, float(d.max()))
print("RESULT", worst, 0)
"""

_INPUTS = ["test/oepi.ckmf", "test/he.ckmf", "test/diff.ckmf", "examples/h2o.ckmf", "examples/ne4.ckmf",
           "test/det.ckmf", "test/chkpnt.ckmf"]


def _run(code):
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("RESULT")][0].split()
    return float(line[1]), int(line[2])


@pytest.mark.skipif(not HAVE_REF, reason="reference tree / build not present")
@pytest.mark.parametrize("rel", _INPUTS)
def test_coefficients_equal_the_references(rel):
    # the same elimination in another order: equal up to its rounding
    worst, n = _run(_COEF.format(root=ROOT, path=os.path.join(REF_INPUTS, rel)))
    assert n > 0
    assert worst < 1e-11, worst


# the reference's inputs with everything they switch on: cusp replacement,
# Cambridge2 two-body, three-body, and (det, chkpnt) several determinants
@pytest.mark.skipif(not HAVE_REF, reason="reference tree / build not present")
@pytest.mark.parametrize("src", [os.path.join(REF_INPUTS, r) for r in _INPUTS] +
                         ["workload:vmc_threebody_16e"])
def test_oracle_matches_reference_with_three_body(src):
    worst, _ = _run(_EVAL.format(root=ROOT, src=src))
    assert worst < 1e-10, worst
