"""Generates tests/golden/inputs/*.npz: the reference QMcBeaver CPU code
(oracle/_ref/libqmcref.so, driven through QMCSCFJastrow::evaluate) on some
of its OWN input files -- real molecules with the features those inputs
switch on: electron-nucleus cusp replacement, Cambridge three-body
Jastrows, several determinants, Cambridge2 / FixedCuspPade two-body
functions.

Each fixture stores the system as this repository's reader builds it from
the input (qmcbeaver_b200.ckmf; system arrays, not the input text), walker
positions and, per call of a sequence -- a full evaluation, then
single-electron moves with rollbacks (QMcBeaver/src/QMCWalker.cpp:254-266)
and an electron placed near a nucleus every third move; full evaluations
at perturbed positions only, for the inputs of FULL_ONLY -- the reference's
log|psi|, sign, grad psi / psi, modified drift, lap psi / psi, E_L,
potentials and singular flag.

Run:  python tests/golden/make_inputs.py      (needs the reference tree)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "inputs")
sys.path.insert(0, ROOT)
from oracle.evaluators import REFERENCE_TREE as REF_INPUTS  # noqa: E402

CASES = {
    # name: (input, walkers, moves)
    "h2o": ("examples/h2o.ckmf", 4, 30),            # cusps + three-body
    "oepi": ("test/oepi.ckmf", 4, 36),              # cusps + three-body
    "chkpnt": ("test/chkpnt.ckmf", 4, 24),          # 2 determinants, cusps + three-body
    "det": ("test/det.ckmf", 3, 30),                # 10 determinants, 480 basis functions, cusps + three-body
    "be_mcscf": ("examples/BeMCSCF.ckmf", 4, 16),   # 10 determinants, cusps
    "ne0p": ("examples/ne0P.ckmf", 4, 24),          # plain Slater-Jastrow
    "annulene": ("examples/10_Annulene-heart-DZd_CCSDT.HF_CC-PVDZ.DMC.ckmf", 3, 40),  # 70 electrons, cusps
    # 28 atoms, 76 electrons, 516 basis functions, FixedCuspPade, cusps: full
    # evaluations only -- the reference's one-electron path copies derivative
    # rows with the full orbital-row width (QMcBeaver/src/QMCWalkerData.cpp:80-93,
    # QMcBeaver/include/Array2D.h:986), wrong when more orbitals are listed
    # than occupied (516 listed, 76 per spin occupied)
    "hmx": ("test/hmx.ckmf", 3, 6),
}
FULL_ONLY = {"hmx"}
QF, DT = 2, 0.01


def run_case(name: str) -> None:
    from qmcbeaver_b200.ckmf import read_ckmf
    from qmcbeaver_b200.system import system_to_arrays
    from oracle.evaluators import ReferenceEvaluator
    rel, W, moves = CASES[name]
    path = os.path.join(REF_INPUTS, rel)
    text = open(path).read()
    s = read_ckmf(path).to_system()
    full_only = name in FULL_ONLY
    ref = ReferenceEvaluator(s, qf_mod=QF, dt=DT, ckmf_text=text, one_e_per_iter=0 if full_only else 1)
    rng = np.random.default_rng(7)
    R = s.initial_positions(W, seed=13)
    N = s.n_electrons
    ws = ref.new_walkers(W)
    whichE, Rseq, outs = [], [], []

    def call(e, Rnow):
        ref.evaluate(ws, Rnow, e)
        whichE.append(e)
        Rseq.append(Rnow.copy())
        outs.append(ref.results(ws))

    call(-1, R)
    prev = None
    for m in range(moves if full_only else 0):
        R = R + 0.15 * rng.standard_normal(R.shape)
        call(-1, R)
    for m in range(0 if full_only else moves):
        e = (m * 5) % N  # both spins, not in order
        if m % 6 == 5 and prev is not None:
            pe, pr = prev
            R[:, pe] = pr
            call(pe, R)
            prev = None
            continue
        old = R[:, e].copy()
        if m % 3 == 0:
            R[:, e] = s.coords[rng.integers(s.n_nuclei, size=W)] + 0.03 * rng.standard_normal((W, 3))
        else:
            R[:, e] = R[:, e] + 0.2 * rng.standard_normal((W, 3))
        call(e, R)
        prev = (e, old)
    keys = ["log_abs_psi", "sign", "grad", "mod_grad", "lap", "e_local", "potential", "ne", "ee", "singular"]
    if full_only:
        # the all-electron path leaves the per-spin determinants that log|psi|
        # and the sign are read from unset
        keys = [k for k in keys if k not in ("log_abs_psi", "sign")]
    data = {k: np.stack([o[k] for o in outs]) for k in keys}
    data.update(whichE=np.array(whichE), R=np.stack(Rseq), qf_mod=np.array(QF), dt=np.array(DT),
                source=np.array(rel))
    data.update({"sys_" + k: v for k, v in system_to_arrays(s).items()})
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
    print(name, rel, "calls", len(whichE), "walkers", W, "N", N, "singular", int(data["singular"].sum()))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        run_case(sys.argv[1])
    else:
        for c in CASES:  # one process per case: the reference keeps its input in globals
            subprocess.check_call([sys.executable, os.path.abspath(__file__), c])
