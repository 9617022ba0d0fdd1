"""Shared checks for the fixtures made from the reference's own input files
(tests/golden/inputs/*.npz, written by tests/golden/make_inputs.py)."""
import glob
import os

import numpy as np

from helpers import GOLDEN_DIR, PARITY_RTOL, compare, cond_bounds, slater_conditions
from qmcbeaver_b200.system import system_from_arrays

INPUT_CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "inputs", "*.npz")))


def load_input_case(name):
    d = np.load(os.path.join(GOLDEN_DIR, "inputs", name + ".npz"))
    return system_from_arrays({k[4:]: d[k] for k in d.files if k.startswith("sys_")}), d


def replay_against_reference(s, d, evaluate, label):
    """Feeds the recorded calls through evaluate(which_e, R) and compares with
    the reference's outputs.  The oracle follows the same calls for each
    walker's Slater condition numbers and (several determinants) the
    laplacian-sum condition number kappa: the 1e-10 bar holds below the
    condition limit, the condition-scaled bound above it, and lap / E_L are
    checked relative to the size of the terms E_L = -lap/2 + V cancels."""
    from oracle.evaluators import OracleEvaluator
    W = d["R"].shape[1]
    orc = OracleEvaluator(s, qf_mod=int(d["qf_mod"]), dt=float(d["dt"]))
    ws = orc.new_walkers(W)
    slope, limit = cond_bounds(s)
    worst = np.zeros(W)
    for i, e in enumerate(d["whichE"]):
        e = int(e)
        R = d["R"][i]
        out = evaluate(e, R)
        orc.evaluate(ws, R, e)
        worst = np.maximum(worst, slater_conditions(orc, ws, s))
        ref = {k: d[k][i] for k in ("log_abs_psi", "sign", "grad", "mod_grad", "lap", "e_local", "potential",
                                     "singular") if k in d.files}
        amp = (np.abs(ref["lap"]) / 2 + np.abs(ref["potential"])) / np.maximum(np.abs(ref["e_local"]), 1.0)
        if s.n_det > 1:
            amp = amp * np.maximum(orc.kappa(ws), 1.0)
        good = worst < limit
        compare(out, ref, PARITY_RTOL, f"{label} call {i} whichE={e}", mask=good, kappa=amp)
        if (~good).any():
            tol = max(PARITY_RTOL, slope * float(worst[~good].max()))
            compare(out, ref, tol, f"{label} call {i} whichE={e} (cond {worst[~good].max():.1e})", mask=~good,
                    kappa=amp)
    return float(worst.max())
