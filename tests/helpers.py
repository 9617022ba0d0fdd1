"""Shared test helpers: golden cases, replay of evaluate sequences, tolerances."""
import glob
import os

import numpy as np

from qmcbeaver_b200.system import system_from_arrays

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))

# Per-call parity of the plain FP64 path against the reference: 1e-10 relative
# (psi ratio via log|psi|, drift, E_L).
PARITY_RTOL = 1e-10


def load_golden(name):
    d = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    sysd = {k[4:]: d[k] for k in d.files if k.startswith("sys_")}
    return system_from_arrays(sysd), d


def rel_err(a, b, floor=1.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def compare(out, ref, rtol, label="", mask=None, kappa=None):
    """Checks one evaluate call's outputs against reference outputs (walkers
    in `mask`, default all non-singular ones).  kappa: per-walker condition
    number of the determinant-weighted laplacian sum (several determinants);
    lap and E_L are checked at rtol * max(kappa, 1)."""
    ok = ref["singular"] == 0 if "singular" in ref else np.ones(len(ref["e_local"]), bool)
    if mask is not None:
        ok = ok & mask
    msgs = []
    amp = np.ones(len(ok)) if kappa is None else np.maximum(np.asarray(kappa, np.float64), 1.0)
    for k, floor in (("e_local", 1.0), ("lap", 1.0), ("potential", 1.0)):
        a, b = np.asarray(out[k], np.float64)[ok], np.asarray(ref[k], np.float64)[ok]
        s = amp[ok] if k != "potential" else np.ones(ok.sum())
        e = float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor) / s)) if a.size else 0.0
        if e > rtol:
            msgs.append(f"{k} {e:.3e}")
    # psi ratio: |d log psi| is the relative error of psi (absent from
    # references recorded on the reference's all-electron path, which leaves
    # the per-spin determinants unset)
    if "log_abs_psi" in ref:
        e = float(np.max(np.abs(out["log_abs_psi"][ok] - ref["log_abs_psi"][ok]))) if ok.any() else 0.0
        if e > rtol:
            msgs.append(f"log_abs_psi {e:.3e}")
    if "sign" in ref and not np.array_equal(out["sign"][ok], ref["sign"][ok]):
        msgs.append("sign")
    for k in ("grad", "mod_grad"):
        a, b = out[k][ok], ref[k][ok]
        scale = np.maximum(np.linalg.norm(b, axis=-1, keepdims=True), 1.0)
        e = float(np.max(np.abs(a - b) / scale)) if a.size else 0.0
        if e > rtol:
            msgs.append(f"{k} {e:.3e}")
    assert not msgs, f"{label}: " + ", ".join(msgs)


def replay(ev_eval, d, rtol, label, kappa=None):
    """Feeds the golden call sequence through ev_eval(which_e, R) -> outputs.
    kappa(which_e, R) -> per-walker laplacian-sum condition numbers (several
    determinants), or None."""
    for i, e in enumerate(d["whichE"]):
        out = ev_eval(int(e), d["R"][i])
        ref = {k: d[k][i] for k in ("log_abs_psi", "sign", "grad", "mod_grad", "lap", "e_local", "potential",
                                     "singular")}
        kap = kappa(int(e), d["R"][i]) if kappa is not None else None
        compare(out, ref, rtol, f"{label} call {i} whichE={e}", kappa=kap)


# Rounding differences between two FP64 implementations grow with the
# condition number of the Slater matrix carried through Sherman-Morrison
# updates (measured: about 1.1e-15 * cond).  The 1e-10 bar applies to walkers
# whose matrices stayed below COND_LIMIT; beyond it the bound is
# COND_SLOPE * cond (a walker that once exceeded the limit stays there).
COND_SLOPE = 2e-15
COND_LIMIT = 5e4
# Several determinants: every determinant's inverse is carried through its
# own Sherman-Morrison chain and the combined ratios take the worst of them
# (measured up to 2.2e-15 * cond once the determinant-mixing amplification
# kappa is divided out), so the bound doubles: 1e-10 up to cond 2.5e4, then
# 4e-15 * cond, each times kappa.
COND_SLOPE_MULTIDET = 4e-15
COND_LIMIT_MULTIDET = 2.5e4


def cond_bounds(system):
    """(slope, limit) of the condition-scaled parity bound for the system."""
    return (COND_SLOPE_MULTIDET, COND_LIMIT_MULTIDET) if system.n_det > 1 else (COND_SLOPE, COND_LIMIT)


def slater_conditions(orc, walkers, system):
    """Largest condition number over the Slater matrices (every determinant,
    both spins) of each walker."""
    c = np.zeros(len(walkers))
    for i, w in enumerate(walkers):
        for beta, n in ((0, system.n_alpha), (1, system.n_beta)):
            if n > 0:
                for det in range(system.n_det):
                    c[i] = max(c[i], np.linalg.cond(orc.inverse(w, beta, det)))
    return c


def place_near_nuclei(R, system, rng, radius=0.03):
    """Moves one electron of every walker to within `radius` bohr of a nucleus
    (inside every cusp-replacement radius of the systems tested), so the
    replacement branch is exercised; returns the electron index per walker."""
    W, N = R.shape[0], R.shape[1]
    es = np.zeros(W, int)
    for w in range(W):
        e = int(rng.integers(N))
        a = int(rng.integers(system.n_nuclei))
        v = rng.standard_normal(3)
        R[w, e] = system.coords[a] + radius * rng.random() * v / np.linalg.norm(v)
        es[w] = e
    return es


def oracle_sequence(s, W, qf, dt, sweeps, sigma, seed, slots_offset=0, min_good=0.2, precision=0, electrons=None,
                    rtol=PARITY_RTOL, slope_factor=1.0):
    """Full evaluation, then single-electron moves of `electrons` (default:
    `sweeps` sweeps of all) through the C ABI and the oracle on the same
    positions, compared call by call at the condition-scaled parity bound
    (rtol below the condition limit, slope_factor x the FP64 slope above)."""
    from oracle.evaluators import OracleEvaluator
    from qmcbeaver_b200.api import QMCB200Functions
    orc = OracleEvaluator(s, qf_mod=qf, dt=dt)
    f = QMCB200Functions(s, W + slots_offset, qf_modification=qf, dt=dt, precision=precision)
    slots = np.arange(W) + slots_offset
    ws = orc.new_walkers(W)
    R = s.initial_positions(W, seed=seed)
    rng = np.random.default_rng(seed + 1)
    N = s.n_electrons
    moved = list(electrons) if electrons is not None else [m % N for m in range(sweeps * N)]
    calls = [(-1, None)] + [(e, None) for e in moved]
    good = np.ones(W, bool)
    worst_cond = np.zeros(W)
    slope, limit = cond_bounds(s)
    for i, (e, _) in enumerate(calls):
        if e >= 0:
            R[:, e] += sigma * rng.standard_normal((W, 3))
        orc.evaluate(ws, R, e)
        ref = orc.results(ws)
        cond = slater_conditions(orc, ws, s)
        worst_cond = np.maximum(worst_cond, cond)
        good &= cond < limit
        out = f.evaluate(slots, R, e)
        kap = orc.kappa(ws)
        compare(out, ref, rtol, f"{s.name} call {i} whichE={e}", mask=good, kappa=kap)
        if (~good).any():
            # ill-conditioned Slater matrices: rounding differences of two
            # FP64 implementations grow as ~cond * 1e-15
            tol = max(rtol, slope_factor * slope * float(worst_cond[~good].max()))
            compare(out, ref, tol, f"{s.name} call {i} whichE={e} (cond {worst_cond[~good].max():.1e})", mask=~good,
                    kappa=kap)
    f.close()
    assert good.mean() >= min_good, f"only {good.sum()} of {W} walkers stayed well conditioned"
    return good.mean()
