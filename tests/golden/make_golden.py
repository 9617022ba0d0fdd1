"""Generates the golden vectors in tests/golden/*.npz from the reference
QMcBeaver CPU code itself (built from its sources by oracle/Makefile into
oracle/_ref/libqmcref.so and driven through QMCSCFJastrow::evaluate).

Each case: a synthetic system, walker positions, then a sequence of
evaluate calls -- a full evaluation (whichE = -1) followed by single-electron
moves (whichE = e, Sherman-Morrison path), including moves that put an
electron back where it was (the reference's rejection path,
QMcBeaver/src/QMCWalker.cpp:254-266).  Recorded per call: log|psi|, sign,
grad(psi)/psi, modified quantum force, lap(psi)/psi, E_L, potentials,
singular flag.

Run:  python tests/golden/make_golden.py      (needs the reference tree)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = {
    # name: (workload, qf_mod, dt, walkers, moves, step sigma, revert every)
    "water_vmc": ("vmc_water_10e", 0, 0.09, 8, 24, 0.3, 5),
    "dmc30_unequal": ("dmc_6nuc_30e", 2, 0.01, 4, 34, 0.15, 7),
    "dmc30_equal": ("dmc_6nuc_30e", 1, 0.01, 2, 8, 0.15, 0),
    # Cambridge2 two-body Jastrow with C = 2 and C = 3 and an inactive function
    "cambridge2_vmc": ("vmc_cambridge2_16e", 2, 0.01, 6, 40, 0.2, 6),
    # twelve determinants (single excitations into every virtual orbital of
    # both spins, doubles)
    "multidet_vmc": ("vmc_multidet_12e", 2, 0.01, 6, 40, 0.2, 6),
    # electron-nucleus cusp replacement, electrons placed inside the
    # replacement radii every third move
    "cusp_dmc30": ("dmc_6nuc_30e", 2, 0.01, 4, 40, 0.15, 7),
    # Cambridge2 two-body + three-body Jastrow with cusp replacement (the
    # combination the reference's own test inputs use)
    "threebody_cusp_vmc": ("vmc_threebody_16e", 2, 0.01, 6, 40, 0.2, 6),
    # the 100-electron / 400-function workload: moves of both spins (electron
    # 9 m mod 100), the walkers kept among 256 candidates whose Slater matrices
    # stay below condition 5e4 over the whole sequence (random 50 x 50
    # orbital matrices are mostly worse conditioned, and two FP64
    # implementations then differ by ~1e-15 cond)
    "c100_dmc": ("mixed_20nuc_100e", 2, 0.01, 6, 16, 0.05, 5),
}
CUSP_CASES = {"cusp_dmc30", "threebody_cusp_vmc"}
ELECTRON_STRIDE = {"c100_dmc": 9}
SYSTEM_SEED = {"c100_dmc": 2}  # the seed-2 molecule has the best-conditioned walkers
WELL_CONDITIONED = {"c100_dmc": (256, 5e4)}


def move_plan(N, moves, revert, stride):
    """(electron, revert?) of each call after the full evaluation."""
    plan, prev = [], None
    for m in range(moves):
        if revert and m % revert == revert - 1 and prev is not None:
            plan.append((prev, True))
            prev = None
            continue
        e = (m * stride) % N
        plan.append((e, False))
        prev = e
    return plan


def pick_walkers(s, qf, dt, W, moves, sigma, revert, stride, candidates, limit):
    """Indices of W of `candidates` walkers whose Slater matrices stay below
    condition `limit` through the move plan (checked with the oracle)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import slater_conditions
    from oracle.evaluators import OracleEvaluator
    orc = OracleEvaluator(s, qf_mod=qf, dt=dt)
    R = s.initial_positions(candidates, seed=11)
    rng = np.random.default_rng(2024)
    disp = sigma * rng.standard_normal((moves, candidates, 3))
    ws = orc.new_walkers(candidates)
    orc.evaluate(ws, R, -1)
    worst = slater_conditions(orc, ws, s)
    last = {}
    for i, (e, back) in enumerate(move_plan(s.n_electrons, moves, revert, stride)):
        if back:
            R[:, e] = last[e]
        else:
            last[e] = R[:, e].copy()
            R[:, e] += disp[i]
        orc.evaluate(ws, R, e)
        worst = np.maximum(worst, slater_conditions(orc, ws, s))
    good = np.argsort(worst)[:W]
    assert worst[good].max() < limit, worst[good]
    return good, disp


def run_case(name: str) -> None:
    import dataclasses
    from qmcbeaver_b200.system import make_system, system_to_arrays
    from oracle.evaluators import ReferenceEvaluator
    workload, qf, dt, W, moves, sigma, revert = CASES[name]
    s = make_system(workload, seed=SYSTEM_SEED.get(name, 1))
    cusp = name in CUSP_CASES
    if cusp:
        s = dataclasses.replace(s, replace_cusps=True)
    stride = ELECTRON_STRIDE.get(name, 1)
    if name in WELL_CONDITIONED:
        good, disp = pick_walkers(s, qf, dt, W, moves, sigma, revert, stride, *WELL_CONDITIONED[name])
        R = s.initial_positions(WELL_CONDITIONED[name][0], seed=11)[good]
        ref = ReferenceEvaluator(s, qf_mod=qf, dt=dt)
        N = s.n_electrons
        ws = ref.new_walkers(W)
        whichE, Rseq, outs = [], [], []

        def call(e, Rnow):
            ref.evaluate(ws, Rnow, e)
            whichE.append(e)
            Rseq.append(Rnow.copy())
            outs.append(ref.results(ws))

        call(-1, R)
        last = {}
        for i, (e, back) in enumerate(move_plan(N, moves, revert, stride)):
            if back:
                R[:, e] = last[e]
            else:
                last[e] = R[:, e].copy()
                R[:, e] += disp[i][good]
            call(e, R)
        save(name, s, qf, dt, W, N, whichE, Rseq, outs)
        return
    ref = ReferenceEvaluator(s, qf_mod=qf, dt=dt)
    rng = np.random.default_rng(2024)
    R = s.initial_positions(W, seed=11)
    if cusp:
        # one electron of each walker within 0.03 bohr of a nucleus
        for w in range(W):
            R[w, int(rng.integers(s.n_electrons))] = s.coords[int(rng.integers(s.n_nuclei))] + 0.03 * rng.random() * \
                rng.standard_normal(3) / np.sqrt(3.0)
    N = s.n_electrons
    ws = ref.new_walkers(W)
    whichE, Rseq, outs = [], [], []

    def call(e, Rnow):
        ref.evaluate(ws, Rnow, e)
        o = ref.results(ws)
        whichE.append(e)
        Rseq.append(Rnow.copy())
        outs.append(o)

    call(-1, R)
    prev = None
    for m in range(moves):
        e = m % N
        if revert and m % revert == revert - 1 and prev is not None:
            # put the last moved electron back (the reference's rollback)
            pe, pr = prev
            R[:, pe] = pr
            call(pe, R)
            prev = None
            continue
        old = R[:, e].copy()
        if cusp and m % 3 == 0:
            R[:, e] = s.coords[int(rng.integers(s.n_nuclei))] + 0.02 * rng.standard_normal((W, 3))
        else:
            R[:, e] = R[:, e] + sigma * rng.standard_normal((W, 3))
        call(e, R)
        prev = (e, old)
    save(name, s, qf, dt, W, N, whichE, Rseq, outs)


def save(name, s, qf, dt, W, N, whichE, Rseq, outs):
    from qmcbeaver_b200.system import system_to_arrays
    keys = ["log_abs_psi", "sign", "grad", "mod_grad", "lap", "e_local", "potential", "ne", "ee", "singular"]
    data = {k: np.stack([o[k] for o in outs]) for k in keys}
    data.update(whichE=np.array(whichE), R=np.stack(Rseq), qf_mod=np.array(qf), dt=np.array(dt))
    data.update({"sys_" + k: v for k, v in system_to_arrays(s).items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
    print(name, "calls", len(whichE), "walkers", W, "N", N)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        run_case(sys.argv[1])
    else:
        for c in CASES:  # one process per case: the reference keeps its input in globals
            subprocess.check_call([sys.executable, os.path.abspath(__file__), c])
