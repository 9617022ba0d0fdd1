"""Generates tests/golden/moves/*.npz: single-electron moves made by the
reference QMcBeaver's own QMCWalker (built from its sources by
oracle/Makefile into oracle/_ref/libqmcref.so, entry point ref_walker_move)
with sampling_method umrigar93_importance_sampling.

Per move: the walker's positions R0, the proposed positions R1, the moved
electron, the modified drift of the original and the trial walker, and the
reference's forward / reverse Green's functions (QMcBeaver/src/QMCWalker.cpp:
179-198, 400-586, 783-926).  Starting positions are the system's initial
walkers with, every other move, one electron placed near a nucleus so that
both the Gaussian and the exponential branch of the move appear.

Run:  python tests/golden/make_moves.py      (needs the reference tree)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "moves")
sys.path.insert(0, ROOT)

CASES = {
    # name: (workload, qf_mod, dt, moves)
    "umrigar93_water": ("vmc_water_10e", 0, 0.09, 40),
    "umrigar93_dmc30": ("dmc_6nuc_30e", 2, 0.01, 40),
}


def run_case(name: str) -> None:
    from qmcbeaver_b200.system import make_system, system_to_arrays
    from oracle.evaluators import ReferenceEvaluator
    workload, qf, dt, moves = CASES[name]
    s = make_system(workload, seed=1)
    ref = ReferenceEvaluator(s, qf_mod=qf, dt=dt,
                             extra_flags={"sampling_method": "umrigar93_importance_sampling"})
    rng = np.random.default_rng(77)
    N = s.n_electrons
    Rs = s.initial_positions(moves, seed=5)
    rec = {k: [] for k in ("R0", "R1", "mg0", "mg1", "gf", "whichE")}
    for m in range(moves):
        R0 = Rs[m].copy()
        if m % 2 == 1:
            R0[m % N] = s.coords[int(rng.integers(s.n_nuclei))] + 0.05 * rng.standard_normal(3)
        o = ref.walker_move(R0, iteration=m + 1, seed=-(1000 + m))
        rec["R0"].append(R0)
        rec["R1"].append(o["R"])
        rec["mg0"].append(o["mg0"])
        rec["mg1"].append(o["mg1"])
        rec["gf"].append(o["gf"])
        rec["whichE"].append(o["whichE"])
    data = {k: np.array(v) for k, v in rec.items()}
    data.update(qf_mod=np.array(qf), dt=np.array(dt))
    data.update({"sys_" + k: v for k, v in system_to_arrays(s).items()})
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
    print(name, "moves", moves, "N", N)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        run_case(sys.argv[1])
    else:
        for c in CASES:  # one process per case: the reference keeps its input in globals
            subprocess.check_call([sys.executable, os.path.abspath(__file__), c])
