"""Times the reference QMcBeaver CPU program (oracle/_ref/QMcBeaver.x, built
from the reference's own sources) on a synthetic workload -- test and CPU-baseline
infrastructure: used only by bench.py's reference arm and cpu_baseline.

Runs P independent processes at once (the reference's manager_worker MPI
mode is exactly independent walker populations plus a reduce), each on its
own walker sample and seed, and reads the reference's own timer table:
"Entire Step" is microseconds per walker-move averaged over n walker-moves
(QMcBeaver/src/QMCManager.cpp:1799-1855 prints it).
"""
from __future__ import annotations

import os
import re
import subprocess
import tempfile
import time
from typing import Dict, Optional

HERE = os.path.dirname(os.path.abspath(__file__))
REF_EXE = os.path.join(HERE, "_ref", "QMcBeaver.x")

_ENTIRE = re.compile(r"Entire Step:\s*\d+\s*\(\s*avg\s*=\s*([0-9.eE+-]+)\s*us,\s*n=\s*(\d+)\)")

RUN_FLAGS = {
    "dmc": {"run_type": "diffusion", "sampling_method": "importance_sampling",
            "QF_modification_type": "umrigar93_unequalelectrons", "energy_modification_type": "umrigar93",
            "walker_reweighting_method": "umrigar93_probability_weighted",
            "branching_method": "nonunit_weight_branching", "population_control_parameter": 100.0},
    "vmc_drift": {"run_type": "variational", "sampling_method": "importance_sampling",
                  "QF_modification_type": "umrigar93_unequalelectrons"},
    "vmc": {"run_type": "variational", "sampling_method": "no_importance_sampling", "QF_modification_type": "none"},
    "vmc_umrigar93": {"run_type": "variational", "sampling_method": "umrigar93_importance_sampling",
                      "QF_modification_type": "umrigar93_unequalelectrons"},
}


def available() -> bool:
    return os.path.exists(REF_EXE)


def run_reference(system, mode: str, dt: float, walkers: int, steps: int, procs: int, energy: float = -1.0,
                  timeout: float = 300.0) -> Dict[str, object]:
    """Returns aggregate walker-moves/s over `procs` concurrent processes."""
    if not available():
        raise FileNotFoundError(REF_EXE)
    work = tempfile.mkdtemp(prefix="qmcref_")
    flags = dict(RUN_FLAGS[mode])
    flags.update({"dt": float(dt), "number_of_walkers": int(walkers), "max_time_steps": int(steps),
                  "equilibration_steps": 1, "one_e_per_iter": 1, "energy": float(energy),
                  "output_interval": 10 ** 6, "walkers_per_pass": 1})
    procs_l = []
    t0 = time.perf_counter()
    for p in range(procs):
        d = os.path.join(work, f"p{p}")
        os.makedirs(d)
        f = dict(flags)
        f["iseed"] = -(1000 + 7 * p)
        system.to_ckmf(os.path.join(d, "run.ckmf"), f)
        log = open(os.path.join(d, "run.log"), "w")
        procs_l.append((subprocess.Popen([REF_EXE, "run.ckmf"], cwd=d, stdout=log, stderr=subprocess.STDOUT), log, d))
    rates, moves, ok = [], 0, True
    for pr, log, d in procs_l:
        try:
            rc = pr.wait(timeout=timeout)
        except subprocess.TimeoutExpired:
            pr.kill()
            rc = -9
        log.close()
        txt = open(os.path.join(d, "run.log")).read()
        m = _ENTIRE.findall(txt)
        if rc != 0 or not m:
            ok = False
            continue
        us, n = float(m[-1][0]), int(m[-1][1])
        rates.append(1e6 / us)
        moves += n
    wall = time.perf_counter() - t0
    return {"ok": ok and len(rates) == procs, "moves_per_s": sum(rates), "per_process": rates, "moves": moves,
            "wall_s": wall, "procs": procs, "mode": mode, "walkers": walkers, "steps": steps, "workdir": work}
