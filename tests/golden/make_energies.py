"""Generates tests/golden/energies/*.json: VMC energies of the reference
QMcBeaver program itself (oracle/_ref/QMcBeaver.x, built from its sources)
on some of its own input files, run as variational calculations with the
inputs' other flags (sampling method, dt, drift limit, cusp replacement,
three-body Jastrow), as P independent processes with different seeds
(the reference's manager-worker mode is independent walker populations
plus a reduce).  The energy and error of each process come from the
reference's own results table ("Energy: E +/- err", blocked);
the processes are combined by inverse-variance weights.

Run:  python tests/golden/make_energies.py      (needs the reference tree)
"""
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "energies")
sys.path.insert(0, ROOT)
from oracle.evaluators import REFERENCE_TREE as REF_INPUTS  # noqa: E402

CASES = {
    # name: (input, processes, walkers, steps, equilibration steps, extra flags)
    "h2o_vmc": ("examples/h2o.ckmf", 16, 40, 8000, 1000, {}),
    # single-electron moves, as the device makes them
    "h2o_vmc_one_e": ("examples/h2o.ckmf", 16, 80, 16000, 2000, {"one_e_per_iter": 1}),
    # diffusion Monte Carlo with the input's DMC settings, single-electron moves
    "h2o_dmc_one_e": ("examples/h2o.ckmf", 16, 100, 30000, 5000,
                      {"one_e_per_iter": 1, "run_type": "diffusion", "energy": -76.36}),
}
_ENERGY = re.compile(r"-+ Energy -+\s*\n\s*([-0-9.eE+]+)\s*\+/-\s*([0-9.eE+-]+)")


def run_case(name: str) -> None:
    from qmcbeaver_b200.ckmf import patch_flags, read_ckmf
    from oracle.refrun import REF_EXE
    rel, P, W, steps, eq, extra = CASES[name]
    path = os.path.join(REF_INPUTS, rel)
    text = open(path).read()
    flags = dict(read_ckmf(path).flags)
    flags.update({k: str(v) for k, v in extra.items()})
    work = tempfile.mkdtemp(prefix="qmcref_e_")
    procs = []
    for p in range(P):
        d = os.path.join(work, f"p{p}")
        os.makedirs(d)
        f = {"run_type": "variational", "max_time_steps": steps, "number_of_walkers": W,
             "equilibration_steps": eq, "iseed": -(4001 + 17 * p), "output_interval": 10 ** 7, "print_configs": 0,
             "optimize_Psi": 0, "walkers_per_pass": 1}
        f.update(extra)
        with open(os.path.join(d, "run.ckmf"), "w") as fh:
            fh.write(patch_flags(text, f))
        log = open(os.path.join(d, "run.log"), "w")
        procs.append((subprocess.Popen([REF_EXE, "run.ckmf"], cwd=d, stdout=log, stderr=subprocess.STDOUT), log, d))
    es, errs = [], []
    for pr, log, d in procs:
        pr.wait()
        log.close()
        m = _ENERGY.search(open(os.path.join(d, "run.log")).read())
        if not m:
            raise RuntimeError(f"no energy in {d}/run.log")
        es.append(float(m.group(1)))
        errs.append(float(m.group(2)))
    w = [1.0 / e ** 2 for e in errs]
    E = sum(wi * ei for wi, ei in zip(w, es)) / sum(w)
    err = (1.0 / sum(w)) ** 0.5
    keep = ("sampling_method", "dt", "QF_modification_type", "one_e_per_iter", "replace_electron_nucleus_cusps",
            "use_three_body_jastrow")
    out = {"input": rel, "energy": E, "error": err, "processes": P, "walkers_per_process": W, "steps": steps,
           "equilibration_steps": eq, "per_process": list(zip(es, errs)),
           "flags": {k: flags.get(k) for k in keep}}
    os.makedirs(OUT, exist_ok=True)
    with open(os.path.join(OUT, name + ".json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(name, E, "+/-", err)


if __name__ == "__main__":
    for c in (sys.argv[1:] or list(CASES)):
        run_case(c)
