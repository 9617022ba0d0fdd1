#!/usr/bin/env python
"""Benchmark of the B200 walker path: walker-moves/s of plain-FP64 DMC on the
30-electron synthetic molecule (6 nuclei, 120 contracted Gaussians, 16,384
walkers, tau = 0.01, drift-diffusion single-electron moves, nonunit-weight
branching, full LU refresh every 50 steps).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One bench step = one whole DMC block of the workload: lcm(N, refresh
interval) = 150 single-electron moves (propose, evaluate, accept/reject) of
every live walker, i.e. 5 sweeps of the 30 electrons with their 5 reweight /
branching passes (after each move of electron 0) and 3 full LU refreshes
(every 50 moves), so every timed region, however short, holds the same
share of each kind of work.  Under torchrun each rank runs an independent
walker population (walkers shard with no data-path collective; weak
scaling); the timed region is bracketed by barriers and the max time over
ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "dmc_6nuc_30e"
DEFAULT_WALKERS = 16384
REFRESH_INTERVAL = 50


def block_moves(N: int) -> int:
    """Single-electron moves per walker in one bench step: the least common
    multiple of the sweep length N (a reweight / branching pass after every
    move of electron 0) and the LU refresh interval."""
    return N * REFRESH_INTERVAL // math.gcd(N, REFRESH_INTERVAL)


def workload_config(system, walkers: int) -> dict:
    """The workload's identity, printed the same way by both arms."""
    N = system.n_electrons
    return {"workload": WORKLOAD, "electrons": N, "nuclei": system.n_nuclei, "basis_functions": system.n_basis,
            "walkers_per_gpu": walkers, "tau": 0.01, "refresh_interval": REFRESH_INTERVAL,
            "moves_per_walker_per_step": block_moves(N),
            "step": f"one DMC block: {block_moves(N)} single-electron moves of every walker "
                    f"({block_moves(N) // N} sweeps with their reweight/branching passes, "
                    f"{block_moves(N) // REFRESH_INTERVAL} LU refreshes)"}


def bytes_per_move(n: int, N: int) -> int:
    """Algorithmic HBM bytes of one FP64 walker-move: the moved spin's inverse
    read + written (2 n^2 8), its gradient / Laplacian rows read for the ratio
    sums (4 n^2 8), the four new derivative rows written (4 n 8), positions
    read (24 N), Jastrow gradients read + written (48 N), new gradients
    written (24 N) and the scalars (24)."""
    return 2 * n * n * 8 + 4 * n * n * 8 + 4 * n * 8 + 24 * N + 48 * N + 24 * N + 24


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(workload: str):
    """Per-walker-move DRAM bytes of the move kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    v = d.get(workload, {}).get("dram_bytes_per_walker_move")
    return float(v) if v is not None else None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dmc_params(seed: int, e0: float, reweight_start: int = 0):
    from qmcbeaver_b200.desc import (QMCB_DMC, QMCB_ECUT_BDJM_PUSH88, QMCB_EMOD_UMRIGAR93, QMCB_IMPORTANCE_SAMPLING,
                                     QMCB_QF_UMRIGAR93_UNEQUAL, run_params)
    return run_params(run_type=QMCB_DMC, sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL,
                      energy_modification=QMCB_EMOD_UMRIGAR93, dt=0.01, refresh_interval=REFRESH_INTERVAL,
                      reweight_start_step=reweight_start, energy_trial=e0, energy_estimated=e0, energy_original=e0,
                      seed=seed, energy_cutoff=QMCB_ECUT_BDJM_PUSH88, population_control=1.0 / 0.01)


EQUIL_SWEEPS = 5
# Equilibrated mean local energy of the 30-electron trial function (Hartree),
# the reference's input `energy` (E_T start, observable cutoff centre).
E_GUESS = -55.0


def cpu_reference_sample(system, walkers: int, steps: int, procs: int, e0: float):
    """The reference CPU program on this workload: its DMC when the population
    survives, else its drift-diffusion VMC steps (same per-move path)."""
    from oracle import refrun
    if not refrun.available():
        return None
    r = refrun.run_reference(system, "dmc", 0.01, walkers, steps, procs, energy=e0)
    if not r["ok"]:
        r = refrun.run_reference(system, "vmc_drift", 0.01, walkers, steps, procs, energy=e0)
        r["note"] = "reference DMC population collapsed on this trial function; timed its drift-diffusion VMC moves"
    return r


def mixed_section(system, W, e0, rank, args):
    """The same DMC workload with the mixed-precision path (FP32 basis and
    orbital rows, FP64 inverse / ratios / refresh / energies) and its local
    energy error against the FP64 path on identical configurations."""
    import torch
    from qmcbeaver_b200.api import QMCB200Functions
    from qmcbeaver_b200.desc import QMCB_PREC_FP64, QMCB_PREC_MIXED, run_params
    from qmcbeaver_b200.replicas import aggregate_timing, replica_seed
    N = system.n_electrons
    p = dmc_params(seed=replica_seed(91, rank), e0=-1.0, reweight_start=EQUIL_SWEEPS * N)
    p.precision = QMCB_PREC_MIXED
    f = QMCB200Functions(system, 2 * W, p)
    f.init_walkers(system.initial_positions(W, seed=2000 + rank))
    f.run_steps(0, EQUIL_SWEEPS * N)
    R_eq = f.get_walkers()["R"]
    p = dmc_params(seed=replica_seed(91, rank), e0=e0)
    p.precision = QMCB_PREC_MIXED
    f.set_params(p)
    f.init_walkers(R_eq)
    P = block_moves(N)
    f.run_steps(0, args.warmup * P)
    steps = max(args.steps // 4, 1) * P
    torch.cuda.synchronize()
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.ExternalStream(f.stream)
    s_ev.record(stream)
    st = f.run_steps(args.warmup * P, steps)
    e_ev.record(stream)
    torch.cuda.synchronize()
    ms, moves = aggregate_timing(s_ev.elapsed_time(e_ev), st.n_moves)
    f.close()
    # local-energy error on identical configurations (256 walkers, 2 sweeps of moves)
    Wc = 256
    a = QMCB200Functions(system, Wc, run_params(precision=QMCB_PREC_FP64, qf_modification=2, dt=0.01))
    b = QMCB200Functions(system, Wc, run_params(precision=QMCB_PREC_MIXED, qf_modification=2, dt=0.01))
    R = np.ascontiguousarray(R_eq[:Wc])
    sl = np.arange(Wc)
    a.evaluate(sl, R, -1)
    b.evaluate(sl, R, -1)
    rng = np.random.default_rng(3)
    errs = []
    for m in range(2 * N):
        e = m % N
        R[:, e] += 0.1 * rng.standard_normal((Wc, 3))
        x, y = a.evaluate(sl, R, e), b.evaluate(sl, R, e)
        ok = (x["status"] == 0) & (y["status"] == 0)
        errs.append(np.abs(x["e_local"] - y["e_local"])[ok])
    a.close()
    b.close()
    err = np.concatenate(errs)
    return {"value": moves / (ms / 1e3), "unit": "walker-moves/s", "steps": steps,
            "el_error_vs_fp64_ha": {"median": float(np.median(err)), "p90": float(np.percentile(err, 90)),
                                    "p99": float(np.percentile(err, 99))},
            "note": "FP32 basis and orbital rows (FP64 accumulation), FP64 inverse, determinant ratio, ratio sums, "
                    "LU refresh and energies"}


def rows_section(args, rank: int):
    """The widened rows on their own workloads: Cambridge2 two-body Jastrow,
    a 12-determinant CI expansion, the three-body Jastrow (with Cambridge2)
    and the reference's water input (cusps, three-body, Umrigar93 moves),
    VMC with drift on the device (timed
    with CUDA events on the library's stream), next to the reference CPU
    program on the same systems (all host cores, a bounded sample)."""
    import torch
    from qmcbeaver_b200.api import QMCB200Functions
    from qmcbeaver_b200.desc import QMCB_IMPORTANCE_SAMPLING, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
    from qmcbeaver_b200.replicas import aggregate_timing, replica_seed
    from qmcbeaver_b200.system import make_system
    from qmcbeaver_b200.desc import QMCB_UMRIGAR93_IMPORTANCE_SAMPLING
    from qmcbeaver_b200.system import system_from_arrays
    out = {}
    # the reference's own water input as this repository's reader builds it
    # (cusp replacement, Cambridge three-body Jastrow; tests/golden/inputs),
    # with its own sampling method
    h2o = np.load(os.path.join(ROOT, "tests", "golden", "inputs", "h2o.npz"))
    h2o = system_from_arrays({k[4:]: h2o[k] for k in h2o.files if k.startswith("sys_")})
    rows = [("vmc_cambridge2_16e", make_system("vmc_cambridge2_16e", seed=1), 8192, QMCB_IMPORTANCE_SAMPLING),
            ("vmc_multidet_12e", make_system("vmc_multidet_12e", seed=1), 8192, QMCB_IMPORTANCE_SAMPLING),
            ("vmc_threebody_16e", make_system("vmc_threebody_16e", seed=1), 8192, QMCB_IMPORTANCE_SAMPLING),
            ("h2o_input_umrigar93", h2o, 8192, QMCB_UMRIGAR93_IMPORTANCE_SAMPLING)]
    for wl, s, W, sampling in rows:
        N = s.n_electrons
        p = run_params(sampling=sampling, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01,
                       refresh_interval=50, seed=replica_seed(17, rank), rel_cutoff=0.0)
        f = QMCB200Functions(s, W, p)
        f.init_walkers(s.initial_positions(W, seed=300 + rank))
        f.run_steps(0, 5 * N)
        steps = max(40 * N, args.warmup)
        torch.cuda.synchronize()
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.ExternalStream(f.stream)
        s_ev.record(stream)
        st = f.run_steps(5 * N, steps)
        e_ev.record(stream)
        torch.cuda.synchronize()
        ms, moves = aggregate_timing(s_ev.elapsed_time(e_ev), st.n_moves)
        f.close()
        row = {"value": moves / (ms / 1e3), "unit": "walker-moves/s", "walkers": W, "steps": steps,
               "electrons": N, "basis_functions": s.n_basis, "determinants": s.n_det,
               "energy": st.sum_weight_energy / max(st.sum_weight, 1e-300)}
        if rank == 0 and not args.no_cpu_baseline:
            from oracle import refrun
            if refrun.available():
                mode = "vmc_umrigar93" if sampling == QMCB_UMRIGAR93_IMPORTANCE_SAMPLING else "vmc_drift"
                r = refrun.run_reference(s, mode, 0.01, 32, 400, os.cpu_count() or 1)
                if r["ok"]:
                    row["cpu_reference"] = {"value": r["moves_per_s"], "unit": "walker-moves/s", "cores": r["procs"],
                                            "sample": f"{r['procs']} processes x 32 walkers x 400 steps of the "
                                                      f"reference's {mode} VMC"}
        out[wl] = row
    return out


def serving_section(args):
    """Poisson arrivals of VMC energy jobs (molecules drawn like the
    uneven-batching workload, 4-40 electrons), run concurrently with
    footprint admission, next to the same jobs solved one after another."""
    from qmcbeaver_b200.serving import Server, make_jobs
    kw = dict(electrons=(4, 40), walkers=(256, 2048), target_error=0.2, max_sweeps=200)
    mix = make_jobs(args.serve_jobs, rate=args.serve_rate, seed=11, **kw)
    res = Server(max_active=16).run(mix)
    seq = make_jobs(args.serve_jobs, rate=args.serve_rate, seed=11, **kw)
    ref = Server(max_active=1).run(seq)
    same = all(abs(a.energy - b.energy) <= 1e-9 * max(1.0, abs(b.energy)) for a, b in zip(mix, seq)
               if len(a.energies) == len(b.energies))
    # the same arrivals with all active jobs stepped as one group per batch
    # of 40 steps (the largest job's sweep)
    grp = make_jobs(args.serve_jobs, rate=args.serve_rate, seed=11, **kw)
    rg = Server(max_active=16, mode="group", batch_steps=40).run(grp)
    return {"jobs": res["jobs"], "arrival_rate_per_s": args.serve_rate, "target_error_ha": kw["target_error"],
            "latency_p50_s": res["latency_p50_s"], "latency_p99_s": res["latency_p99_s"],
            "walker_moves_per_s": res["walker_moves_per_s"],
            "sequential": {"latency_p50_s": ref["latency_p50_s"], "latency_p99_s": ref["latency_p99_s"],
                           "walker_moves_per_s": ref["walker_moves_per_s"]},
            "group_mode": {"latency_p50_s": rg["latency_p50_s"], "latency_p99_s": rg["latency_p99_s"],
                           "walker_moves_per_s": rg["walker_moves_per_s"], "jobs": rg["jobs"]},
            "same_results_alone_and_mixed": bool(same)}


def _batch_compare(jobs, B, timed):
    """One group over the jobs' handles (tuned first) against the same steps
    run handle after handle and on all handles' streams at once; wall-clock
    walker-moves/s around synchronous batches of B steps."""
    from qmcbeaver_b200.api import QMCB200Functions, QMCB200Group
    from qmcbeaver_b200.desc import QMCB_IMPORTANCE_SAMPLING, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
    hs = []
    for j in jobs:
        p = run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01,
                       seed=j.seed, rel_cutoff=0.0)
        f = QMCB200Functions(j.system, j.walkers, p)
        f.init_walkers(j.system.initial_positions(j.walkers, seed=j.seed))
        hs.append(f)
    g = QMCB200Group(hs)
    step = 0
    tune_t0 = time.perf_counter()
    while g.config()["chosen"] < 0:
        g.run_steps(step, B)
        step += B
    tune_s = time.perf_counter() - tune_t0

    def timed_run(run_batch):
        nonlocal step
        moves = 0.0
        t0 = time.perf_counter()
        for _ in range(timed):
            moves += run_batch(step)
            step += B
        return moves / (time.perf_counter() - t0)

    def grouped(s0):
        return sum(st.n_moves for st in g.run_steps(s0, B))

    def one_by_one(s0):
        return sum(f.run_steps(s0, B).n_moves for f in hs)

    def streams(s0):
        for f in hs:
            f.run_steps_async(s0, B)
        return sum(f.steps_collect().n_moves for f in hs)

    r_group = timed_run(grouped)
    r_seq = timed_run(one_by_one)
    r_streams = timed_run(streams)
    cfg = g.config()
    g.close()
    for f in hs:
        f.close()
    ne = [j.system.n_electrons for j in jobs]
    return {"molecules": len(jobs), "electrons": [min(ne), max(ne)], "walkers": sum(j.walkers for j in jobs),
            "steps_per_batch": B, "timed_batches": timed, "unit": "walker-moves/s",
            "group": r_group, "one_handle_after_another": r_seq, "concurrent_streams": r_streams,
            "group_speedup_vs_sequential": r_group / r_seq, "group_speedup_vs_streams": r_group / r_streams,
            "tuning": {"configurations": cfg["n_configs"], "chosen": cfg["chosen"], "buckets": cfg["n_buckets"],
                       "warps_per_block": cfg["warps_per_block"], "tuning_batches_s": tune_s}}


def batching_section(args):
    """The uneven-batching workload: 64 synthetic molecules, even electron
    counts uniform in 4-200, basis 4N, N/5 nuclei with Z in {1, 6, 7, 8},
    orthonormalised random orbital coefficients; walkers per molecule
    uniform in 256-2048 (the workload's 256-8192 capped at 2048 so that all
    64 walker populations fit in HBM together: this layout keeps every
    walker's orbital rows, derivative rows and inverses resident).  VMC
    importance-sampled steps, 100 per batch.  Next to it the same comparison
    for 64 small molecules (4-40 electrons, the serving jobs' sizes), where
    each molecule's step is a short kernel."""
    from qmcbeaver_b200.serving import make_jobs
    out = _batch_compare(make_jobs(64, rate=1.0, seed=23, electrons=(4, 200), walkers=(256, 2048),
                                   orbitals="random"), B=100, timed=2)
    out["small_molecules"] = _batch_compare(make_jobs(64, rate=1.0, seed=29, electrons=(4, 40), walkers=(256, 2048),
                                                      orbitals="random"), B=40, timed=5)
    return out


def run_reference_arm(args, rank: int):
    """The reference's own CPU program on the same workload and bench step:
    every step is one run of the unmodified QMcBeaver.x per host core (64
    walkers each, distinct seeds) over one DMC block of single-electron moves;
    walker-moves/s from the reference's own "Entire Step" timer, summed over
    the processes, averaged over the timed steps."""
    if rank != 0:
        return
    from qmcbeaver_b200.system import make_system
    from oracle import refrun
    system = make_system(WORKLOAD, seed=1)
    procs = os.cpu_count() or 1
    if not refrun.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/QMcBeaver.x not built (reference tree absent at build time)"}))
        return
    P = block_moves(system.n_electrons)
    walkers = 64
    for _ in range(args.warmup):
        cpu_reference_sample(system, walkers=walkers, steps=P, procs=procs, e0=E_GUESS)
    vals, last = [], None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        last = cpu_reference_sample(system, walkers=walkers, steps=P, procs=procs, e0=E_GUESS)
        vals.append(last["moves_per_s"])
    wall = time.perf_counter() - t0
    v = float(np.mean(vals)) if vals else 0.0
    sample = (f"each step: {procs} processes x {walkers} walkers x {P} single-electron moves of the reference's "
              f"{last['mode']} ({last.get('note', 'full DMC')})")
    out = {"metric": "walker-moves/s", "value": v, "unit": "walker-moves/s", "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(args.steps, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": dict(workload_config(system, args.walkers), parallelism="single"),
           "cpu_baseline": {"value": v, "unit": "walker-moves/s", "cores": procs, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": v, "unit": "walker-moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40, help="timed bench steps (whole DMC blocks, 150 moves each)")
    ap.add_argument("--warmup", type=int, default=3, help="untimed bench steps (whole DMC blocks)")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--walkers", type=int, default=DEFAULT_WALKERS)
    ap.add_argument("--e2e-steps", type=int, default=2, help="bench steps timed end to end, one API call per move")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the mixed-precision and serving sections")
    ap.add_argument("--serve-jobs", type=int, default=24)
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--case", choices=["multidet_small", "group_small"],
                    help="run one small profiling workload instead of the benchmark")
    args = ap.parse_args()
    if args.case:
        profile_case(args.case)
        return
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    from qmcbeaver_b200.api import QMCB200Functions
    from qmcbeaver_b200.replicas import aggregate_timing, reduce_energy, replica_seed
    from qmcbeaver_b200.system import make_system

    system = make_system(WORKLOAD, seed=1)
    W = args.walkers
    N, n = system.n_electrons, system.n_alpha
    R0 = system.initial_positions(W, seed=1000 + rank)
    # equilibration: drift-diffusion moves with the weights held at 1 (the
    # reference keeps dW = 1 for its first 100 steps, QMcBeaver/src/QMCWalker.cpp:1071),
    # then E_T = E_est = E_orig = the equilibrated mean local energy
    eq_steps = EQUIL_SWEEPS * N
    f = QMCB200Functions(system, 2 * W, dmc_params(seed=replica_seed(77, rank), e0=-1.0, reweight_start=eq_steps))
    f.init_walkers(R0)
    f.run_steps(0, eq_steps)
    R_eq = f.get_walkers()["R"]
    e0 = float(np.mean(f.get_walkers()["e_local"]))
    f.set_params(dmc_params(seed=replica_seed(77, rank), e0=e0))
    f.init_walkers(R_eq)
    def barrier():
        if dist is not None:
            dist.barrier()

    P = block_moves(N)
    # warm-up
    f.run_steps(0, args.warmup * P)
    stream = torch.cuda.ExternalStream(f.stream)
    f.set_profiling(True)
    f.kernel_stats(reset=True)
    barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start.record(stream)
        st = f.run_steps(args.warmup * P, args.steps * P)
        t_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = t_start.elapsed_time(t_end)
    ks = f.kernel_stats(reset=True)
    f.set_profiling(False)
    ms, moves = aggregate_timing(ms, st.n_moves)
    value = moves / (ms / 1e3)
    ensemble = reduce_energy(st.sum_weight, st.sum_weight_energy, st.sum_weight_energy2, st.n_walkers,
                             st.final_weight)

    # roofline of the move kernel (dominant): algorithmic bytes per launch / launch time
    mv = ks["move"]
    avg_ms = mv["ms"] / max(mv["launches"], 1)
    walkers_per_launch = st.n_moves / max(mv["launches"], 1)
    bpm = bytes_per_move(n, N)
    achieved = bpm * walkers_per_launch / (avg_ms / 1e3) / 1e9
    peak, peak_kind = read_peaks()
    tr = read_traffic(WORKLOAD)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tr * walkers_per_launch) if tr is not None else None,
                "peak_kind": peak_kind, "kernel": "k_move", "algorithmic_bytes_per_walker_move": bpm,
                "walkers_per_launch": walkers_per_launch, "avg_launch_ms": avg_ms}
    launches = int(sum(v["launches"] for v in ks.values()))

    # end to end through the public API: one qmcb_run_steps call per step, with
    # the host's trial energy uploaded before and the step statistics read back after
    from qmcbeaver_b200.desc import RunParams, StepStats
    import ctypes
    barrier()
    p = dmc_params(seed=replica_seed(77, rank), e0=e0)
    e_est = e0
    sw = swe = 0.0
    step0 = (args.warmup + args.steps) * P
    e2e_moves_per_walker = args.e2e_steps * P
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_moves = 0.0
    # each step's E_T goes up before it is enqueued; its statistics come back
    # while the next step runs (two batches in flight), so the host's trial
    # energy follows the statistics one step behind
    f.set_params(p)
    f.run_steps_async(step0, 1)
    for s in range(e2e_moves_per_walker):
        if s + 1 < e2e_moves_per_walker:
            f.set_params(p)
            f.run_steps_async(step0 + s + 1, 1)
        st2 = f.steps_collect()
        e2e_moves += st2.n_moves
        if st2.sum_weight > 0:
            sw += st2.sum_weight
            swe += st2.sum_weight_energy
            e_est = swe / sw
        if st2.final_weight > 0:
            p.energy_estimated = e_est
            p.energy_trial = e_est - p.population_control * np.log(st2.final_weight / W)
        elif st2.n_walkers > 0:
            p.energy_trial = e_est
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s, e2e_moves = aggregate_timing(e2e_s, e2e_moves)
    e2e = {"value": e2e_moves / e2e_s, "unit": "walker-moves/s", "h2d_bytes_per_step": P * ctypes.sizeof(RunParams),
           "d2h_bytes_per_step": P * (ctypes.sizeof(StepStats) + 16),
           "steps": args.e2e_steps, "ms_per_step": 1e3 * e2e_s / max(args.e2e_steps, 1),
           "api": "qmcb_set_params + qmcb_run_steps_async(step, 1) per single-electron move, statistics collected "
                  "one move behind with qmcb_steps_collect (host E_T in, move statistics out); bytes per bench step"}

    # reference-facing evaluate (QMCFunctions::evaluate shape) with host buffers
    slots = np.arange(min(W, 4096), dtype=np.int32)
    Rh = np.ascontiguousarray(R_eq[: len(slots)])
    f2 = QMCB200Functions(system, len(slots), dmc_params(seed=1, e0=e0))
    f2.evaluate(slots, Rh, -1)
    rng = np.random.default_rng(5)
    t0 = time.perf_counter()
    n_eval = 2 * N
    for s in range(n_eval):
        e = s % N
        Rh[:, e] += 0.1 * rng.standard_normal((len(slots), 3))
        f2.evaluate(slots, Rh, e)
    ev_s = time.perf_counter() - t0
    f2.close()
    e2e_eval = {"value": len(slots) * n_eval / ev_s, "unit": "walker-moves/s", "walkers": len(slots),
                "h2d_bytes_per_step": len(slots) * (3 * N * 8 + 4),
                "d2h_bytes_per_step": len(slots) * (6 * N * 8 + 7 * 8 + 1),
                "api": "qmcb_evaluate(which_e, host R[num][N][3]) per step, no Markov chain"}

    out = {"metric": "walker-moves/s", "value": value, "unit": "walker-moves/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": dict(workload_config(system, W), parallelism=f"replicas{world}" if world > 1 else "single",
                          l2="inputs larger than L2: walker state %.0f MB per GPU" % (f.state_bytes() / 1e6)),
           "run": {"walker_moves": moves, "final_walkers": st.n_walkers,
                   "single_electron_steps": args.steps * P, "kernel_launches_by_kind": {k: v["launches"] for k, v in ks.items()}},
           "roofline": roofline, "gpu_launches": launches, "kernels": ks, "e2e": e2e, "e2e_evaluate_api": e2e_eval,
           "energy": {"mean_weighted_E_L": ensemble["energy"], "walkers_all_ranks": ensemble["walkers"],
                      "acceptance": st.sum_accept / max(st.n_moves, 1), "singular": st.n_singular}}
    clocks = clk.summary()
    if clocks is not None:
        out["clocks"] = clocks
    f.close()
    if not args.no_extras:
        out["mixed"] = mixed_section(system, W, e0, rank, args)
        out["rows"] = rows_section(args, rank)
        if world == 1:
            out["serving"] = serving_section(args)
            out["batching"] = batching_section(args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_sample(system, walkers=64, steps=1500, procs=os.cpu_count() or 1, e0=E_GUESS)
        if r is not None:
            out["cpu_baseline"] = {"value": r["moves_per_s"], "unit": "walker-moves/s", "cores": r["procs"],
                                   "kind": "reference",
                                   "sample": f"{r['procs']} processes x {r['walkers']} walkers x {r['steps']} steps "
                                             f"of the reference's {r['mode']} ({r.get('note', 'full DMC')})"}
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
