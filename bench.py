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


def read_bf16_peak() -> float:
    """Measured dense bf16 tensor throughput (TFLOP/s, burst), else the
    pool's earlier measurement."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["bf16_tflops"])
    return 1590.0


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
                      seed=seed, energy_cutoff=QMCB_ECUT_BDJM_PUSH88, population_control=1.0 / 0.01,
                      walker_deletion=1)


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


def el_errors(system, prec, W=256, sweeps=1, seed=3, R=None):
    """Per-walker |E_L - E_L(FP64)| of precision `prec` on identical
    configurations: a full evaluation, then `sweeps` sweeps of
    single-electron moves through the evaluate entry point."""
    from qmcbeaver_b200.api import QMCB200Functions
    from qmcbeaver_b200.desc import QMCB_PREC_FP64, run_params
    a = QMCB200Functions(system, W, run_params(precision=QMCB_PREC_FP64, qf_modification=2, dt=0.01))
    b = QMCB200Functions(system, W, run_params(precision=prec, qf_modification=2, dt=0.01))
    R = np.ascontiguousarray(R[:W] if R is not None else system.initial_positions(W, seed=seed))
    sl = np.arange(W)
    a.evaluate(sl, R, -1)
    b.evaluate(sl, R, -1)
    rng = np.random.default_rng(seed)
    errs = []
    N = system.n_electrons
    for m in range(sweeps * N):
        e = m % N
        R[:, e] += 0.1 * rng.standard_normal((W, 3))
        x, y = a.evaluate(sl, R, e), b.evaluate(sl, R, e)
        ok = (x["status"] == 0) & (y["status"] == 0)
        errs.append(np.abs(x["e_local"] - y["e_local"])[ok])
    a.close()
    b.close()
    err = np.concatenate(errs)
    return {"median": float(np.median(err)), "p99": float(np.percentile(err, 99)), "max": float(err.max()),
            "samples": int(err.size), "within_1e-5_ha": float(np.mean(err <= 1e-5))}


PREC_NAMES = {0: "fp64", 1: "mixed_fp32_rows", 2: "int8_slices_tcgen05", 3: "bf16_tcgen05", 4: "bf16x3_tcgen05"}


def precision_section(args, rank: int):
    """The 100-electron workload (20 nuclei, 400 basis functions, 65,536
    walkers, DMC as the main workload) in five arithmetic modes: plain
    FP64 (one warp per walker, FP64 tensor-pipe contraction), FP32 basis and
    orbital rows, the batched tensor-core contraction of int8 digit
    planes (tcgen05 kind::i8, FP64-equivalent rows), and the same batched
    contraction with BF16 operands and FP32 accumulation (tcgen05 kind::f16),
    plain and split into hi + lo with three products, each timed with CUDA
    events over two DMC blocks (200 moves per walker: 2 branching passes, 4
    LU refreshes), with per-kernel times; then the per-walker local-energy
    error of each mode against FP64 on identical configurations, on this
    workload, the 30-electron one and the reference's water input."""
    import torch
    from qmcbeaver_b200.api import QMCB200Functions
    from qmcbeaver_b200.desc import (QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC, QMCB_PREC_FP64, QMCB_PREC_INT8_SLICES,
                                     QMCB_PREC_MIXED)
    from qmcbeaver_b200.replicas import aggregate_timing, replica_seed
    from qmcbeaver_b200.system import make_system, system_from_arrays
    system = make_system("mixed_20nuc_100e", seed=1)
    W = args.c3_walkers
    N, n = system.n_electrons, system.n_alpha
    out = {"workload": "mixed_20nuc_100e", "walkers": W, "electrons": N, "basis_functions": system.n_basis,
           "modes": {}}
    R_eq = None
    reduced = (QMCB_PREC_INT8_SLICES, QMCB_PREC_BF16X3_TC, QMCB_PREC_BF16_TC, QMCB_PREC_MIXED)
    for prec in (QMCB_PREC_FP64,) + reduced:
        p = dmc_params(seed=replica_seed(91, rank), e0=-1.0, reweight_start=10 ** 9)
        p.precision = prec
        f = QMCB200Functions(system, 2 * W, p)
        f.init_walkers(system.initial_positions(W, seed=2000 + rank))
        f.run_steps(0, 2 * N)
        wk = f.get_walkers()
        e0 = float(np.mean(wk["e_local"]))
        if R_eq is None:
            R_eq = wk["R"]
        p = dmc_params(seed=replica_seed(91, rank), e0=e0)
        p.precision = prec
        f.set_params(p)
        f.init_walkers(wk["R"])
        f.run_steps(0, N)
        f.set_profiling(True)
        f.kernel_stats(reset=True)
        steps = 2 * block_moves(N)
        torch.cuda.synchronize()
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.ExternalStream(f.stream)
        s_ev.record(stream)
        st = f.run_steps(N, steps)
        e_ev.record(stream)
        torch.cuda.synchronize()
        ms, moves = aggregate_timing(s_ev.elapsed_time(e_ev), st.n_moves)
        ks = f.kernel_stats(reset=True)
        f.close()
        mode = {"value": moves / (ms / 1e3), "unit": "walker-moves/s", "steps": steps, "ms": ms,
                "kernels_ms": {k: round(v["ms"], 3) for k, v in ks.items() if v["launches"]},
                "final_walkers": st.n_walkers}
        mv = ks["move"]
        wpl = st.n_moves / max(mv["launches"], 1)  # walkers per move launch
        mode["move_kernel_roofline"] = {
            "bound": "hbm", "algorithmic_bytes_per_walker_move": bytes_per_move(n, N),
            "achieved_gbs": bytes_per_move(n, N) * wpl / (mv["ms"] / mv["launches"] / 1e3) / 1e9,
            "peak_gbs": read_peaks()[0]}
        mode["move_kernel_roofline"]["frac"] = mode["move_kernel_roofline"]["achieved_gbs"] / read_peaks()[0]
        if prec == QMCB_PREC_INT8_SLICES:
            # tensor ops the contraction issues per launch: tiles of 25
            # walkers x 32-orbital tiles x 32-byte K steps x 36 digit-pair
            # MMAs (8 digit planes, pairs i + j < 8) of 128 x 32 x 32 int8
            # multiply-adds
            mm = ks["rows_mma"]
            ops = (-(-wpl // 25)) * (-(-n // 32)) * (-(-system.n_basis // 32)) * 36 * 2 * 128 * 32 * 32
            peak_tops = 2.0 * read_bf16_peak()
            mode["contraction_roofline"] = {
                "bound": "tensor", "kernel": "k_rows_mma", "achieved_tops": ops / (mm["ms"] / mm["launches"] / 1e3) / 1e12,
                "peak_tops": peak_tops, "peak_kind": "int8 dense = 2 x measured bf16 dense burst",
                "avg_launch_ms": mm["ms"] / mm["launches"]}
            mode["contraction_roofline"]["frac"] = mode["contraction_roofline"]["achieved_tops"] / peak_tops
        if prec in (QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC):
            # tiles of 25 walkers x 32-orbital tiles x 16-function K steps x
            # 1 or 3 MMAs of 128 x 32 x 16 BF16 multiply-adds
            mm = ks["rows_mma"]
            per = 3 if prec == QMCB_PREC_BF16X3_TC else 1
            ops = (-(-wpl // 25)) * (-(-n // 32)) * (-(-system.n_basis // 16)) * per * 2 * 128 * 32 * 16
            peak_tf = read_bf16_peak()
            mode["contraction_roofline"] = {
                "bound": "tensor", "kernel": "k_rows_mma_bf", "achieved_tflops": ops / (mm["ms"] / mm["launches"] / 1e3) / 1e12,
                "peak_tflops": peak_tf, "peak_kind": "measured bf16 dense burst",
                "avg_launch_ms": mm["ms"] / mm["launches"]}
            mode["contraction_roofline"]["frac"] = mode["contraction_roofline"]["achieved_tflops"] / peak_tf
        out["modes"][PREC_NAMES[prec]] = mode
    fp = out["modes"]["fp64"]["value"]
    for k, v in out["modes"].items():
        v["vs_fp64"] = v["value"] / fp
    h2o = np.load(os.path.join(ROOT, "tests", "golden", "inputs", "h2o.npz"))
    h2o = system_from_arrays({k[4:]: h2o[k] for k in h2o.files if k.startswith("sys_")})
    err = {}
    for name, s, R in (("mixed_20nuc_100e", system, R_eq), ("dmc_6nuc_30e", make_system("dmc_6nuc_30e", seed=1), None),
                       ("h2o_input", h2o, None)):
        err[name] = {PREC_NAMES[p]: el_errors(s, p, R=R) for p in reduced}
    out["el_error_vs_fp64_ha"] = err
    out["note"] = ("int8_slices_tcgen05: basis values and MO coefficients scaled per 32-function block and cut into 8 int8 "
                   "digit planes, "
                   "tcgen05.mma kind::i8 with exact int32 accumulation, FP64 recombination; FP64 inverse, "
                   "Sherman-Morrison update, ratio sums, refresh and energies. bf16_tcgen05: basis values and MO "
                   "coefficients rounded to BF16, tcgen05.mma kind::f16 with FP32 accumulation in TMEM over all "
                   "of K. bf16x3_tcgen05: the split-precision variant, hi + lo BF16 per value, hi.hi + hi.lo + "
                   "lo.hi accumulated in FP32. mixed_fp32_rows: FP32 basis and orbital rows, FP64 inverse and "
                   "energies.")
    return out


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
    """Serving: Poisson arrivals of VMC energy jobs at 1, 10, 30 and 100
    jobs/s.  Synthetic molecules drawn like the uneven-batching workload
    (4-200 electrons, basis 4N, N/5 nuclei, random orthonormal orbitals,
    256-1,024 walkers) are run to 0.2 Ha or a sweep cap: their local-energy
    spread (10-1,000 Ha) would need 1e9-1e12 samples for 1 mHa.  Each rate
    runs with the jobs' handles on concurrent streams; at 10 jobs/s also as
    one group per batch and one job at a time.  Then jobs on the reference's
    water input (cusp replacement, three-body Jastrow), whose trial function
    reaches the 1 mHa target of the serving workload in a few seconds of
    device time, arrive at 1 job/s.  At 10 jobs/s the arrivals also run with
    every job on split-BF16 tensor-core orbital rows, and the water jobs also
    on tensor-core rows at FP64 accuracy."""
    from qmcbeaver_b200.serving import Server, make_input_jobs, make_jobs
    from qmcbeaver_b200.system import system_from_arrays
    kw = dict(electrons=(4, 200), walkers=(256, 1024), target_error=0.2, max_sweeps=24, orbitals="random")
    out = {"jobs_per_rate": args.serve_jobs, "electrons": [4, 200], "target_error_ha": 0.2, "rates": {}}

    def summary(r):
        return {k: r[k] for k in ("jobs", "latency_p50_s", "latency_p99_s", "walker_moves_per_s", "wall_s")}

    for rate in (1.0, 10.0, 30.0, 100.0):
        r = Server(max_active=16).run(make_jobs(args.serve_jobs, rate=rate, seed=11, **kw))
        out["rates"][str(rate)] = {"streams": summary(r)}
    rate = 10.0
    mix = make_jobs(args.serve_jobs, rate=rate, seed=11, **kw)
    rg = Server(max_active=16, mode="group", batch_steps=50).run(make_jobs(args.serve_jobs, rate=rate, seed=11, **kw))
    out["rates"][str(rate)]["group"] = summary(rg)
    seq = make_jobs(args.serve_jobs, rate=rate, seed=11, **kw)
    rs = Server(max_active=1).run(seq)
    out["rates"][str(rate)]["one_at_a_time"] = summary(rs)
    # the same arrivals with every job on split-BF16 tensor-core orbital rows
    # (FP32 accumulation, FP64 inverse, refresh and energies)
    from qmcbeaver_b200.desc import QMCB_PREC_BF16X3_TC, QMCB_PREC_INT8_SLICES
    rb = Server(max_active=16).run(make_jobs(args.serve_jobs, rate=rate, seed=11, precision=QMCB_PREC_BF16X3_TC,
                                             **kw))
    out["rates"][str(rate)]["streams_bf16x3_rows"] = summary(rb)
    rm = Server(max_active=16).run(mix)
    out["same_results_alone_and_mixed"] = bool(all(
        abs(a.energy - b.energy) <= 1e-9 * max(1.0, abs(b.energy)) for a, b in zip(mix, seq)
        if len(a.energies) == len(b.energies)))
    h2o = np.load(os.path.join(ROOT, "tests", "golden", "inputs", "h2o.npz"))
    h2o = system_from_arrays({k[4:]: h2o[k] for k in h2o.files if k.startswith("sys_")})
    # the input's own time step; 500 equilibration sweeps (the blocked error
    # of a drifting series overstates the error), 8,192-16,384 walkers
    jobs = make_input_jobs(3, rate=1.0, system=h2o, seed=5, walkers=(8192, 16384), target_error=1e-3,
                           max_sweeps=6000, equil_sweeps=500, dt=0.01)
    r = Server(max_active=8).run(jobs)
    out["h2o_input_1mha"] = dict(summary(r), target_error_ha=1e-3, equil_sweeps=500,
                                 sweeps=[int(len(j.energies)) for j in jobs],
                                 errors_ha=[j.error for j in jobs], energies_ha=[j.energy for j in jobs])
    # the same 1 mHa jobs on tensor-core rows at FP64 accuracy (int8 digit planes)
    jobs = make_input_jobs(3, rate=1.0, system=h2o, seed=5, walkers=(8192, 16384), target_error=1e-3,
                           max_sweeps=6000, equil_sweeps=500, dt=0.01)
    for j in jobs:
        j.precision = QMCB_PREC_INT8_SLICES
    r = Server(max_active=8).run(jobs)
    out["h2o_input_1mha_int8_rows"] = dict(summary(r), target_error_ha=1e-3, equil_sweeps=500,
                                           sweeps=[int(len(j.energies)) for j in jobs],
                                           errors_ha=[j.error for j in jobs], energies_ha=[j.energy for j in jobs])
    return out


def _batch_compare(jobs, B, timed, precision=0, refresh_interval=0):
    """One group over the jobs' handles (tuned first) against the same steps
    run handle after handle and on all handles' streams at once; wall-clock
    walker-moves/s around synchronous batches of B steps.  precision: the
    orbital rows' arithmetic (QMCB_PREC_*); refresh_interval: the FP64
    inverse refresh (0: none)."""
    from qmcbeaver_b200.api import QMCB200Functions, QMCB200Group
    from qmcbeaver_b200.desc import QMCB_IMPORTANCE_SAMPLING, QMCB_QF_UMRIGAR93_UNEQUAL, run_params
    hs = []
    for j in jobs:
        p = run_params(sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01,
                       seed=j.seed, rel_cutoff=0.0, precision=precision, refresh_interval=refresh_interval)
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
    orthonormalised random orbital coefficients, walkers per molecule uniform
    in 256-8192 (every walker's orbital rows, derivative rows and inverses
    resident: about 120 GB for the 64 populations; if the device has less
    free memory the walker range is scaled down until they fit, and the
    range used is reported).  VMC importance-sampled steps, 50 per batch.
    Next to it the same comparison for 64 small molecules (4-40 electrons,
    the serving jobs' sizes), where each molecule's step is a short kernel,
    and both workloads again on the split-BF16 tensor-core orbital rows with
    an FP64 refresh every 50 moves."""
    from qmcbeaver_b200.serving import device_budget, make_jobs, state_footprint
    hi = 8192
    while True:
        jobs = make_jobs(64, rate=1.0, seed=23, electrons=(4, 200), walkers=(256, hi), orbitals="random")
        need = sum(state_footprint(j.system, j.walkers) // 2 for j in jobs)
        if need <= 0.9 * device_budget(1.0) or hi <= 1024:
            break
        hi //= 2
    out = _batch_compare(jobs, B=50, timed=2)
    out["walker_range"] = [256, hi]
    out["state_gb"] = need / 1e9
    small = make_jobs(64, rate=1.0, seed=29, electrons=(4, 40), walkers=(256, 2048), orbitals="random")
    out["small_molecules"] = _batch_compare(small, B=40, timed=5)
    # the configuration's FP32/BF16 orbital path with an FP64 refresh: every
    # member's rows from the split-BF16 tensor-core contraction with FP32
    # accumulation (FP32-class rows), the inverse refreshed in FP64 every 50 moves
    from qmcbeaver_b200.desc import QMCB_PREC_BF16X3_TC
    out["bf16x3_rows_fp64_refresh"] = _batch_compare(jobs, B=50, timed=2, precision=QMCB_PREC_BF16X3_TC,
                                                     refresh_interval=50)
    out["small_molecules"]["bf16x3_rows_fp64_refresh"] = _batch_compare(small, B=40, timed=5,
                                                                        precision=QMCB_PREC_BF16X3_TC,
                                                                        refresh_interval=50)
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


def profile_case(name: str) -> None:
    """Small fixed workloads for kernel captures (one GPU, a few hundred MB
    on the device): "multidet_small" runs 4N importance-sampled VMC steps of
    the 12-electron / 12-determinant system with 8,192 walkers (the
    several-determinant move kernel); "group_small" runs three batches of 40
    steps of 16 molecules of 4-40 electrons (256-2,048 walkers each) as one
    group in configuration 0 (the group move kernel); "rows_small" runs 6
    importance-sampled VMC steps of the 100-electron / 400-function system
    with 16,384 walkers under QMCB_PREC_INT8_SLICES (the tensor-core
    contraction k_rows_mma, its prep kernel and the move kernel on rows),
    "rows_bf16x3_small" the same under QMCB_PREC_BF16X3_TC (k_rows_mma_bf);
    "refresh_100e" sets up 16,384 walkers of the 100-electron system (one
    full evaluation) and runs 50 FP64 steps, the last of which refreshes
    every walker's inverses (the second k_full launch)."""
    from qmcbeaver_b200.api import QMCB200Functions, QMCB200Group
    from qmcbeaver_b200.desc import run_params
    from qmcbeaver_b200.system import make_system
    if name == "multidet_small":
        s = make_system("vmc_multidet_12e", seed=1)
        W = 8192
        f = QMCB200Functions(s, W, run_params(sampling=1, qf_modification=2, dt=0.01, seed=3, rel_cutoff=0.0))
        f.init_walkers(s.initial_positions(W, seed=1))
        st = f.run_steps(0, 4 * s.n_electrons)
        print("ok", st.n_moves)
        f.close()
    elif name == "group_small":
        from qmcbeaver_b200.serving import make_jobs
        jobs = make_jobs(16, rate=1.0, seed=29, electrons=(4, 40), walkers=(256, 2048), orbitals="random")
        hs = []
        for j in jobs:
            f = QMCB200Functions(j.system, j.walkers, run_params(sampling=1, qf_modification=2, dt=0.01,
                                                                 seed=j.seed, rel_cutoff=0.0))
            f.init_walkers(j.system.initial_positions(j.walkers, seed=j.seed))
            hs.append(f)
        g = QMCB200Group(hs)
        g.set_config(0)
        for b in range(3):
            st = g.run_steps(b * 40, 40)
        print("ok", sum(x.n_moves for x in st), g.config())
        g.close()
        for f in hs:
            f.close()
    elif name in ("rows_small", "rows_bf16x3_small"):
        from qmcbeaver_b200.desc import QMCB_PREC_BF16X3_TC, QMCB_PREC_INT8_SLICES
        s = make_system("mixed_20nuc_100e", seed=1)
        W = 16384  # 4.8 GB of walker state, 240 / 134 MB of operand planes: larger than L2
        prec = QMCB_PREC_INT8_SLICES if name == "rows_small" else QMCB_PREC_BF16X3_TC
        f = QMCB200Functions(s, W, run_params(sampling=1, qf_modification=2, dt=0.01, seed=3, rel_cutoff=0.0,
                                              precision=prec))
        f.init_walkers(s.initial_positions(W, seed=1))
        st = f.run_steps(0, 6)
        print("ok", st.n_moves)
        f.close()
    elif name == "refresh_100e":
        s = make_system("mixed_20nuc_100e", seed=1)
        W = 16384
        f = QMCB200Functions(s, W, run_params(sampling=1, qf_modification=2, dt=0.01, seed=3, rel_cutoff=0.0,
                                              refresh_interval=50))
        f.init_walkers(s.initial_positions(W, seed=1))
        st = f.run_steps(0, 50)
        print("ok", st.n_moves)
        f.close()
    else:
        raise SystemExit(f"unknown case {name}")




def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40, help="timed bench steps (whole DMC blocks, 150 moves each)")
    ap.add_argument("--warmup", type=int, default=3, help="untimed bench steps (whole DMC blocks)")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--walkers", type=int, default=DEFAULT_WALKERS)
    ap.add_argument("--e2e-steps", type=int, default=2, help="bench steps timed end to end, one API call per move")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the precision, rows, serving and batching sections")
    ap.add_argument("--c3-walkers", type=int, default=65536, help="walkers of the 100-electron precision workload")
    ap.add_argument("--section", choices=["precision", "rows", "serving", "batching"],
                    help="run one extra section alone and print it")
    ap.add_argument("--serve-jobs", type=int, default=12)
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--case", choices=["multidet_small", "group_small", "rows_small", "rows_bf16x3_small",
                                       "refresh_100e"],
                    help="run one small profiling workload instead of the benchmark")
    args = ap.parse_args()
    if args.case:
        profile_case(args.case)
        return
    if args.section:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        fn = {"precision": precision_section, "rows": rows_section, "serving": lambda a, r: serving_section(a),
              "batching": lambda a, r: batching_section(a)}[args.section]
        print(json.dumps({args.section: fn(args, 0)}))
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

    # reference-facing evaluate (QMCFunctions::evaluate shape) with host
    # buffers: qmcb_evaluate_moved sends the moved electron's position up and
    # brings back what a Metropolis driver reads after the call (psi, the
    # modified drift of every electron for the Green's functions, E_L, the
    # kinetic and potential terms, the singular flag), into page-locked host
    # arrays; next to it the all-positions qmcb_evaluate with every output
    from qmcbeaver_b200.api import OUT_E_LOCAL, OUT_LAP, OUT_MOD_GRAD, OUT_PE, OUT_PSI, OUT_STATUS
    nW = min(W, 4096)
    slots = torch.arange(nW, dtype=torch.int32).pin_memory().numpy()
    Rh = np.ascontiguousarray(R_eq[:nW])
    f2 = QMCB200Functions(system, nW, dmc_params(seed=1, e0=e0))
    f2.evaluate(slots, Rh, -1)
    pin = {k: torch.zeros(shape, dtype=dt).pin_memory().numpy() for k, shape, dt in
           (("log_abs_psi", (nW,), torch.float64), ("sign", (nW,), torch.float64),
            ("grad", (nW, N, 3), torch.float64), ("mod_grad", (nW, N, 3), torch.float64),
            ("lap", (nW,), torch.float64), ("e_local", (nW,), torch.float64), ("pe", (nW, 3), torch.float64),
            ("status", (nW,), torch.uint8))}
    mask = OUT_PSI | OUT_MOD_GRAD | OUT_LAP | OUT_E_LOCAL | OUT_PE | OUT_STATUS
    rng = np.random.default_rng(5)
    n_eval = 2 * N
    disp = 0.1 * rng.standard_normal((n_eval, nW, 3))
    # the driver's proposals, prepared in page-locked memory before the timed
    # loop; the loop calls the C entry point with the argument pointers a
    # compiled driver would pass (ctypes, pointers taken once)
    r_up = torch.zeros((n_eval, nW, 3), dtype=torch.float64).pin_memory().numpy()
    for s in range(n_eval):
        r_up[s] = Rh[:, s % N] + disp[s]
    lib2 = f2.lib
    out_ptrs = [pin[k].ctypes.data for k in ("log_abs_psi", "sign", "grad", "mod_grad", "lap", "e_local", "pe",
                                             "status")]
    slots_ptr, r_ptr = slots.ctypes.data, r_up.ctypes.data
    rc = lib2.qmcb_evaluate_moved(f2.h, 0, slots_ptr, nW, r_ptr, mask, *out_ptrs)  # untimed: first launches
    t0 = time.perf_counter()
    for s in range(n_eval):
        rc |= lib2.qmcb_evaluate_moved(f2.h, s % N, slots_ptr, nW, r_ptr + s * nW * 24, mask, *out_ptrs)
    ev_s = time.perf_counter() - t0
    if rc:
        raise RuntimeError(lib2.qmcb_last_error(f2.h))
    t0 = time.perf_counter()
    for s in range(n_eval):
        e = s % N
        Rh[:, e] += disp[s]
        f2.evaluate(slots, Rh, e)
    full_s = time.perf_counter() - t0
    f2.close()
    e2e_eval = {"value": nW * n_eval / ev_s, "unit": "walker-moves/s", "walkers": nW,
                "h2d_bytes_per_step": nW * (3 * 8 + 4),
                "d2h_bytes_per_step": nW * (3 * N * 8 + 7 * 8 + 1),
                "api": "qmcb_evaluate_moved(which_e, moved electron's position, outputs psi | mod_grad | lap | "
                       "e_local | pe | status) per single-electron move through the C ABI; slots, positions and "
                       "every output in page-locked host arrays (the drifts stored by the kernel over the bus, "
                       "the per-walker values by one packet-wide store kernel)",
                "all_positions_all_outputs": {
                    "value": nW * n_eval / full_s, "unit": "walker-moves/s",
                    "h2d_bytes_per_step": nW * (3 * N * 8 + 4), "d2h_bytes_per_step": nW * (6 * N * 8 + 7 * 8 + 1),
                    "api": "qmcb_evaluate(which_e, host R[num][N][3]) with every output, pageable numpy arrays"}}

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
        out["precision"] = precision_section(args, rank)
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
