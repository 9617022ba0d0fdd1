"""Serving loop: independent VMC energy jobs of different molecule sizes
admitted by device-memory footprint and run concurrently on one GPU.

Each job owns a handle (walker state, inverses and accumulators resident on
the device) and the handle's CUDA stream; the loop keeps every admitted job
busy with asynchronous step batches (``qmcb_run_steps_async``), so kernels
of different jobs overlap on the GPU, and admits new arrivals as soon as
slots and memory free up -- continuous batching at the job level.  A job is
one VMC energy evaluation (QMCManager::run on a variational input,
QMcBeaver/src/QMCManager.cpp:683-801): equilibration sweeps, then sweeps
until the blocked standard error of the energy reaches the job's target.

A job's random streams depend only on its own seed and walker slots, so its
energies are the same whether it runs alone or in a mix (up to the
summation order of the per-step ensemble sums).

With ``mode="group"`` the admitted jobs are instead stepped together: one
group (``qmcb_group_*``) over all active jobs runs a batch of
``batch_steps`` steps of every job in one persistent launch per bucket per
step, rebuilt whenever a job joins or leaves.  Each job's energy blocks
are then its batches (the same whether it runs alone or in a mix).
"""
from __future__ import annotations

import dataclasses
import math
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from .api import QMCB200Functions, QMCB200Group
from .desc import (QMCB_IMPORTANCE_SAMPLING, QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC, QMCB_PREC_FP64,
                   QMCB_PREC_INT8_SLICES, QMCB_QF_UMRIGAR93_UNEQUAL, QMCB_VMC, run_params)
from .system import MolecularSystem, make_random_molecule


@dataclasses.dataclass
class Job:
    job_id: int
    system: MolecularSystem
    walkers: int
    target_error: float
    seed: int = 1
    arrival: float = 0.0          # seconds after the start of the run
    dt: float = 0.01
    equil_sweeps: int = 5
    min_blocks: int = 16
    max_sweeps: int = 400
    precision: int = QMCB_PREC_FP64
    # filled while running
    energies: List[float] = dataclasses.field(default_factory=list)
    moves: float = 0.0
    admitted: Optional[float] = None
    finished: Optional[float] = None
    energy: Optional[float] = None
    error: Optional[float] = None

    @property
    def latency(self) -> Optional[float]:
        return None if self.finished is None else self.finished - self.arrival


def blocked_error(samples: Sequence[float], nblocks: int = 8) -> float:
    """Standard error of the mean from `nblocks` contiguous block means
    (the blocking idea of QMCProperty::newSample, QMcBeaver/src/QMCProperty.cpp:427-478)."""
    x = np.asarray(samples, np.float64)
    if len(x) < 2 * nblocks:
        return math.inf
    m = np.array([b.mean() for b in np.array_split(x, nblocks)])
    return float(m.std(ddof=1) / math.sqrt(len(m)))


def state_footprint(system: MolecularSystem, walkers: int, precision: int = QMCB_PREC_FP64) -> int:
    """Device bytes a job's handle allocates for its walker state
    (the per-walker block of the library, 2x walker capacity, 256-byte
    blocks): positions, Slater rows / derivatives / inverse per spin (two
    inverse copies for spins above 16 electrons), per-electron arrays,
    scalars; for the tensor-core rows modes also their operand planes, block
    scales and the step's rows (the library's qmcb_state_bytes)."""
    def pad4(x):
        return (x + 3) & ~3
    N, na, nb = system.n_electrons, system.n_alpha, system.n_beta
    ginv = max(na, nb) > 16  # inverses in HBM, two copies (kStagedInverseMax)
    words = pad4(3 * N)
    for n in (na, nb):
        words += pad4(n * n) + pad4(3 * n * n) + pad4(n * n) + (2 * pad4(n * n) if ginv else pad4(n * n))
    words += 4 * pad4(3 * N) + pad4(24)
    words = (words + 31) & ~31
    cap = 2 * walkers
    total = cap * words * 8
    if precision in (QMCB_PREC_INT8_SLICES, QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC):
        K = system.n_basis
        tiles = -(-cap // 25)                      # 25 walkers (125 of 128 rows) per tile
        total += 8 * cap * 5 * max(na, nb)         # the step's rows
        nt = [max(-(-n // 32), 1) for n in (na, nb)]  # 32-orbital tiles per spin
        if precision == QMCB_PREC_INT8_SLICES:
            ks = -(-K // 32)                       # 8 int8 digit planes, a scale per 32-function block
            total += sum(t * ks * (8 * 1024 + 32 * 8) for t in nt) + tiles * ks * (8 * 4096 + 128 * 8)
        else:
            ks = -(-K // 16)                       # hi / lo BF16 planes, 16 functions per K step
            total += sum(t * ks * 2 * 1024 for t in nt) + tiles * ks * 2 * 4096
    return total


def device_budget(fraction: float = 0.8) -> int:
    """Bytes of device memory the server may hand to walker state: a
    fraction of what the current device has free (cudaMemGetInfo)."""
    import torch
    free, _ = torch.cuda.mem_get_info()
    return int(fraction * free)


class Server:
    """Admits jobs in arrival order while the sum of their device footprints
    stays under `hbm_budget` bytes (default: 80% of the device memory free
    when the server starts) and at most `max_active` run at once."""

    def __init__(self, hbm_budget: Optional[int] = None, max_active: int = 16, mode: str = "streams",
                 batch_steps: int = 64):
        if mode not in ("streams", "group"):
            raise ValueError(f"unknown serving mode {mode!r}")
        self.hbm_budget = int(hbm_budget) if hbm_budget is not None else device_budget()
        self.max_active = int(max_active)
        self.mode = mode
        self.batch_steps = int(batch_steps)

    def _handle(self, job: Job) -> QMCB200Functions:
        # both modes refresh every 50 moves (in group mode a batch that holds
        # a refresh runs as launches instead of a captured graph)
        p = run_params(run_type=QMCB_VMC, sampling=QMCB_IMPORTANCE_SAMPLING,
                       qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=job.dt, refresh_interval=50,
                       seed=job.seed, precision=job.precision, rel_cutoff=0.0)
        f = QMCB200Functions(job.system, (2 if self.mode == "streams" else 1) * job.walkers, p)
        f.init_walkers(job.system.initial_positions(job.walkers, seed=job.seed))
        return f

    def _start(self, job: Job) -> Dict:
        N = job.system.n_electrons
        f = self._handle(job)
        f.run_steps_async(0, job.equil_sweeps * N)
        return {"f": f, "step": job.equil_sweeps * N, "phase": "equil", "N": N}

    def _finish(self, j: Job, t0: float) -> None:
        j.finished = time.perf_counter() - t0
        j.energy = float(np.mean(j.energies))
        j.error = blocked_error(j.energies)

    def _done(self, j: Job) -> bool:
        err = blocked_error(j.energies)
        return (len(j.energies) >= j.min_blocks and err <= j.target_error) or len(j.energies) >= j.max_sweeps

    def run(self, jobs: Sequence[Job], poll_sleep: float = 0.0) -> Dict[str, object]:
        if self.mode == "group":
            return self._run_group(jobs)
        pending = sorted(jobs, key=lambda j: j.arrival)
        queue: List[Job] = []
        active: Dict[int, Dict] = {}
        used = 0
        t0 = time.perf_counter()
        done: List[Job] = []
        total_moves = 0.0
        while pending or queue or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            # admission by device footprint (walkers + inverses + rows)
            while queue and len(active) < self.max_active:
                j = queue[0]
                need = state_footprint(j.system, j.walkers, j.precision)
                if active and used + need > self.hbm_budget:
                    break
                queue.pop(0)
                j.admitted = now
                active[j.job_id] = dict(self._start(j), job=j, need=need)
                used += need
            progressed = False
            for jid in list(active.keys()):
                a = active[jid]
                f, j = a["f"], a["job"]
                if not f.steps_done():
                    continue
                progressed = True
                st = f.steps_collect()
                if a["phase"] == "equil":
                    a["phase"] = "run"
                else:
                    j.moves += st.n_moves
                    total_moves += st.n_moves
                    if st.sum_weight > 0:
                        j.energies.append(st.sum_weight_energy / st.sum_weight)
                    if self._done(j):
                        self._finish(j, t0)
                        f.close()
                        used -= a["need"]
                        del active[jid]
                        done.append(j)
                        continue
                f.run_steps_async(a["step"], a["N"])
                a["step"] += a["N"]
            if not progressed and poll_sleep > 0:
                time.sleep(poll_sleep)
        return self._summary(done, total_moves, time.perf_counter() - t0)

    def _run_group(self, jobs: Sequence[Job]) -> Dict[str, object]:
        """Active jobs stepped together, batch_steps steps per batch; a job's
        first ceil(equil_sweeps N / batch_steps) batches equilibrate."""
        pending = sorted(jobs, key=lambda j: j.arrival)
        queue: List[Job] = []
        active: Dict[int, Dict] = {}
        used = 0
        t0 = time.perf_counter()
        done: List[Job] = []
        total_moves = 0.0
        group = None
        B = self.batch_steps
        while pending or queue or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            changed = False
            while queue and len(active) < self.max_active:
                j = queue[0]
                need = state_footprint(j.system, j.walkers, j.precision) // 2
                if active and used + need > self.hbm_budget:
                    break
                queue.pop(0)
                j.admitted = now
                eq = -(-j.equil_sweeps * j.system.n_electrons // B)
                active[j.job_id] = {"f": self._handle(j), "job": j, "need": need, "step": 0, "equil": eq}
                used += need
                changed = True
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                continue
            if changed or group is None:
                if group is not None:
                    group.close()
                order = list(active.keys())
                group = QMCB200Group([active[k]["f"] for k in order])
            stats = group.run_steps([active[k]["step"] for k in order], B)
            for k, st in zip(order, stats):
                a = active[k]
                a["step"] += B
                if a["equil"] > 0:
                    a["equil"] -= 1
                    continue
                j = a["job"]
                j.moves += st.n_moves
                total_moves += st.n_moves
                if st.sum_weight > 0:
                    j.energies.append(st.sum_weight_energy / st.sum_weight)
                if self._done(j):
                    self._finish(j, t0)
                    done.append(j)
            finished = [k for k in order if active[k]["job"].finished is not None]
            if finished:
                group.close()
                group = None
                for k in finished:
                    active[k]["f"].close()
                    used -= active[k]["need"]
                    del active[k]
        if group is not None:
            group.close()
        return self._summary(done, total_moves, time.perf_counter() - t0)

    @staticmethod
    def _summary(done: List[Job], total_moves: float, wall: float) -> Dict[str, object]:
        lat = np.array([j.latency for j in done])
        return {"jobs": len(done), "wall_s": wall, "walker_moves": total_moves,
                "walker_moves_per_s": total_moves / wall if wall > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "results": {j.job_id: (j.energy, j.error, len(j.energies)) for j in done}}


def make_jobs(n_jobs: int, rate: float, seed: int = 1, electrons=(4, 40), walkers=(256, 2048),
              target_error: float = 0.2, max_sweeps: int = 400, precision: int = QMCB_PREC_FP64,
              orbitals: str = "core") -> List[Job]:
    """Poisson arrivals at `rate` jobs/s of synthetic molecules drawn like the
    uneven-batching workload: even electron count uniform in `electrons`,
    basis size 4 N, N/5 nuclei with Z in {1, 6, 7, 8}, walkers uniform in
    `walkers`; orbitals "core" (approximate core-Hamiltonian orbitals) or
    "random" (orthonormalised random coefficients, cheap for large bases)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for i in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        ne = int(rng.integers(electrons[0] // 2, electrons[1] // 2 + 1)) * 2
        nn = max(1, ne // 5)
        box = 2.0 + 1.5 * nn ** (1.0 / 3.0) * 2.0
        sysm = make_random_molecule(ne, nn, 4 * ne, box, (1, 6, 7, 8), seed=seed * 1000 + i,
                                    min_sep=1.4, name=f"job{i}-{ne}e", orbitals=orbitals)
        W = int(rng.integers(walkers[0], walkers[1] + 1))
        jobs.append(Job(job_id=i, system=sysm, walkers=W, target_error=target_error, seed=seed * 7919 + i,
                        arrival=t, max_sweeps=max_sweeps, precision=precision))
    return jobs


def make_input_jobs(n_jobs: int, rate: float, system: MolecularSystem, seed: int = 1, walkers=(1024, 4096),
                    target_error: float = 1e-3, max_sweeps: int = 4000, min_blocks: int = 16,
                    equil_sweeps: int = 5, dt: float = 0.01) -> List[Job]:
    """Poisson arrivals at `rate` jobs/s of VMC energy jobs on one given
    system (for example one of the reference's input files), walkers uniform
    in `walkers`, each equilibrated for `equil_sweeps` all-electron sweeps
    (samples not kept) and run to `target_error` Hartree."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for i in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        W = int(rng.integers(walkers[0], walkers[1] + 1))
        jobs.append(Job(job_id=i, system=system, walkers=W, target_error=target_error, seed=seed * 7919 + i,
                        arrival=t, max_sweeps=max_sweeps, min_blocks=min_blocks, equil_sweeps=equil_sweeps,
                        dt=dt))
    return jobs

