"""Multi-GPU layout of the walker path: independent walker populations, one
per rank (the reference's manager_worker MPI mode runs independent walker
populations per process and only reduces property accumulators,
QMcBeaver/src/QMCManager.cpp:318-355).

There is no data-path collective: each rank owns its walkers end to end.
The exchanges are the small reductions the reference also performs --
timing (max over ranks), walker-move counts, and the weighted energy sums
of QMCManager::gatherProperties / synchronizeDMCEnsemble -- done with
torch.distributed (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

from typing import Dict, Tuple

import torch
import torch.distributed as dist


def replica_seed(base: int, rank: int) -> int:
    """Distinct random streams per rank (the reference offsets SPRNG streams
    by rank, QMcBeaver/src/Random.cpp:98-100)."""
    return int(base) + 7919 * int(rank)


def _device() -> torch.device:
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def aggregate_timing(ms: float, moves: float) -> Tuple[float, float]:
    """(max time over ranks, total walker-moves) -- whole-job throughput is
    total / max."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms), float(moves)
    dev = _device()
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    m = torch.tensor([moves], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(m, op=dist.ReduceOp.SUM)
    return float(t.item()), float(m.item())


def reduce_energy(sum_w: float, sum_we: float, sum_we2: float, n_walkers: int,
                  weight: float) -> Dict[str, float]:
    """Ensemble energy over all ranks from the per-rank weighted sums
    (QMCManager::gatherProperties, QMcBeaver/src/QMCManager.cpp:318-338):
    mean, variance of the weighted local energy, total walkers and weight."""
    v = [sum_w, sum_we, sum_we2, float(n_walkers), weight]
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        t = torch.tensor(v, dtype=torch.float64, device=_device())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        v = [float(x) for x in t.tolist()]
    sw, swe, swe2, nw, wt = v
    mean = swe / sw if sw > 0 else float("nan")
    var = swe2 / sw - mean * mean if sw > 0 else float("nan")
    return {"energy": mean, "variance": var, "sum_weight": sw, "walkers": int(nw), "weight": wt}


def trial_energy(e_est: float, total_weight: float, target_weight: float, c: float) -> float:
    """E_T = E_est - c ln(W / W0) on the ensemble totals
    (QMCManager::updateTrialEnergy, QMcBeaver/src/QMCManager.cpp:2263-2310)."""
    import math
    ratio = total_weight / target_weight
    return e_est - c * (math.log(ratio) if ratio > 1e-250 else 0.0)
