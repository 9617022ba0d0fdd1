"""Python host side of the walker path over the C ABI (include/qmcb200.h).

:class:`QMCB200Functions` mirrors QMcBeaver's ``QMCFunctions`` interface
(QMcBeaver/include/QMCFunctions.h:67-70): ``evaluate`` takes a batch of walker
slots and electron positions and returns psi, grad(psi)/psi, lap(psi)/psi
and the local energy; ``run_steps`` runs the Metropolis / DMC steps of
QMCRun::step (QMcBeaver/src/QMCRun.cpp:1179-1236) on device-resident
walkers.  Every call goes through libqmcb200.so; there is no CPU fallback,
and a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional, Sequence

import numpy as np

from .desc import (QMCB_DMC, QMCB_VMC, PackedSystem, RunParams, StepStats, run_params)
from .system import MolecularSystem

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libqmcb200.so")

# Every symbol declared in include/qmcb200.h.
EXPORTS = [
    "qmcb_version", "qmcb_last_error", "qmcb_create", "qmcb_destroy", "qmcb_set_params", "qmcb_get_params",
    "qmcb_num_electrons", "qmcb_max_walkers", "qmcb_evaluate", "qmcb_evaluate_device", "qmcb_init_walkers",
    "qmcb_run_steps", "qmcb_num_walkers", "qmcb_get_walkers", "qmcb_copy_slot", "qmcb_synchronize",
    "qmcb_stream", "qmcb_set_walker_weights", "qmcb_branch", "qmcb_set_profiling", "qmcb_get_kernel_stats",
    "qmcb_branch_weights_noalloc", "qmcb_run_steps_async", "qmcb_steps_done", "qmcb_steps_collect",
    "qmcb_state_bytes", "qmcb_fit_cusps", "qmcb_run_step_configs",
    "qmcb_group_create", "qmcb_group_destroy", "qmcb_group_last_error", "qmcb_group_run_steps", "qmcb_group_config",
    "qmcb_group_set_config", "qmcb_evaluate_moved", "qmcb_alloc_slot", "qmcb_free_slot", "qmcb_get_rows",
]

# qmcb_evaluate_moved output selection (QMCB_OUT_*)
OUT_PSI, OUT_GRAD, OUT_MOD_GRAD, OUT_LAP, OUT_E_LOCAL, OUT_PE, OUT_STATUS = 1, 2, 4, 8, 16, 32, 64
OUT_ALL = 127

KERNELS = ["move", "branch", "copy", "energy", "refresh", "rows_prep", "rows_mma"]

_lib: Optional[C.CDLL] = None


class QMCBError(RuntimeError):
    pass


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libqmcb200.so (built by qmcbeaver_b200.build); raises when absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise QMCBError(f"{path} not found: run qmcbeaver_b200.build.build() (nvcc, sm_100a)")
    L = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.qmcb_version.restype = C.c_char_p
    L.qmcb_last_error.restype = C.c_char_p
    L.qmcb_last_error.argtypes = [vp]
    L.qmcb_create.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.qmcb_fit_cusps.argtypes = [vp, C.c_int, vp]
    L.qmcb_destroy.argtypes = [vp]
    L.qmcb_set_params.argtypes = [vp, vp]
    L.qmcb_get_params.argtypes = [vp, vp]
    L.qmcb_num_electrons.argtypes = [vp]
    L.qmcb_max_walkers.argtypes = [vp]
    L.qmcb_evaluate.argtypes = [vp, C.c_int, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.qmcb_evaluate_device.argtypes = [vp, C.c_int, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.qmcb_evaluate_moved.argtypes = [vp, C.c_int, vp, C.c_int, vp, C.c_uint, vp, vp, vp, vp, vp, vp, vp, vp]
    L.qmcb_alloc_slot.argtypes = [vp, C.POINTER(C.c_int)]
    L.qmcb_get_rows.argtypes = [vp, C.c_int, C.POINTER(C.c_int), vp]
    L.qmcb_free_slot.argtypes = [vp, C.c_int]
    L.qmcb_init_walkers.argtypes = [vp, C.c_int, vp]
    L.qmcb_run_steps.argtypes = [vp, C.c_int, C.c_int, vp]
    L.qmcb_num_walkers.argtypes = [vp]
    L.qmcb_get_walkers.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
    L.qmcb_copy_slot.argtypes = [vp, C.c_int, C.c_int]
    L.qmcb_synchronize.argtypes = [vp]
    L.qmcb_stream.argtypes = [vp]
    L.qmcb_stream.restype = vp
    L.qmcb_set_walker_weights.argtypes = [vp, C.c_int, vp]
    L.qmcb_branch.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
    L.qmcb_set_profiling.argtypes = [vp, C.c_int]
    L.qmcb_get_kernel_stats.argtypes = [vp, vp, C.c_int]
    L.qmcb_run_steps_async.argtypes = [vp, C.c_int, C.c_int]
    L.qmcb_group_create.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.qmcb_group_destroy.argtypes = [vp]
    L.qmcb_group_last_error.argtypes = [vp]
    L.qmcb_group_last_error.restype = C.c_char_p
    L.qmcb_group_run_steps.argtypes = [vp, vp, C.c_int, vp]
    L.qmcb_group_config.argtypes = [vp, vp, vp, vp, vp, vp]
    L.qmcb_group_set_config.argtypes = [vp, C.c_int]
    L.qmcb_run_step_configs.argtypes = [vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int), vp]
    L.qmcb_steps_done.argtypes = [vp]
    L.qmcb_steps_collect.argtypes = [vp, vp]
    L.qmcb_state_bytes.argtypes = [vp]
    L.qmcb_state_bytes.restype = C.c_size_t
    L.qmcb_branch_weights_noalloc.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_int, vp, vp, vp,
                                              vp]
    _lib = L
    return L


def _ptr(a: Optional[np.ndarray]):
    # the address as an int: ctypes.data_as builds a pointer object per call
    # (microseconds each, a tenth of a single-electron evaluate at 4,096
    # walkers); the caller keeps the array alive across the call
    return None if a is None else a.ctypes.data


class QMCB200Functions:
    """Walker-batch evaluator with device-resident walker state.

    ``evaluate(slots, R, which_e)`` is ``QMCFunctions::evaluate`` for the walkers
    stored in ``slots`` (QMcBeaver/src/QMCSCFJastrow.cpp:91-181): which_e = -1
    evaluates all electrons (LU inverse), which_e = e updates electron e
    (Sherman-Morrison) on top of the slot's stored state.
    """

    def __init__(self, system: MolecularSystem, max_walkers: int, params: Optional[RunParams] = None, **kw):
        self.lib = load_library()
        self.system = system
        self.N = system.n_electrons
        self.packed = PackedSystem(system)
        h = C.c_void_p()
        rc = self.lib.qmcb_create(C.byref(self.packed.desc), int(max_walkers), C.byref(h))
        if rc != 0:
            raise QMCBError(f"qmcb_create failed ({rc}): {self.lib.qmcb_last_error(None).decode()}")
        self.h = h
        self.max_walkers = int(max_walkers)
        self.set_params(params if params is not None else run_params(**kw))

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise QMCBError(f"{what} failed ({rc}): {self.lib.qmcb_last_error(self.h).decode()}")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.qmcb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: RunParams) -> None:
        self.params = p
        self._check(self.lib.qmcb_set_params(self.h, C.byref(p)), "qmcb_set_params")

    # ---------------------------------------------------------------- evaluate
    def evaluate(self, slots: Sequence[int], R: np.ndarray, which_e: int = -1) -> Dict[str, np.ndarray]:
        slots_a = np.ascontiguousarray(slots, dtype=np.int32)
        num = len(slots_a)
        R = np.ascontiguousarray(R, dtype=np.float64).reshape(num, self.N, 3)
        out = dict(
            log_abs_psi=np.zeros(num), sign=np.zeros(num), grad=np.zeros((num, self.N, 3)),
            mod_grad=np.zeros((num, self.N, 3)), lap=np.zeros(num), e_local=np.zeros(num),
            pe=np.zeros((num, 3)), status=np.zeros(num, np.uint8))
        rc = self.lib.qmcb_evaluate(self.h, int(which_e), _ptr(slots_a), num, _ptr(R), _ptr(out["log_abs_psi"]),
                                    _ptr(out["sign"]), _ptr(out["grad"]), _ptr(out["mod_grad"]), _ptr(out["lap"]),
                                    _ptr(out["e_local"]), _ptr(out["pe"]), _ptr(out["status"]))
        self._check(rc, "qmcb_evaluate")
        out["potential"] = out["pe"][:, 0]
        out["ne"] = out["pe"][:, 1]
        out["ee"] = out["pe"][:, 2]
        out["kinetic"] = -0.5 * out["lap"]
        return out

    def evaluate_moved(self, slots: Sequence[int], r_moved: np.ndarray, which_e: int, out_mask: int = OUT_ALL,
                       out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """qmcb_evaluate_moved: electron which_e of every walker in `slots`
        moved to r_moved[num][3] (the other positions are the stored ones);
        returns the outputs selected in out_mask.  `out` may hold
        preallocated (for example page-locked) arrays to fill."""
        slots_a = np.ascontiguousarray(slots, dtype=np.int32)
        num = len(slots_a)
        r = np.ascontiguousarray(r_moved, dtype=np.float64).reshape(num, 3)
        if out is None:
            out = dict(log_abs_psi=np.zeros(num), sign=np.zeros(num), grad=np.zeros((num, self.N, 3)),
                       mod_grad=np.zeros((num, self.N, 3)), lap=np.zeros(num), e_local=np.zeros(num),
                       pe=np.zeros((num, 3)), status=np.zeros(num, np.uint8))
        rc = self.lib.qmcb_evaluate_moved(self.h, int(which_e), _ptr(slots_a), num, _ptr(r), int(out_mask),
                                          _ptr(out["log_abs_psi"]), _ptr(out["sign"]), _ptr(out["grad"]),
                                          _ptr(out["mod_grad"]), _ptr(out["lap"]), _ptr(out["e_local"]),
                                          _ptr(out["pe"]), _ptr(out["status"]))
        self._check(rc, "qmcb_evaluate_moved")
        return out

    def get_rows(self, num: int) -> np.ndarray:
        """qmcb_get_rows: the orbital rows [num][5][n] of the last
        single-electron move made in a tensor-core rows mode."""
        n = C.c_int()
        self._check(self.lib.qmcb_get_rows(self.h, 0, C.byref(n), None), "qmcb_get_rows")
        out = np.zeros((num, 5, n.value))
        self._check(self.lib.qmcb_get_rows(self.h, int(num), C.byref(n), _ptr(out)), "qmcb_get_rows")
        return out

    def alloc_slot(self) -> int:
        s = C.c_int()
        self._check(self.lib.qmcb_alloc_slot(self.h, C.byref(s)), "qmcb_alloc_slot")
        return s.value

    def free_slot(self, slot: int) -> None:
        self._check(self.lib.qmcb_free_slot(self.h, int(slot)), "qmcb_free_slot")

    # ------------------------------------------------------------ Markov chain
    def init_walkers(self, R: np.ndarray) -> None:
        R = np.ascontiguousarray(R, dtype=np.float64)
        self._check(self.lib.qmcb_init_walkers(self.h, int(R.shape[0]), _ptr(R)), "qmcb_init_walkers")

    def run_steps(self, first_step: int, n_steps: int) -> StepStats:
        st = StepStats()
        self._check(self.lib.qmcb_run_steps(self.h, int(first_step), int(n_steps), C.byref(st)), "qmcb_run_steps")
        return st

    def run_step_configs(self, step: int) -> "tuple[np.ndarray, StepStats]":
        """One step that also returns its configuration records (the
        reference's print_configs output; qmcb_run_step_configs): array
        [2 * live walkers][6N + 4] of R, lap(D)/D, grad(D)/D, ln J, PE,
        weight -- the trial walker (weight p) then the original (1 - p)."""
        n = self.num_walkers()
        rec = np.zeros((2 * max(n, 1), 6 * self.N + 4))
        cnt = C.c_int()
        st = StepStats()
        self._check(self.lib.qmcb_run_step_configs(self.h, int(step), _ptr(rec), n, C.byref(cnt), C.byref(st)),
                    "qmcb_run_step_configs")
        return rec[:cnt.value], st

    def run_steps_async(self, first_step: int, n_steps: int) -> None:
        self._check(self.lib.qmcb_run_steps_async(self.h, int(first_step), int(n_steps)), "qmcb_run_steps_async")

    def steps_done(self) -> bool:
        r = self.lib.qmcb_steps_done(self.h)
        if r < 0:
            self._check(-r, "qmcb_steps_done")
        return r == 1

    def steps_collect(self) -> StepStats:
        st = StepStats()
        self._check(self.lib.qmcb_steps_collect(self.h, C.byref(st)), "qmcb_steps_collect")
        return st

    def state_bytes(self) -> int:
        return int(self.lib.qmcb_state_bytes(self.h))

    def num_walkers(self) -> int:
        return int(self.lib.qmcb_num_walkers(self.h))

    def get_walkers(self, n: Optional[int] = None) -> Dict[str, np.ndarray]:
        n = self.num_walkers() if n is None else n
        out = dict(R=np.zeros((n, self.N, 3)), weight=np.zeros(n), e_local=np.zeros(n), log_abs_psi=np.zeros(n),
                   sign=np.zeros(n))
        rc = self.lib.qmcb_get_walkers(self.h, n, _ptr(out["R"]), _ptr(out["weight"]), _ptr(out["e_local"]),
                                       _ptr(out["log_abs_psi"]), _ptr(out["sign"]))
        self._check(rc, "qmcb_get_walkers")
        return out

    def copy_slot(self, src: int, dst: int) -> None:
        self._check(self.lib.qmcb_copy_slot(self.h, int(src), int(dst)), "qmcb_copy_slot")

    def set_walker_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float64)
        self._check(self.lib.qmcb_set_walker_weights(self.h, len(w), _ptr(w)), "qmcb_set_walker_weights")

    def branch(self, step: int) -> int:
        n = C.c_int()
        self._check(self.lib.qmcb_branch(self.h, int(step), C.byref(n)), "qmcb_branch")
        return n.value

    def set_profiling(self, on: bool) -> None:
        self._check(self.lib.qmcb_set_profiling(self.h, 1 if on else 0), "qmcb_set_profiling")

    def kernel_stats(self, reset: bool = False) -> Dict[str, Dict[str, float]]:
        buf = np.zeros(2 * len(KERNELS))
        self._check(self.lib.qmcb_get_kernel_stats(self.h, _ptr(buf), 1 if reset else 0), "qmcb_get_kernel_stats")
        return {k: {"ms": float(buf[2 * i]), "launches": int(buf[2 * i + 1])} for i, k in enumerate(KERNELS)}

    def synchronize(self) -> None:
        self._check(self.lib.qmcb_synchronize(self.h), "qmcb_synchronize")

    @property
    def stream(self) -> int:
        return int(self.lib.qmcb_stream(self.h) or 0)


class QMCB200Group:
    """Several handles (systems of different sizes, each with its own
    walkers) stepped together: one persistent launch per bucket of similar
    shared-memory need per step, the launch configuration tuned by timing
    the first batches, batches replayed as CUDA graphs (qmcb_group_*).
    The members keep their own state: get_walkers etc. on a member read what
    the group's steps left there."""

    def __init__(self, members: "list[QMCB200Functions]"):
        self.lib = load_library()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.h for m in self.members])
        g = C.c_void_p()
        rc = self.lib.qmcb_group_create(arr, len(self.members), C.byref(g))
        if rc != 0:
            raise QMCBError(f"qmcb_group_create failed ({rc}): {self.lib.qmcb_group_last_error(None).decode()}")
        self.g = g

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise QMCBError(f"{what} failed ({rc}): {self.lib.qmcb_group_last_error(self.g).decode()}")

    def close(self) -> None:
        if getattr(self, "g", None):
            self.lib.qmcb_group_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_steps(self, first_steps, n_steps: int) -> "list[StepStats]":
        """Member i runs steps first_steps[i] .. + n_steps - 1 (an int:
        the same first step for every member)."""
        n = len(self.members)
        if isinstance(first_steps, int):
            first_steps = [first_steps] * n
        fs = (C.c_int * n)(*[int(x) for x in first_steps])
        st = (StepStats * n)()
        self._check(self.lib.qmcb_group_run_steps(self.g, fs, int(n_steps), st), "qmcb_group_run_steps")
        return list(st)

    def config(self) -> Dict[str, int]:
        v = [C.c_int() for _ in range(5)]
        self._check(self.lib.qmcb_group_config(self.g, *[C.byref(x) for x in v]), "qmcb_group_config")
        return dict(zip(("n_configs", "chosen", "last", "n_buckets", "warps_per_block"), [x.value for x in v]))

    def set_config(self, config: int) -> None:
        self._check(self.lib.qmcb_group_set_config(self.g, int(config)), "qmcb_group_set_config")


def fit_cusps(system: MolecularSystem) -> "tuple[np.ndarray, np.ndarray]":
    """The electron-nucleus cusp replacement records of both spins
    (qmcb_fit_cusps; host only): arrays [n_nuclei][orbital rows][8] of rc,
    sgn0, C, alpha_0..alpha_4 for the mo_alpha / mo_beta rows."""
    from .desc import PackedSystem
    lib = load_library()
    p = PackedSystem(system)
    out = []
    for beta in (0, 1):
        rows = len(system.active_orbitals(bool(beta)))
        a = np.zeros((system.n_nuclei, max(rows, 1), 8))
        rc = lib.qmcb_fit_cusps(C.byref(p.desc), beta, a.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise QMCBError(lib.qmcb_last_error(None).decode())
        out.append(a[:, :rows])
    return out[0], out[1]


__all__ = ["QMCB200Functions", "QMCB200Group", "fit_cusps", "QMCBError", "load_library", "run_params", "QMCB_VMC", "QMCB_DMC", "EXPORTS"]
