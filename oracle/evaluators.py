"""ctypes front ends of the oracle (C restatement) and of the reference build.

TEST INFRASTRUCTURE ONLY.  Both expose the same calls:

    ev = OracleEvaluator(system, qf_mod=..., dt=...)   # or ReferenceEvaluator
    ws = ev.new_walkers(n)
    ev.evaluate(ws, R, which_e)          # QMCSCFJastrow::evaluate
    out = ev.results(ws)                 # dict of numpy arrays
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from typing import Dict, List, Optional

import numpy as np

from qmcbeaver_b200.desc import PackedSystem, QMCB_QF_NONE
from qmcbeaver_b200.system import MolecularSystem

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqmcref.so")
REF_EXE = os.path.join(HERE, "_ref", "QMcBeaver.x")
# The QMcBeaver source tree the checker builds and reads its input files from:
# QMCB_REFERENCE_TREE, else the read-only mount of the build container.  Every
# test and fixture script takes the location from here.
REFERENCE_TREE = os.environ.get("QMCB_REFERENCE_TREE") or "/root/reference/QMcBeaver"

SCALARS = ["e_local", "kinetic", "potential", "ne", "ee", "U", "U_xx", "D_xx", "det_a", "det_b", "singular",
           "log_abs_psi", "sign", "psi"]

QF_NAMES = {0: "none", 1: "umrigar93_equalelectrons", 2: "umrigar93_unequalelectrons"}


def build_port() -> str:
    """Compiles oracle/qmc_oracle.c (gcc) if the library is missing or stale."""
    src = os.path.join(HERE, "qmc_oracle.c")
    if not os.path.exists(PORT_SO) or os.path.getmtime(PORT_SO) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "port", "CXX=g++"])
    return PORT_SO


def reference_available() -> bool:
    return os.path.exists(REF_SO) or os.path.isdir(os.path.join(REFERENCE_TREE, "src"))


def build_reference() -> str:
    if not os.path.exists(REF_SO):
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", "CXX=/usr/bin/g++",
                               f"REF={REFERENCE_TREE}"])
    return REF_SO


class _Base:
    N: int

    def results(self, walkers) -> Dict[str, np.ndarray]:
        n = len(walkers)
        sc = np.zeros((n, 14))
        g = np.zeros((n, self.N, 3))
        mg = np.zeros((n, self.N, 3))
        buf = np.zeros(14)
        gb = np.zeros((self.N, 3))
        mb = np.zeros((self.N, 3))
        for i, w in enumerate(walkers):
            self._get(w, buf.ctypes.data_as(C.c_void_p), gb.ctypes.data_as(C.c_void_p),
                      mb.ctypes.data_as(C.c_void_p))
            sc[i] = buf
            g[i] = gb
            mg[i] = mb
        out = {k: sc[:, i].copy() for i, k in enumerate(SCALARS)}
        out["grad"] = g
        out["mod_grad"] = mg
        out["lap"] = -2.0 * out["kinetic"]
        return out


class OracleEvaluator(_Base):
    """The C restatement (oracle/qmc_oracle.c)."""

    def __init__(self, system: MolecularSystem, qf_mod: int = QMCB_QF_NONE, qf_a: float = 0.5, dt: float = 0.09):
        self.lib = C.CDLL(build_port())
        L = self.lib
        L.orc_system_new.restype = C.c_void_p
        L.orc_system_new.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.orc_walker_new.restype = C.c_void_p
        L.orc_walker_new.argtypes = [C.c_void_p]
        L.orc_walker_clone.restype = C.c_void_p
        L.orc_walker_clone.argtypes = [C.c_void_p]
        L.orc_walker_copy.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_walker_free.argtypes = [C.c_void_p]
        L.orc_evaluate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.orc_walker_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_walker_inverse.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_walker_slater_grad.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_walker_inverse_det.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.orc_walker_kappa.argtypes = [C.c_void_p]
        L.orc_walker_kappa.restype = C.c_double
        L.orc_basis_at.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        self.packed = PackedSystem(system)
        if system.replace_cusps:
            # the fitted replacement records come from the library's fit
            # (pinned against the reference's own fit by tests/test_cusp.py)
            from qmcbeaver_b200.api import fit_cusps
            self.packed.set_cusp_tables(*fit_cusps(system))
        self.system = system
        self.N = system.n_electrons
        self.sys = L.orc_system_new(C.byref(self.packed.desc), qf_mod, qf_a, dt)

    def new_walkers(self, n: int) -> List[int]:
        return [self.lib.orc_walker_new(self.sys) for _ in range(n)]

    def clone(self, w):
        return self.lib.orc_walker_clone(w)

    def copy(self, dst, src):
        self.lib.orc_walker_copy(dst, src)

    def free(self, ws):
        for w in ws:
            self.lib.orc_walker_free(w)

    def evaluate(self, walkers, R: np.ndarray, which_e: int) -> None:
        R = np.ascontiguousarray(R, np.float64)
        arr = (C.c_void_p * len(walkers))(*walkers)
        self.lib.orc_evaluate(self.sys, arr, R.ctypes.data_as(C.c_void_p), len(walkers), which_e)

    def _get(self, w, a, b, c):
        self.lib.orc_walker_get(w, a, b, c)

    def slater_grad(self, walkers) -> np.ndarray:
        """grad(D)/D [n][N][3], the Slater part of the drift (QMCWalkerData::D_x)."""
        out = np.zeros((len(walkers), self.N, 3))
        for i, w in enumerate(walkers):
            self.lib.orc_walker_slater_grad(w, out[i].ctypes.data_as(C.c_void_p))
        return out

    def inverse(self, w, beta: int, det: int = 0) -> np.ndarray:
        """Inverse Slater matrix of determinant `det` of one spin."""
        n = self.system.n_beta if beta else self.system.n_alpha
        out = np.zeros((n, n))
        self.lib.orc_walker_inverse_det(w, beta, det, out.ctypes.data_as(C.c_void_p))
        return out

    def kappa(self, walkers) -> np.ndarray:
        """Per walker: sum_c |termPR_c lap_c| / max(|lap(D)/D|, 1), the factor
        by which the determinant-weighted laplacian sum amplifies rounding
        (1 or less for one determinant)."""
        return np.array([self.lib.orc_walker_kappa(w) for w in walkers])

    def basis_at(self, r) -> np.ndarray:
        out = np.zeros((5, self.system.n_basis))
        r = np.ascontiguousarray(r, np.float64)
        self.lib.orc_basis_at(self.sys, r.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
        return out


class ReferenceEvaluator(_Base):
    """The reference QMcBeaver code itself (oracle/_ref/libqmcref.so), driven
    through its own QMCSCFJastrow::evaluate.  One system per process: the
    reference keeps its input in a global."""

    _loaded: Optional[str] = None

    def __init__(self, system: MolecularSystem, qf_mod: int = QMCB_QF_NONE, qf_a: float = 0.5, dt: float = 0.09,
                 max_batch: int = 256, ckmf_text: Optional[str] = None, one_e_per_iter: int = 1,
                 extra_flags: Optional[dict] = None):
        """`ckmf_text`: run this input (a reference .ckmf, flags patched for
        the batch size, the QF options and dt) instead of one written from
        `system`; `system` must then be the same input read by
        qmcbeaver_b200.ckmf.  `one_e_per_iter` = 0 selects the reference's
        all-electron evaluation path (full evaluations only).  `extra_flags`
        are further input flags (e.g. sampling_method for walker_move)."""
        if ReferenceEvaluator._loaded is not None:
            raise RuntimeError("the reference library holds one system per process")
        self.lib = C.CDLL(build_reference())
        L = self.lib
        L.ref_init.argtypes = [C.c_char_p]
        L.ref_walker_new.restype = C.c_void_p
        L.ref_walker_clone.restype = C.c_void_p
        L.ref_walker_clone.argtypes = [C.c_void_p]
        L.ref_walker_free.argtypes = [C.c_void_p]
        L.ref_evaluate.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.ref_walker_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_walker_inverse.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.ref_cusp_params.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.ref_walker_move.argtypes = [C.c_void_p, C.c_int, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
        self.system = system
        self.N = system.n_electrons
        self.max_batch = max_batch
        fd, path = tempfile.mkstemp(suffix=".ckmf")
        os.close(fd)
        flags = {"walkers_per_pass": max_batch, "number_of_walkers": max_batch,
                 "QF_modification_type": QF_NAMES[qf_mod],
                 "umrigar93_equalelectrons_parameter": float(qf_a), "dt": float(dt),
                 # read_flags starts the run at dt_equilibration (QMcBeaver/src/QMCFlags.cpp:915-916)
                 "dt_equilibration": float(dt)}
        flags.update(extra_flags or {})
        if ckmf_text is None:
            system.to_ckmf(path, flags)
        else:
            from qmcbeaver_b200.ckmf import patch_flags, strip_three_body
            flags.update({"replace_electron_nucleus_cusps": 1 if system.replace_cusps else 0,
                          "use_three_body_jastrow": 0,
                          "one_e_per_iter": int(one_e_per_iter),
                          "print_configs": 0, "optimize_Psi": 0})
            if not system.three_body:
                ckmf_text = strip_three_body(ckmf_text)
            with open(path, "w") as fh:
                fh.write(patch_flags(ckmf_text, flags))
        L.ref_init(path.encode())
        os.unlink(path)
        ReferenceEvaluator._loaded = path

    def new_walkers(self, n: int) -> List[int]:
        return [self.lib.ref_walker_new() for _ in range(n)]

    def clone(self, w):
        return self.lib.ref_walker_clone(w)

    def free(self, ws):
        for w in ws:
            self.lib.ref_walker_free(w)

    def evaluate(self, walkers, R: np.ndarray, which_e: int) -> None:
        R = np.ascontiguousarray(R, np.float64)
        for s in range(0, len(walkers), self.max_batch):
            chunk = walkers[s:s + self.max_batch]
            arr = (C.c_void_p * len(chunk))(*chunk)
            self.lib.ref_evaluate(arr, R[s:s + len(chunk)].ctypes.data_as(C.c_void_p), len(chunk), which_e)

    def _get(self, w, a, b, c):
        self.lib.ref_walker_get(w, a, b, c)

    def cusp_params(self, beta: int) -> np.ndarray:
        """The reference's own fitted cusp records [nucleus][orbital row][8]
        (rc, sgn0, C, alpha_0..alpha_4) of one spin."""
        rows = len(self.system.active_orbitals(bool(beta)))
        out = np.zeros((self.system.n_nuclei, rows, 8))
        buf = np.zeros(8)
        for i in range(self.system.n_nuclei):
            for k in range(rows):
                self.lib.ref_cusp_params(beta, i, k, buf.ctypes.data_as(C.c_void_p))
                out[i, k] = buf
        return out

    def walker_move(self, R0: np.ndarray, iteration: int, seed: int) -> Dict[str, np.ndarray]:
        """One move of the reference's own QMCWalker from R0[N][3] with the
        input's sampling_method (ref_walker_move): the proposed positions R,
        gf = [ln G(R -> R'), ln G(R' -> R), G(R' -> R) / G(R -> R')], the
        modified drift of the original (mg0) and trial (mg1) walkers, and
        the electron moved (whichE, -1 = all)."""
        R0 = np.ascontiguousarray(R0, np.float64)
        out = dict(R=np.zeros((self.N, 3)), gf=np.zeros(3), mg=np.zeros((2, self.N, 3)))
        e = self.lib.ref_walker_move(R0.ctypes.data_as(C.c_void_p), int(iteration), int(seed),
                                     out["R"].ctypes.data_as(C.c_void_p), out["gf"].ctypes.data_as(C.c_void_p),
                                     out["mg"].ctypes.data_as(C.c_void_p))
        out["whichE"] = e
        out["mg0"], out["mg1"] = out.pop("mg")
        return out

    def inverse(self, w, beta: int) -> np.ndarray:
        n = self.system.n_beta if beta else self.system.n_alpha
        out = np.zeros((n, n))
        self.lib.ref_walker_inverse(w, beta, out.ctypes.data_as(C.c_void_p))
        return out
