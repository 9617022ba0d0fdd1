"""ctypes mirror of the C-ABI structs in include/qmcb200.h and the packing of
a :class:`~qmcbeaver_b200.system.MolecularSystem` into ``qmcb_system_desc``."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .system import PADE_MAX, MolecularSystem

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

# constants of include/qmcb200.h
QMCB_VMC, QMCB_DMC = 0, 1
QMCB_NO_IMPORTANCE_SAMPLING, QMCB_IMPORTANCE_SAMPLING, QMCB_UMRIGAR93_IMPORTANCE_SAMPLING = 0, 1, 2
QMCB_QF_NONE, QMCB_QF_UMRIGAR93_EQUAL, QMCB_QF_UMRIGAR93_UNEQUAL = 0, 1, 2
QMCB_EMOD_NONE, QMCB_EMOD_UMRIGAR93, QMCB_EMOD_MODIFIED_UMRIGAR93 = 0, 1, 2
QMCB_RW_SIMPLE_SYMMETRIC, QMCB_RW_SIMPLE_ASYMMETRIC, QMCB_RW_UMRIGAR93_PROBABILITY_WEIGHTED = 0, 1, 2
QMCB_PREC_FP64, QMCB_PREC_MIXED, QMCB_PREC_INT8_SLICES, QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC = 0, 1, 2, 3, 4
QMCB_ST_SINGULAR, QMCB_ST_NAN = 1, 2
QMCB_ECUT_NONE, QMCB_ECUT_UMRIGAR93, QMCB_ECUT_BDJM_PUSH88 = 0, 1, 2


class SystemDesc(C.Structure):
    _fields_ = [
        ("n_nuclei", C.c_int), ("nuc_xyz", _dp), ("nuc_charge", _dp),
        ("n_alpha", C.c_int), ("n_beta", C.c_int),
        ("n_basis", C.c_int), ("bf_atom", _ip), ("bf_powers", _ip), ("bf_nprim", _ip), ("bf_prim_offset", _ip),
        ("n_prim_total", C.c_int), ("prim_exponent", _dp), ("prim_coeff", _dp),
        ("mo_alpha", _dp), ("mo_beta", _dp),
        ("n_pade", C.c_int), ("pade_num", _dp), ("pade_den", _dp), ("pade_nnum", _ip), ("pade_nden", _ip),
        ("corr_type", _ip), ("corr_param", _dp),
        ("ee_pade", C.c_int * 3), ("en_pade_up", _ip), ("en_pade_dn", _ip),
        ("n_det", C.c_int), ("n_act_alpha", C.c_int), ("n_act_beta", C.c_int),
        ("det_occ_alpha", _ip), ("det_occ_beta", _ip), ("ci_coeff", _dp),
        ("replace_cusps", C.c_int), ("cusp_alpha", _dp), ("cusp_beta", _dp),
        ("n_tb", C.c_int), ("tb_nen", _ip), ("tb_nee", _ip), ("tb_C", _ip), ("tb_cutoff", _dp),
        ("tb_offset", _ip), ("tb_coeff", _dp), ("tb_pair", _ip),
    ]


class RunParams(C.Structure):
    _fields_ = [
        ("run_type", C.c_int), ("sampling", C.c_int), ("qf_modification", C.c_int), ("qf_equal_a", C.c_double),
        ("dt", C.c_double), ("dt_effective", C.c_double), ("energy_modification", C.c_int),
        ("reweighting", C.c_int), ("energy_trial", C.c_double), ("energy_estimated", C.c_double),
        ("branching_threshold", C.c_double), ("fusion_threshold", C.c_double),
        ("old_walker_acceptance", C.c_int), ("refresh_interval", C.c_int), ("precision", C.c_int),
        ("seed", C.c_uint64), ("population_control", C.c_double), ("target_walkers", C.c_int),
        ("reweight_start_step", C.c_int), ("energy_original", C.c_double), ("rel_cutoff", C.c_double),
        ("limit_branching", C.c_int), ("energy_cutoff", C.c_int), ("exact_single_electron_gf", C.c_int),
        ("dynamic_time_step", C.c_int), ("walker_deletion", C.c_int), ("equilibration_steps", C.c_int),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("sum_weight", C.c_double), ("sum_weight_energy", C.c_double), ("sum_weight_energy2", C.c_double),
        ("sum_accept", C.c_double), ("n_moves", C.c_double), ("final_weight", C.c_double),
        ("n_walkers", C.c_int), ("n_singular", C.c_int),
    ]


def run_params(**kw) -> RunParams:
    p = RunParams()
    p.run_type = QMCB_VMC
    p.sampling = QMCB_NO_IMPORTANCE_SAMPLING
    p.qf_modification = QMCB_QF_NONE
    p.qf_equal_a = 0.5
    p.dt = 0.09
    p.dt_effective = -1.0
    p.energy_modification = QMCB_EMOD_NONE
    p.reweighting = QMCB_RW_UMRIGAR93_PROBABILITY_WEIGHTED
    p.energy_trial = 0.0
    p.energy_estimated = 0.0
    p.branching_threshold = 2.0
    p.fusion_threshold = 0.45
    p.old_walker_acceptance = 50
    p.refresh_interval = 0
    p.precision = QMCB_PREC_FP64
    p.seed = 12345
    p.population_control = 1.0
    p.target_walkers = 0
    p.reweight_start_step = 100
    p.energy_original = 0.0
    p.rel_cutoff = 100.0
    p.limit_branching = 1
    p.energy_cutoff = QMCB_ECUT_NONE
    p.walker_deletion = 0
    p.equilibration_steps = 0
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    if p.dt_effective < 0:
        p.dt_effective = p.dt
    return p


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


class PackedSystem:
    """Owns the numpy buffers a ``qmcb_system_desc`` points into."""

    def __init__(self, s: MolecularSystem):
        self.system = s
        atom, pw, nprim, off, ex, co = s.flat_basis()
        npade, num, den, nn, nd, ee, en_up, en_dn, ctype, cparam = s.pade_tables()
        self._keep = dict(
            nuc_xyz=np.ascontiguousarray(s.coords, np.float64),
            nuc_z=np.ascontiguousarray(s.Z, np.float64),
            atom=atom, pw=np.ascontiguousarray(pw), nprim=nprim, off=off, ex=ex, co=co,
            mo_a=np.ascontiguousarray(s.mo_alpha(), np.float64),
            mo_b=np.ascontiguousarray(s.mo_beta(), np.float64) if s.n_beta else np.zeros((1, s.n_basis)),
            num=np.ascontiguousarray(num), den=np.ascontiguousarray(den), nn=nn, nd=nd,
            en_up=en_up, en_dn=en_dn, ctype=np.ascontiguousarray(ctype, np.int32),
            cparam=np.ascontiguousarray(cparam, np.float64),
            occ_a=np.ascontiguousarray(s.det_columns(False) if s.n_det > 1 else np.zeros(1), np.int32),
            occ_b=np.ascontiguousarray(s.det_columns(True) if s.n_det > 1 and s.n_beta else np.zeros(1), np.int32),
            ci=np.ascontiguousarray(s.ci_coeffs if s.n_det > 1 else np.ones(1), np.float64),
        )
        k = self._keep
        d = SystemDesc()
        d.n_nuclei = s.n_nuclei
        d.nuc_xyz = _d(k["nuc_xyz"])
        d.nuc_charge = _d(k["nuc_z"])
        d.n_alpha = s.n_alpha
        d.n_beta = s.n_beta
        d.n_basis = s.n_basis
        d.bf_atom = _i(k["atom"])
        d.bf_powers = _i(k["pw"])
        d.bf_nprim = _i(k["nprim"])
        d.bf_prim_offset = _i(k["off"])
        d.n_prim_total = len(k["ex"])
        d.prim_exponent = _d(k["ex"])
        d.prim_coeff = _d(k["co"])
        d.mo_alpha = _d(k["mo_a"])
        d.mo_beta = _d(k["mo_b"])
        d.n_pade = npade
        d.pade_num = _d(k["num"])
        d.pade_den = _d(k["den"])
        d.pade_nnum = _i(k["nn"])
        d.pade_nden = _i(k["nd"])
        d.corr_type = _i(k["ctype"])
        d.corr_param = _d(k["cparam"])
        for i in range(3):
            d.ee_pade[i] = int(ee[i])
        d.en_pade_up = _i(k["en_up"])
        d.en_pade_dn = _i(k["en_dn"])
        d.n_det = s.n_det
        d.n_act_alpha = len(s.active_orbitals(False))
        d.n_act_beta = len(s.active_orbitals(True))
        d.det_occ_alpha = _i(k["occ_a"])
        d.det_occ_beta = _i(k["occ_b"])
        d.ci_coeff = _d(k["ci"])
        d.replace_cusps = 1 if s.replace_cusps else 0
        tb = s.three_body_tables()
        self._keep.update({"tb_" + k: v for k, v in tb.items()})
        d.n_tb = int(len(tb["nen"])) if tb["used"] else 0
        d.tb_nen = _i(self._keep["tb_nen"])
        d.tb_nee = _i(self._keep["tb_nee"])
        d.tb_C = _i(self._keep["tb_C"])
        d.tb_cutoff = _d(self._keep["tb_cutoff"])
        d.tb_offset = _i(self._keep["tb_offset"])
        d.tb_coeff = _d(self._keep["tb_coeff"])
        d.tb_pair = _i(self._keep["tb_pair"])
        self.desc = d

    def set_cusp_tables(self, alpha: np.ndarray, beta: np.ndarray) -> None:
        """Passes fitted cusp records (qmcb_fit_cusps) instead of fitting again."""
        self._keep["cusp_a"] = np.ascontiguousarray(alpha, np.float64)
        self._keep["cusp_b"] = np.ascontiguousarray(beta, np.float64)
        self.desc.cusp_alpha = _d(self._keep["cusp_a"])
        self.desc.cusp_beta = _d(self._keep["cusp_b"])
        assert PADE_MAX == 16
