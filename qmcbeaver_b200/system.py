"""Molecular system description for the Slater-Jastrow walker path.

A :class:`MolecularSystem` holds exactly what QMcBeaver reads from the
``&geometry``, ``&basis``, ``&wavefunction`` and ``&Jastrow`` sections of a
``.ckmf`` input for a single-determinant, restricted, all-electron
calculation with Pade two-body Jastrows:

* nuclei: label, charge Z, position  (QMcBeaver/src/QMCMolecule.cpp, readGeometry)
* contracted Cartesian Gaussians per atom: type string (``s``, ``px``,
  ``dxy`` ...), primitive exponents and raw contraction coefficients
  (QMcBeaver/src/QMCBasisFunctionCoefficients.cpp:84-127; the coefficients
  are used as given, QMcBeaver/src/QMCBasisFunction.cpp:381, so any
  normalisation is folded in here)
* MO coefficients, orbital rows x basis columns, and the occupied orbitals of
  each spin (QMcBeaver/src/QMCWavefunction.cpp:873-905)
* Pade correlation functions u(r) = P(r) / Q(r), P(0) = 0, Q(0) = 1, for the
  up-down, up-up, down-down electron pairs and for each nucleus type
  (QMcBeaver/src/FixedCuspPadeCorrelationFunction.cpp:34-77)

It also generates the seeded synthetic molecules the benchmark and tests run
(:func:`make_system`) and writes them as ``.ckmf`` text so the reference CPU
code reads bit-identical doubles (``%.17g``).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

ELEMENT = {1: "H", 2: "He", 3: "Li", 4: "Be", 5: "B", 6: "C", 7: "N", 8: "O", 9: "F", 10: "Ne"}

SHELL_TYPES = {
    "s": ["s"],
    "p": ["px", "py", "pz"],
    "d": ["dxx", "dyy", "dzz", "dxy", "dxz", "dyz"],
}

PADE_MAX = 16  # coefficients per polynomial (degree <= 15), matches qmcb200.h
CORR_PADE, CORR_CAMBRIDGE2 = 0, 1


def type_to_powers(t: str) -> Tuple[int, int, int]:
    """Cartesian powers of a basis type string, as type_to_xyz
    (QMcBeaver/src/QMCBasisFunctionCoefficients.cpp:39-82)."""
    t = t.lower()
    lnames = "spdfghi"
    l = lnames.index(t[0])
    if len(t) - 1 != l:
        raise ValueError(f"basis type {t!r} does not have angular momentum {l}")
    return (t.count("x"), t.count("y"), t.count("z"))


@dataclasses.dataclass
class BasisFunction:
    type: str
    exponents: np.ndarray  # (P,)
    coefficients: np.ndarray  # (P,) raw, normalisation folded in

    @property
    def powers(self) -> Tuple[int, int, int]:
        return type_to_powers(self.type)


@dataclasses.dataclass
class Pade:
    """u(r) = sum_i num[i] r^i / sum_i den[i] r^i with num[0] = 0, den[0] = 1."""
    num: Sequence[float]
    den: Sequence[float]

    @staticmethod
    def fixed_cusp(cusp: float, b: float) -> "Pade":
        # FixedCuspPade with one numerator constant and one denominator
        # parameter: numerator [0, cusp], denominator [1, b]
        # (QMcBeaver/src/FixedCuspPadeCorrelationFunction.cpp:56-72).
        return Pade(num=[0.0, float(cusp)], den=[1.0, float(b)])

    def evaluate(self, r: float) -> Tuple[float, float, float]:
        """(u, u', u'') with the reference's operation order
        (QMcBeaver/src/FixedCuspPadeCorrelationFunction.cpp:89-111,
        QMcBeaver/src/Polynomial.cpp:127-148)."""
        a, ap, app = _poly_all(self.num, r)
        b, bp, bpp = _poly_all(self.den, r)
        aDIVb = a / b
        bpDIVb = bp / b
        apDIVb = ap / b
        f = aDIVb
        df = apDIVb - bpDIVb * aDIVb
        d2f = (app - bpp * aDIVb) / b - 2 * bpDIVb * df
        return f, df, d2f


@dataclasses.dataclass
class Cambridge2:
    """u(r) = (fL r - 1)^C alpha(fL r) for fL r <= 1, zero beyond, with alpha
    the polynomial of Cambridge2CorrelationFunction::initializeParameters
    (QMcBeaver/src/Cambridge2CorrelationFunction.cpp): alpha_0 = p[1],
    alpha_1 = g / (-1)^C / fL + alpha_0 C (g the cusp constant), alpha_i = p[i]."""
    fL: float
    C: int
    alpha: Sequence[float]
    active: bool = True
    # the input's own parameters (L, cusp constant g, scale f), kept for
    # writing the function back out; derived from fL / alpha when zero
    L: float = 0.0
    g: float = 0.0
    f: float = 1.0

    def input_parameters(self) -> Tuple[List[float], List[float]]:
        """(Parameters, Constants) of a ckmf block giving this function."""
        if self.L > 0.0 or not self.active:
            L, g, f = self.L, self.g, self.f
        else:
            L, f = self.fL, 1.0
            g = (self.alpha[1] - self.alpha[0] * self.C) * (-1.0) ** self.C * self.fL
        return [L, self.alpha[0]] + list(self.alpha[2:]), [g, float(self.C), 0.0, f]

    @staticmethod
    def from_parameters(params: Sequence[float], constants: Sequence[float], a_diag: float = -1e-5) -> "Cambridge2":
        g = float(constants[0])
        C = int(constants[1])
        f = float(constants[3]) if len(constants) >= 4 else 1.0
        L = float(params[0])
        fL = f * L
        active = not (L <= 0.0 or fL > 100.0)
        if not active and a_diag >= 0.0:
            raise ValueError(f"Cambridge2 with L = {L}")
        a0 = float(params[1])
        # an inactive function is never evaluated; its alpha_1 is left at 0
        a1 = g / (-1.0) ** C / fL + a0 * C if fL != 0.0 else 0.0
        a = [a0, a1] + [float(x) for x in params[2:]]
        return Cambridge2(fL=fL, C=C, alpha=a, active=active, L=L, g=g, f=f)

    def evaluate(self, r: float) -> Tuple[float, float, float]:
        if not self.active:
            return 0.0, 0.0, 0.0
        d = self.fL * r - 1.0
        if d > 0.0:
            return 0.0, 0.0, 0.0
        P, ap, app = _poly_all(self.alpha, self.fL * r)
        dP_r, dP_rr = self.fL * ap, self.fL * self.fL * app
        dpc = d ** self.C
        dpc_r = self.C * self.fL * dpc / d
        dpc_rr = (self.C - 1.0) * self.fL * dpc_r / d
        return dpc * P, dpc_r * P + dpc * dP_r, dpc_rr * P + dpc_r * dP_r * 2.0 + dpc * dP_rr


def _poly_all(c: Sequence[float], x: float) -> Tuple[float, float, float]:
    n = len(c) - 1
    f = c[n]
    df = 0.0
    d2f = 0.0
    for i in range(n - 1, -1, -1):
        d2f = d2f * x + df
        df = df * x + f
        f = f * x + c[i]
    return f, df, 2 * d2f


@dataclasses.dataclass
class MolecularSystem:
    labels: List[str]
    Z: np.ndarray  # (M,) float charges
    coords: np.ndarray  # (M,3)
    basis: List[List[BasisFunction]]  # per atom
    mo: np.ndarray  # (n_orb, K), orbital rows
    n_alpha: int
    n_beta: int
    alpha_occ: np.ndarray  # indices of occupied orbitals (alpha)
    beta_occ: np.ndarray
    ee_anti: Optional[Pade]
    ee_para_up: Optional[Pade]
    ee_para_dn: Optional[Pade]
    en_up: Dict[str, Pade]  # by nucleus label
    en_dn: Dict[str, Pade]
    name: str = "synthetic"
    # several determinants: rows of `mo` occupied by each determinant (each
    # row increasing) and the CI coefficients; None = the one determinant
    # alpha_occ / beta_occ
    det_alpha: Optional[np.ndarray] = None  # (n_det, n_alpha)
    det_beta: Optional[np.ndarray] = None   # (n_det, n_beta)
    ci_coeffs: Optional[np.ndarray] = None  # (n_det,)
    # electron-nucleus cusp replacement of the orbitals (replace_electron_nucleus_cusps)
    replace_cusps: bool = False
    # three-body (e-e-n) Jastrow per nucleus label: (up-down, up-up, down-down)
    three_body: Dict[str, tuple] = dataclasses.field(default_factory=dict)

    # ------------------------------------------------------------------ sizes
    @property
    def n_nuclei(self) -> int:
        return len(self.labels)

    @property
    def n_electrons(self) -> int:
        return self.n_alpha + self.n_beta

    @property
    def n_basis(self) -> int:
        return sum(len(fs) for fs in self.basis)

    @property
    def charge(self) -> int:
        return int(round(float(self.Z.sum()))) - self.n_electrons

    def flat_basis(self):
        """Flattened basis tables in the reference's function order
        (atoms in geometry order, functions in file order;
        QMcBeaver/src/QMCBasisFunction.cpp:177-201)."""
        atom, pw, nprim, off, ex, co = [], [], [], [], [], []
        for a, fs in enumerate(self.basis):
            for f in fs:
                atom.append(a)
                pw.append(f.powers)
                nprim.append(len(f.exponents))
                off.append(len(ex))
                ex.extend(float(v) for v in f.exponents)
                co.extend(float(v) for v in f.coefficients)
        return (np.asarray(atom, np.int32), np.asarray(pw, np.int32).reshape(-1, 3),
                np.asarray(nprim, np.int32), np.asarray(off, np.int32),
                np.asarray(ex, np.float64), np.asarray(co, np.float64))

    @property
    def n_det(self) -> int:
        return 1 if self.det_alpha is None else int(np.asarray(self.det_alpha).shape[0])

    def active_orbitals(self, beta: bool) -> np.ndarray:
        """Rows of `mo` used by some determinant of the spin, increasing
        (QMCWavefunction::makeCoefficients, QMcBeaver/src/QMCWavefunction.cpp:873-905)."""
        if self.det_alpha is None:
            return np.asarray(self.beta_occ if beta else self.alpha_occ)
        return np.unique(np.asarray(self.det_beta if beta else self.det_alpha))

    def det_columns(self, beta: bool) -> np.ndarray:
        """(n_det, n) active-row index of every determinant column."""
        act = self.active_orbitals(beta)
        occ = np.asarray(self.det_beta if beta else self.det_alpha).reshape(self.n_det, -1)
        return np.searchsorted(act, occ).astype(np.int32)

    def mo_alpha(self) -> np.ndarray:
        return np.ascontiguousarray(self.mo[self.active_orbitals(False)])

    def mo_beta(self) -> np.ndarray:
        return np.ascontiguousarray(self.mo[self.active_orbitals(True)])

    def three_body_tables(self) -> Dict[str, np.ndarray]:
        """Three-body function tables for the descriptor: distinct functions
        with their NeN, Nee, C, cutoff and coefficient offsets, and per nucleus
        (geometry order) the function of each pair kind (-1: none)."""
        funcs: List[object] = []
        pair = np.full((max(self.n_nuclei, 1), 3), -1, np.int32)
        for a, l in enumerate(self.labels):
            for kind, f in enumerate(self.three_body.get(l, (None, None, None))):
                if f is None:
                    continue
                for i, g in enumerate(funcs):
                    if g is f:
                        pair[a, kind] = i
                        break
                else:
                    funcs.append(f)
                    pair[a, kind] = len(funcs) - 1
        nen = np.array([f.nen for f in funcs] or [0], np.int32)
        nee = np.array([f.nee for f in funcs] or [0], np.int32)
        Cs = np.array([f.C for f in funcs] or [0], np.int32)
        cut = np.array([f.cutoff for f in funcs] or [0.0], np.float64)
        off = np.cumsum([0] + [len(f.coeffs) for f in funcs])[:-1].astype(np.int32) if funcs else np.zeros(1, np.int32)
        coef = np.concatenate([np.asarray(f.coeffs, np.float64) for f in funcs]) if funcs else np.zeros(1)
        return dict(used=bool(funcs), nen=nen, nee=nee, C=Cs, cutoff=cut, offset=off,
                    coeff=np.ascontiguousarray(coef), pair=np.ascontiguousarray(pair.reshape(-1)))

    def pade_tables(self):
        """Correlation-function table + indices: ee[3] = (anti, up-up, dn-dn),
        en_up[M], en_dn[M]; -1 means no correlation function for that pair.
        Returns (n, num, den, nnum, nden, ee, en_up, en_dn, ctype, cparam)."""
        funcs: List[object] = []

        def add(p) -> int:
            if p is None:
                return -1
            funcs.append(p)
            return len(funcs) - 1

        ee = [add(self.ee_anti), add(self.ee_para_up), add(self.ee_para_dn)]
        en_up = [add(self.en_up.get(l)) for l in self.labels]
        en_dn = [add(self.en_dn.get(l)) for l in self.labels]
        nfun = max(1, len(funcs))
        num = np.zeros((nfun, PADE_MAX))
        den = np.zeros((nfun, PADE_MAX))
        nn = np.zeros(nfun, np.int32)
        nd = np.zeros(nfun, np.int32)
        ctype = np.zeros(nfun, np.int32)
        cparam = np.zeros((nfun, 4))
        for i, p in enumerate(funcs):
            if isinstance(p, Cambridge2):
                if len(p.alpha) > PADE_MAX:
                    raise ValueError("Cambridge2 polynomial too long")
                num[i, : len(p.alpha)] = p.alpha
                nn[i] = len(p.alpha)
                den[i, 0] = 1.0
                nd[i] = 1
                ctype[i] = CORR_CAMBRIDGE2
                cparam[i] = (p.fL, float(p.C), 1.0 if p.active else 0.0, 0.0)
            else:
                if len(p.num) > PADE_MAX or len(p.den) > PADE_MAX:
                    raise ValueError("Pade polynomial too long")
                num[i, : len(p.num)] = p.num
                den[i, : len(p.den)] = p.den
                nn[i] = len(p.num)
                nd[i] = len(p.den)
        return (len(funcs), num, den, nn, nd, np.asarray(ee, np.int32),
                np.asarray(en_up, np.int32), np.asarray(en_dn, np.int32), ctype, cparam)

    def nuclear_repulsion(self) -> float:
        """V_nn as calc_P_nn (QMcBeaver/src/QMCPotential_Energy.cpp:285-307)."""
        v = 0.0
        M = self.n_nuclei
        for i in range(M):
            for j in range(i + 1, M):
                d = self.coords[i] - self.coords[j]
                r = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
                v += (self.Z[i] * self.Z[j]) / r
        return float(v)

    def check_exponent_cache(self) -> None:
        """The reference reuses exp(-a r^2) when consecutive primitives share an
        exponent, and the cache is not reset between atoms
        (QMcBeaver/src/QMCBasisFunction.cpp:310,372-379).  A system where the
        last exponent of one atom equals the first exponent of the next would
        make the reference reuse a stale value; refuse such systems."""
        prev_last = None
        for fs in self.basis:
            if not fs:
                continue
            first = float(fs[0].exponents[0])
            if prev_last is not None and abs(prev_last - first) <= 1e-10:
                raise ValueError("exponent shared across atom boundary (stale exp cache in reference)")
            prev_last = float(fs[-1].exponents[-1])

    # ------------------------------------------------------------ positions
    def initial_positions(self, n_walkers: int, seed: int = 1, sigma: float = 0.8) -> np.ndarray:
        """Electrons placed by Gaussians around nuclei, electron e on nucleus
        e-th in a charge-weighted round robin.  Returns (W, N, 3) float64."""
        rng = np.random.default_rng(seed)
        order: List[int] = []
        zs = [max(1, int(round(z))) for z in self.Z]
        left = list(zs)
        while len(order) < self.n_electrons:
            progressed = False
            for a in range(self.n_nuclei):
                if left[a] > 0 and len(order) < self.n_electrons:
                    order.append(a)
                    left[a] -= 1
                    progressed = True
            if not progressed:
                left = list(zs)
        # alternate spins over nuclei: alpha electrons take even slots
        a_slots = order[0::2][: self.n_alpha]
        b_slots = order[1::2][: self.n_beta]
        while len(a_slots) < self.n_alpha:
            a_slots.append(order[len(a_slots) % len(order)])
        while len(b_slots) < self.n_beta:
            b_slots.append(order[len(b_slots) % len(order)])
        centers = self.coords[np.asarray(a_slots + b_slots)]
        R = centers[None, :, :] + sigma * rng.standard_normal((n_walkers, self.n_electrons, 3))
        return np.ascontiguousarray(R, dtype=np.float64)

    # ------------------------------------------------------------ ckmf text
    def to_ckmf(self, path: str, flags: Optional[Dict[str, object]] = None) -> None:
        """Writes a QMcBeaver input with the sections the reference parses:
        &flags (key line / value line, QMcBeaver/src/QMCFlags.cpp:198-206),
        &geometry, &basis, &wavefunction, &Jastrow."""
        f = dict(DEFAULT_FLAGS)
        # up and down electrons share parameters only when their functions
        # agree (QMcBeaver/src/QMCJastrowParameters.cpp:880-900)
        linked = (self.ee_para_dn == self.ee_para_up or self.n_beta < 2) and \
            (self.n_beta == 0 or self.en_dn == self.en_up)
        f.update({
            "link_Jastrow_parameters": 1 if linked else 0,
            "replace_electron_nucleus_cusps": 1 if self.replace_cusps else 0,
            # three-body blocks are written per pair kind with coefficients
            # that already satisfy the Gaussian-elimination constraints
            "use_three_body_jastrow": 1 if self.three_body else 0,
            "link_NEE_Jastrows": 0,
            "reproduce_NE_with_NEE_jastrow": 1,
            "reproduce_EE_with_NEE_jastrow": 1,
            "atoms": self.n_nuclei,
            "charge": self.charge,
            "norbitals": self.mo.shape[0],
            "nbasisfunc": self.n_basis,
            "ndeterminants": self.n_det,
            "trial_function_type": "restricted",
        })
        if flags:
            f.update(flags)
        g = "%.17g"
        out: List[str] = ["# synthetic system " + self.name, "", "&flags"]
        for k, v in f.items():
            out.append(k)
            out.append(" " + (g % v if isinstance(v, float) else str(v)))
        out.append("&")
        out.append("&geometry")
        for l, z, c in zip(self.labels, self.Z, self.coords):
            out.append(f"{l} {int(round(z))} {g % c[0]} {g % c[1]} {g % c[2]}")
        out.append("&")
        out.append("&basis")
        for l, fs in zip(self.labels, self.basis):
            maxg = max(len(b.exponents) for b in fs)
            out.append(f"{l} {len(fs)} {maxg}")
            for b in fs:
                out.append(f"  {len(b.exponents)} {b.type}")
                for e, c in zip(b.exponents, b.coefficients):
                    out.append(f"    {g % e} {g % c}")
        out.append("&")
        out.append("&wavefunction")
        for row in self.mo:
            out.append(" ".join(g % v for v in row))
        out.append("")
        dets_a = [self.alpha_occ] if self.det_alpha is None else list(self.det_alpha)
        dets_b = [self.beta_occ] if self.det_beta is None else list(self.det_beta)
        for title, dets in (("Alpha Occupation", dets_a), ("Beta Occupation", dets_b)):
            out.append(title)
            for occ in dets:
                row = np.zeros(self.mo.shape[0], int)
                row[np.asarray(occ, int)] = 1
                out.append(" ".join(str(v) for v in row))
            out.append("")
        out.append("CI Coeffs")
        ci = [1.0] if self.ci_coeffs is None else list(self.ci_coeffs)
        out.append(" ".join(g % v for v in ci))
        out.append("")
        out.append("&")
        out.append("")
        out.append("&Jastrow")

        def block(p1: str, p2: str, p) -> None:
            out.append(f"ParticleTypes:\t{p1}\t{p2}")
            if isinstance(p, Cambridge2):
                params, consts = p.input_parameters()
                out.append("CorrelationFunctionType:\tCambridge2")
                out.append("NumberOfParameterTypes:\t2")
                out.append(f"NumberOfParametersOfEachType:\t1\t{len(params) - 1}")
                out.append("Parameters:\t" + "\t".join(g % v for v in params))
                out.append("NumberOfConstantTypes:\t4")
                out.append("NumberOfConstantsOfEachType:\t1\t1\t1\t1")
                out.append("Constants:\t" + "\t".join(g % v for v in consts))
                out.append("")
                return
            # FixedCuspPade: numerator [0, constant, parameters of type 0],
            # denominator [1, parameters of type 1]
            if len(p.num) < 2 or p.num[0] != 0.0 or p.den[0] != 1.0:
                raise ValueError("ckmf writer needs u = (c r + ...) / (1 + ...)")
            nparams, dparams = list(p.num[2:]), list(p.den[1:])
            out.append("CorrelationFunctionType:\tFixedCuspPade")
            out.append("NumberOfParameterTypes:\t2")
            out.append(f"NumberOfParametersOfEachType:\t{len(nparams)}\t{len(dparams)}")
            out.append("Parameters:\t" + "\t".join(g % v for v in nparams + dparams))
            out.append("NumberOfConstantTypes:\t1")
            out.append("NumberOfConstantsOfEachType:\t1")
            out.append("Constants:\t" + g % p.num[1])
            out.append("")

        if self.ee_anti is not None and self.n_alpha > 0 and self.n_beta > 0:
            block("Electron_up", "Electron_down", self.ee_anti)
        if self.ee_para_up is not None and self.n_alpha > 1:
            block("Electron_up", "Electron_up", self.ee_para_up)
        if self.ee_para_dn is not None and self.n_beta > 1:
            block("Electron_down", "Electron_down", self.ee_para_dn)
        for l in dict.fromkeys(self.labels):
            if l in self.en_up:
                block("Electron_up", l, self.en_up[l])
            if l in self.en_dn and self.n_beta > 0:
                block("Electron_down", l, self.en_dn[l])
        kinds = (("Electron_up", "Electron_down"), ("Electron_up", "Electron_up"), ("Electron_down", "Electron_down"))
        for l in dict.fromkeys(self.labels):
            for (p2, p3), tb in zip(kinds, self.three_body.get(l, (None, None, None))):
                if tb is None or (p2 == p3 == "Electron_up" and self.n_alpha < 2) or \
                        (p2 == p3 == "Electron_down" and self.n_beta < 2) or \
                        (p2 != p3 and (self.n_alpha < 1 or self.n_beta < 1)):
                    continue
                out.append(f"ParticleTypes: {l} {p2} {p3}")
                out.append("threeBodyCorrelationFunctionType: Cambridge")
                out.append("NumberOfParameterTypes: 2")
                out.append(f"NumberOfParametersOfEachType: {tb.nen} {tb.nee}")
                out.append("Parameters:")
                out.append(" ".join(g % v for v in tb.input_parameters()))
                out.append(f"C: {tb.C}")
                out.append(f"Cutoff: {g % tb.cutoff}")
                out.append("")
        out.append("&Jastrow")
        out.append("")
        with open(path, "w") as fh:
            fh.write("\n".join(out))


DEFAULT_FLAGS: Dict[str, object] = {
    "run_type": "variational",
    "dt": 0.09,
    "number_of_walkers": 1,
    "max_time_steps": 10,
    "max_time": -1,
    "one_e_per_iter": 1,
    "warn_verbosity": 0,
    "sampling_method": "no_importance_sampling",
    "QF_modification_type": "none",
    "energy_modification_type": "none",
    "energy_cutoff_type": "none",
    "walker_reweighting_method": "umrigar93_probability_weighted",
    "branching_method": "nonunit_weight_branching",
    "branching_threshold": 2.0,
    "fusion_threshold": 0.45,
    "equilibration_steps": 0,
    "walker_initialization_method": "dans_walker_initialization",
    "replace_electron_nucleus_cusps": 0,
    "use_three_body_jastrow": 0,
    "link_Jastrow_parameters": 1,
    "optimize_Psi": 0,
    "iseed": -1000,
    "walkers_per_pass": 1,
    "output_interval": 100,
    "energy": -1.0,
    "chip_and_mike_are_cool": "Yea_Baby!",
}


# ----------------------------------------------------------------- generator
def _double_factorial(n: int) -> int:
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _overlap_1d(m: int, p: float) -> float:
    # int x^(2m) exp(-p x^2) dx
    return _double_factorial(2 * m - 1) / (2.0 * p) ** m * math.sqrt(math.pi / p)


def _self_overlap(powers, ea: float, eb: float) -> float:
    p = ea + eb
    s = 1.0
    for m in powers:
        s *= _overlap_1d(m, p)
    return s


def _contracted(rng: np.random.Generator, t: str, exps: np.ndarray, raw: np.ndarray) -> BasisFunction:
    """Primitive normalisation folded into the coefficients, then the
    contraction normalised to unit self-overlap."""
    pw = type_to_powers(t)
    c = np.array([raw[i] / math.sqrt(_self_overlap(pw, exps[i], exps[i])) for i in range(len(exps))])
    s = 0.0
    for i in range(len(exps)):
        for j in range(len(exps)):
            s += c[i] * c[j] * _self_overlap(pw, exps[i], exps[j])
    c = c / math.sqrt(s)
    return BasisFunction(t, exps.copy(), c)


def _shell(rng: np.random.Generator, kind: str, nprim: int) -> List[BasisFunction]:
    exps = np.sort(10.0 ** rng.uniform(-1.0, 2.0, nprim))[::-1].copy()
    raw = rng.standard_normal(nprim)
    return [_contracted(rng, t, exps, raw) for t in SHELL_TYPES[kind]]


def _place_nuclei(rng: np.random.Generator, M: int, box: float, min_sep: float) -> np.ndarray:
    pts: List[np.ndarray] = []
    tries = 0
    while len(pts) < M:
        tries += 1
        if tries > 200000:
            raise RuntimeError("cannot place nuclei")
        p = rng.uniform(-box / 2, box / 2, 3)
        if all(np.linalg.norm(p - q) >= min_sep for q in pts):
            pts.append(p)
    return np.asarray(pts)


def _distribute_basis(rng: np.random.Generator, Z: Sequence[int], K: int, nprim: int) -> List[List[BasisFunction]]:
    """Round robin over atoms adding shells until exactly K functions exist.
    Heavy atoms cycle s, p, s, d, p ...; hydrogen cycles s, p, s, s, p."""
    heavy = ["s", "p", "s", "d", "p", "s", "d", "p"]
    light = ["s", "p", "s", "s", "p"]
    size = {"s": 1, "p": 3, "d": 6}
    basis: List[List[BasisFunction]] = [[] for _ in Z]
    idx = [0] * len(Z)
    left = K
    while left > 0:
        for a, z in enumerate(Z):
            if left == 0:
                break
            pat = heavy if z > 2 else light
            kind = pat[idx[a] % len(pat)]
            idx[a] += 1
            if size[kind] > left:
                kind = "s"
            basis[a].extend(_shell(rng, kind, nprim))
            left -= size[kind]
    return basis


def _random_mo(rng: np.random.Generator, K: int, n: int) -> np.ndarray:
    A = rng.normal(0.0, 1.0 / math.sqrt(K), (K, K))
    Q, _ = np.linalg.qr(A)
    return np.ascontiguousarray(Q[:, :n].T)  # orbital rows


def _overlap_1d_table(imax: int, jmax: int, a, b, A, B) -> np.ndarray:
    """Obara-Saika table of 1D overlaps <(x-A)^i e^{-a(x-A)^2} | (x-B)^j e^{-b(x-B)^2}>
    for i <= imax, j <= jmax (Obara & Saika, J. Chem. Phys. 84, 3963 (1986)),
    vectorised over arrays of exponent / centre pairs."""
    p = a + b
    P = (a * A + b * B) / p
    XPA, XPB = P - A, P - B
    S = np.zeros(np.broadcast(a, b, A, B).shape + (imax + 1, jmax + 1))
    S[..., 0, 0] = np.sqrt(np.pi / p) * np.exp(-a * b / p * (A - B) ** 2)
    o = 1.0 / (2.0 * p)
    for i in range(imax + 1):
        for j in range(jmax + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                v = XPA * S[..., i - 1, j]
                if i > 1:
                    v = v + (i - 1) * o * S[..., i - 2, j]
                if j > 0:
                    v = v + j * o * S[..., i - 1, j - 1]
            else:
                v = XPB * S[..., i, j - 1]
                if j > 1:
                    v = v + (j - 1) * o * S[..., i, j - 2]
            S[..., i, j] = v
    return S


def core_hamiltonian_orbitals(s: "MolecularSystem", n: int, block: int = 256) -> np.ndarray:
    """Lowest n orbitals of an approximate core Hamiltonian in the system's
    basis: exact overlap S and kinetic T (Obara-Saika), nuclear attraction in
    the Mulliken approximation V_ab = S_ab (v_a + v_b) / 2 with v_a = -sum_C
    Z_C <1/r_C>_a (own centre: the radial expectation of the contraction;
    other centres: the point value 1/R).  Solves T + V = S C e.
    Returns the orbital rows (n, K)."""
    atom, pw, nprim, off, ex, co = s.flat_basis()
    K = len(atom)
    pf = np.repeat(np.arange(K), nprim)
    Pn = len(ex)
    Ac = s.coords[atom[pf]]
    pa = pw[pf]
    S = np.zeros((K, K))
    T = np.zeros((K, K))
    jj_all = np.arange(Pn)
    for r0 in range(0, Pn, block):
        ii = np.arange(r0, min(Pn, r0 + block))[:, None]
        jj = jj_all[None, :]
        a, b = np.broadcast_arrays(ex[ii], ex[jj])
        Sd, Td = [], []
        for d in range(3):
            tab = _overlap_1d_table(2 if pa[:, d].max() <= 2 else pa[:, d].max(), pa[:, d].max() + 2,
                                    a, b, Ac[ii, d], Ac[jj, d])
            i_ = np.broadcast_to(pa[ii, d], a.shape)
            j_ = np.broadcast_to(pa[jj, d], a.shape)
            row = np.take_along_axis(tab, i_[..., None, None], -2)[..., 0, :]
            s0 = np.take_along_axis(row, j_[..., None], -1)[..., 0]
            sp2 = np.take_along_axis(row, (j_ + 2)[..., None], -1)[..., 0]
            sm2 = np.take_along_axis(row, np.maximum(j_ - 2, 0)[..., None], -1)[..., 0]
            t = -2.0 * b * b * sp2 + b * (2 * j_ + 1) * s0 - 0.5 * j_ * (j_ - 1) * np.where(j_ >= 2, sm2, 0.0)
            Sd.append(s0)
            Td.append(t)
        cc = co[ii] * co[jj]
        sp = cc * Sd[0] * Sd[1] * Sd[2]
        tp = cc * (Td[0] * Sd[1] * Sd[2] + Sd[0] * Td[1] * Sd[2] + Sd[0] * Sd[1] * Td[2])
        fi = np.broadcast_to(pf[ii], a.shape)
        fj = np.broadcast_to(pf[jj], a.shape)
        np.add.at(S, (fi, fj), sp)
        np.add.at(T, (fi, fj), tp)
    v = np.zeros(K)
    for k in range(K):
        L = int(pw[k].sum())
        sl = slice(off[k], off[k] + nprim[k])
        e_, c_ = ex[sl], co[sl]
        pij = e_[:, None] + e_[None, :]
        cij = c_[:, None] * c_[None, :]
        num = np.sum(cij * math.gamma(L + 1) / (2 * pij ** (L + 1)))
        den = np.sum(cij * math.gamma(L + 1.5) / (2 * pij ** (L + 1.5)))
        for C in range(s.n_nuclei):
            if C == atom[k]:
                v[k] -= s.Z[C] * num / den
            else:
                v[k] -= s.Z[C] / np.linalg.norm(s.coords[C] - s.coords[atom[k]])
    H = T + 0.5 * S * (v[:, None] + v[None, :])
    w, U = np.linalg.eigh(S)
    keep = w > 1e-8 * w.max()
    X = U[:, keep] / np.sqrt(w[keep])
    _, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    return np.ascontiguousarray(C[:, :n].T)


def _jastrows(labels: Sequence[str], Z: Sequence[float]):
    ee_anti = Pade.fixed_cusp(0.5, 1.0)
    ee_para = Pade.fixed_cusp(0.25, 1.0)
    en = {l: Pade.fixed_cusp(-float(z), 1.5) for l, z in zip(labels, Z)}
    return ee_anti, ee_para, en


def _assemble(name, Zs, coords, basis, n_alpha, n_beta, rng, jastrow=True, orbitals="random") -> MolecularSystem:
    labels = [ELEMENT[int(z)] for z in Zs]
    K = sum(len(b) for b in basis)
    n_orb = max(n_alpha, n_beta)
    mo = _random_mo(rng, K, n_orb)
    if jastrow:
        ee_anti, ee_para, en = _jastrows(labels, Zs)
    else:
        ee_anti = ee_para = None
        en = {}
    sysm = MolecularSystem(
        labels=labels, Z=np.asarray(Zs, np.float64), coords=np.asarray(coords, np.float64),
        basis=basis, mo=mo, n_alpha=n_alpha, n_beta=n_beta,
        alpha_occ=np.arange(n_alpha), beta_occ=np.arange(n_beta),
        ee_anti=ee_anti, ee_para_up=ee_para, ee_para_dn=ee_para,
        en_up=dict(en), en_dn=dict(en), name=name)
    if orbitals == "core":
        sysm.mo = core_hamiltonian_orbitals(sysm, n_orb)
    sysm.check_exponent_cache()
    return sysm


def with_cambridge2(s: MolecularSystem, seed: int = 1) -> MolecularSystem:
    """The same molecule with Cambridge2 two-body functions of the shape the
    reference's inputs use (QMcBeaver/test/oepi.ckmf &Jastrow): e-e cusp
    constants 1/2 (up-down) and 1/4 (parallel), e-n cusp constant 0,
    C = 3 (C = 2 for the down-down pair), L in [0.13, 0.25] so each
    function reaches 4 to 8 bohr, 8 to 12 alpha coefficients; the last
    nucleus type's down-electron function is inactive (L = 0)."""
    rng = np.random.default_rng(seed)

    def fn(g: float, C: int, n: int, active: bool = True) -> Cambridge2:
        L = float(rng.uniform(0.13, 0.25)) if active else 0.0
        a = rng.normal(0.0, 1.5, n).tolist()
        return Cambridge2.from_parameters([L] + a, [g, C])

    types = list(dict.fromkeys(s.labels))
    en_up = {l: fn(0.0, 3, 8 + (i % 5)) for i, l in enumerate(types)}
    en_dn = {l: fn(0.0, 3, 8, active=(i != len(types) - 1)) for i, l in enumerate(types)}
    return dataclasses.replace(s, ee_anti=fn(0.5, 3, 8), ee_para_up=fn(0.25, 3, 9), ee_para_dn=fn(0.25, 2, 8),
                               en_up=en_up, en_dn=en_dn, name=s.name + " cambridge2")


def with_three_body(s: MolecularSystem, seed: int = 1, nen: int = 4, nee: int = 4, scale: float = 0.5,
                    separate_kinds: bool = True) -> MolecularSystem:
    """The same molecule with Cambridge three-body functions on every nucleus
    type, of the reference inputs' shape (QMcBeaver/test/oepi.ckmf: NeN =
    Nee = 4, C = 3, cutoff L so that each reaches 2.5 to 4 bohr); with
    separate_kinds the up-up and down-down pairs get their own functions."""
    from .threebody import random_three_body
    rng = np.random.default_rng(seed)
    tb = {}
    for l in dict.fromkeys(s.labels):
        ud = random_three_body(rng, nen, nee, 3, float(rng.uniform(0.25, 0.4)), scale)
        if separate_kinds:
            uu = random_three_body(rng, nen, nee, 3, float(rng.uniform(0.25, 0.4)), scale)
            dd = random_three_body(rng, nen, nee, 2, float(rng.uniform(0.25, 0.4)), scale)
            tb[l] = (ud, uu, dd)
        else:
            tb[l] = (ud, ud, ud)
    return dataclasses.replace(s, three_body=tb, name=s.name + " three-body")


def with_determinants(s: MolecularSystem, n_det: int = 9, n_virtual: int = 4, seed: int = 1,
                      ci_scale: float = 0.3) -> MolecularSystem:
    """The same molecule with a CI expansion over the lowest
    max(n_alpha, n_beta) + n_virtual orbitals of the approximate core
    Hamiltonian: the ground determinant, one single excitation of each spin
    into every virtual orbital (so every listed orbital is active in both
    spins), then distinct random doubles (one electron of each spin) up to
    n_det; CI coefficients 1 and N(0, ci_scale).  The shape of the
    reference's multi-determinant inputs (QMcBeaver/examples/BeMCSCF.ckmf)."""
    rng = np.random.default_rng(seed)
    na, nb = s.n_alpha, s.n_beta
    n_orb = max(na, nb) + n_virtual
    mo = core_hamiltonian_orbitals(s, n_orb)
    ground = (tuple(range(na)), tuple(range(nb)))
    dets = [ground]

    def excite(occ, n, v):
        o = list(occ)
        o[int(rng.integers(n))] = v
        return tuple(sorted(o))

    for v in range(max(na, nb), n_orb):
        if na > 0:
            dets.append((excite(ground[0], na, v), ground[1]))
        if nb > 0:
            dets.append((ground[0], excite(ground[1], nb, v)))
    tries = 0
    while len(dets) < n_det and tries < 10000 and na > 0 and nb > 0:
        tries += 1
        key = (excite(ground[0], na, int(rng.integers(na, n_orb))), excite(ground[1], nb, int(rng.integers(nb, n_orb))))
        if key not in dets:
            dets.append(key)
    if len(dets) < n_det:
        raise ValueError("not enough distinct excitations")
    dets = dets[:max(n_det, 1 + (na > 0) * n_virtual + (nb > 0) * n_virtual)]
    nd = len(dets)
    ci = np.concatenate([[1.0], rng.normal(0.0, ci_scale, nd - 1)])
    return dataclasses.replace(
        s, mo=mo, alpha_occ=np.arange(na), beta_occ=np.arange(nb),
        det_alpha=np.array([d[0] for d in dets], np.int64).reshape(nd, na),
        det_beta=np.array([d[1] for d in dets], np.int64).reshape(nd, nb),
        ci_coeffs=ci, name=s.name + f" {nd} determinants")


def make_water_like(seed: int = 1, jastrow: bool = True) -> MolecularSystem:
    """The small VMC system: O at the origin, H at (+-1.43, 1.11, 0) bohr,
    5 up + 5 down electrons, 24 contracted Cartesian Gaussians with 3
    primitives (O: 2 s + 2 p + 1 d shell = 14; each H: 2 s + 1 p = 5)."""
    rng = np.random.default_rng(seed)
    Zs = [8, 1, 1]
    coords = [[0.0, 0.0, 0.0], [1.43, 1.11, 0.0], [-1.43, 1.11, 0.0]]
    basis = []
    for z in Zs:
        fs: List[BasisFunction] = []
        kinds = ["s", "s", "p", "p", "d"] if z == 8 else ["s", "s", "p"]
        for k in kinds:
            fs.extend(_shell(rng, k, 3))
        basis.append(fs)
    return _assemble("water-like C1 (3 nuclei, 10 e, 24 bf)", Zs, coords, basis, 5, 5, rng, jastrow)


def make_random_molecule(n_elec: int, n_nuclei: int, n_basis: int, box: float, z_choices: Sequence[int],
                         seed: int = 1, min_sep: float = 1.8, jastrow: bool = True,
                         name: Optional[str] = None, orbitals: str = "core") -> MolecularSystem:
    """Synthetic molecule: nuclei uniform in a cube (minimum separation),
    Z drawn from z_choices (the draw whose total charge is closest to the
    electron count is kept), n_elec/2 up and n_elec/2 down electrons,
    n_basis contracted Cartesian Gaussians with 3 primitives each.
    orbitals = "core": lowest orbitals of the approximate core Hamiltonian
    (a trial function whose local energy is tame enough for DMC population
    control); "random": QR-orthonormalised Gaussian coefficients."""
    rng = np.random.default_rng(seed)
    best = None
    for _ in range(256):
        Zs = list(rng.choice(z_choices, n_nuclei))
        d = abs(sum(Zs) - n_elec)
        if best is None or d < best[0]:
            best = (d, Zs)
        if d == 0:
            break
    Zs = [int(z) for z in best[1]]
    coords = _place_nuclei(rng, n_nuclei, box, min_sep)
    basis = _distribute_basis(rng, Zs, n_basis, 3)
    na = n_elec - n_elec // 2
    nb = n_elec // 2
    return _assemble(name or f"synthetic ({n_nuclei} nuclei, {n_elec} e, {n_basis} bf)",
                     Zs, coords, basis, na, nb, rng, jastrow, orbitals)


# The benchmark / parity workloads, named by what they are.
WORKLOADS = {
    "vmc_water_10e": dict(kind="water", walkers=100, run="vmc", dt=0.09, importance=False),
    "dmc_6nuc_30e": dict(kind="random", n_elec=30, n_nuclei=6, n_basis=120, box=6.0, z=(1, 6, 7, 8),
                         walkers=16384, run="dmc", dt=0.01, importance=True, refresh=50),
    "mixed_20nuc_100e": dict(kind="random", n_elec=100, n_nuclei=20, n_basis=400, box=12.0, z=(1, 6, 8),
                             walkers=65536, run="dmc", dt=0.01, importance=True, refresh=50),
    # Cambridge2 two-body Jastrow (the form of the reference's own test inputs)
    "vmc_cambridge2_16e": dict(kind="random", n_elec=16, n_nuclei=4, n_basis=64, box=5.0, z=(1, 6, 7, 8),
                               walkers=4096, run="vmc", dt=0.01, importance=True, refresh=50,
                               correlation="cambridge2"),
    # Cambridge2 two-body and Cambridge three-body Jastrow (the reference's test inputs' form)
    "vmc_threebody_16e": dict(kind="random", n_elec=16, n_nuclei=4, n_basis=64, box=5.0, z=(1, 6, 7, 8),
                              walkers=4096, run="vmc", dt=0.01, importance=True, refresh=50,
                              correlation="cambridge2", three_body=True),
    # twelve determinants (singles and doubles into four virtual orbitals)
    "vmc_multidet_12e": dict(kind="random", n_elec=12, n_nuclei=3, n_basis=48, box=4.5, z=(1, 6, 7, 8),
                             walkers=4096, run="vmc", dt=0.01, importance=True, refresh=50,
                             determinants=(12, 4)),
}


def make_system(workload: str, seed: int = 1, jastrow: bool = True) -> MolecularSystem:
    w = WORKLOADS[workload]
    if w["kind"] == "water":
        return make_water_like(seed, jastrow)
    s = make_random_molecule(w["n_elec"], w["n_nuclei"], w["n_basis"], w["box"], w["z"], seed=seed,
                             jastrow=jastrow, name=workload)
    if jastrow and w.get("correlation") == "cambridge2":
        s = with_cambridge2(s, seed=seed + 1)
        s.name = workload
    if jastrow and w.get("three_body"):
        s = with_three_body(s, seed=seed + 3)
        s.name = workload
    if "determinants" in w:
        nd, nv = w["determinants"]
        s = with_determinants(s, nd, nv, seed=seed + 2)
        s.name = workload
    return s


# ------------------------------------------------------------ serialisation
def system_to_arrays(s: MolecularSystem) -> Dict[str, np.ndarray]:
    """Flat arrays (npz friendly) that rebuild the system exactly."""
    types, atom, nprim, ex, co = [], [], [], [], []
    for a, fs in enumerate(s.basis):
        for f in fs:
            types.append(f.type)
            atom.append(a)
            nprim.append(len(f.exponents))
            ex.extend(float(v) for v in f.exponents)
            co.extend(float(v) for v in f.coefficients)

    def pade_arr(p) -> np.ndarray:
        # row 0: [len, numerator...], row 1: [len, denominator...]; a
        # Cambridge2 function is stored as row 0 = [-len, alpha...],
        # row 1 = [fL, C, active, ...]
        out = np.full((2, PADE_MAX + 1), np.nan)
        if isinstance(p, Cambridge2):
            out[0, 0] = -len(p.alpha)
            out[0, 1:1 + len(p.alpha)] = p.alpha
            out[1, 0:3] = (p.fL, p.C, 1.0 if p.active else 0.0)
        elif p is not None:
            out[0, 0] = len(p.num)
            out[0, 1:1 + len(p.num)] = p.num
            out[1, 0] = len(p.den)
            out[1, 1:1 + len(p.den)] = p.den
        return out

    return dict(
        labels=np.array(s.labels), Z=s.Z, coords=s.coords, bf_type=np.array(types), bf_atom=np.array(atom),
        bf_nprim=np.array(nprim), prim_exp=np.array(ex), prim_coef=np.array(co), mo=s.mo,
        n_alpha=np.array(s.n_alpha), n_beta=np.array(s.n_beta), alpha_occ=s.alpha_occ, beta_occ=s.beta_occ,
        ee_anti=pade_arr(s.ee_anti), ee_para_up=pade_arr(s.ee_para_up), ee_para_dn=pade_arr(s.ee_para_dn),
        en_up=np.stack([pade_arr(s.en_up.get(l)) for l in s.labels]),
        en_dn=np.stack([pade_arr(s.en_dn.get(l)) for l in s.labels]),
        name=np.array(s.name), replace_cusps=np.array(1 if s.replace_cusps else 0),
        three_body=_three_body_arr(s),
        **({} if s.det_alpha is None else dict(det_alpha=np.asarray(s.det_alpha), det_beta=np.asarray(s.det_beta),
                                              ci_coeffs=np.asarray(s.ci_coeffs, np.float64))))


TB_MAX = 512  # coefficients per serialised three-body function


def _three_body_arr(s: MolecularSystem) -> np.ndarray:
    """[M][3][4 + TB_MAX]: NeN, Nee, C, cutoff, coefficients (NeN = 0: none)."""
    out = np.zeros((max(s.n_nuclei, 1), 3, 4 + TB_MAX))
    for a, l in enumerate(s.labels):
        for k, f in enumerate(s.three_body.get(l, (None, None, None))):
            if f is not None:
                out[a, k, :4] = (f.nen, f.nee, f.C, f.cutoff)
                out[a, k, 4:4 + len(f.coeffs)] = f.coeffs
    return out


def _three_body_of(arr, labels) -> Dict[str, tuple]:
    from .threebody import ThreeBody
    out: Dict[str, tuple] = {}
    for a, l in enumerate(labels):
        fs = []
        for k in range(3):
            nen, nee, C, cut = arr[a, k, :4]
            if nen == 0:
                fs.append(None)
                continue
            n = int(nen) * int(nen) * int(nee)
            fs.append(ThreeBody(nen=int(nen), nee=int(nee), C=int(C), cutoff=float(cut),
                                coeffs=np.array(arr[a, k, 4:4 + n])))
        if any(f is not None for f in fs):
            out[l] = tuple(fs)
    return out


def system_from_arrays(d) -> MolecularSystem:
    def pade_of(a):
        a = np.asarray(a)
        if np.isnan(a[0, 0]):
            return None
        if a[0, 0] < 0:
            n = int(-a[0, 0])
            return Cambridge2(fL=float(a[1, 0]), C=int(a[1, 1]), alpha=list(a[0, 1:1 + n]), active=bool(a[1, 2]))
        nn, nd = int(a[0, 0]), int(a[1, 0])
        return Pade(num=list(a[0, 1:1 + nn]), den=list(a[1, 1:1 + nd]))

    labels = [str(x) for x in d["labels"]]
    basis: List[List[BasisFunction]] = [[] for _ in labels]
    p = 0
    for t, a, n in zip(d["bf_type"], d["bf_atom"], d["bf_nprim"]):
        basis[int(a)].append(BasisFunction(str(t), np.array(d["prim_exp"][p:p + n]), np.array(d["prim_coef"][p:p + n])))
        p += int(n)
    en_up = {}
    en_dn = {}
    for i, l in enumerate(labels):
        pu, pd = pade_of(d["en_up"][i]), pade_of(d["en_dn"][i])
        if pu is not None:
            en_up[l] = pu
        if pd is not None:
            en_dn[l] = pd
    return MolecularSystem(
        labels=labels, Z=np.array(d["Z"], np.float64), coords=np.array(d["coords"], np.float64), basis=basis,
        mo=np.array(d["mo"], np.float64), n_alpha=int(d["n_alpha"]), n_beta=int(d["n_beta"]),
        alpha_occ=np.array(d["alpha_occ"]), beta_occ=np.array(d["beta_occ"]),
        ee_anti=pade_of(d["ee_anti"]), ee_para_up=pade_of(d["ee_para_up"]), ee_para_dn=pade_of(d["ee_para_dn"]),
        en_up=en_up, en_dn=en_dn, name=str(d["name"]),
        det_alpha=np.array(d["det_alpha"]) if "det_alpha" in d else None,
        det_beta=np.array(d["det_beta"]) if "det_beta" in d else None,
        ci_coeffs=np.array(d["ci_coeffs"], np.float64) if "ci_coeffs" in d else None,
        replace_cusps=bool(int(d["replace_cusps"])) if "replace_cusps" in d else False,
        three_body=_three_body_of(np.asarray(d["three_body"]), labels) if "three_body" in d else {})
