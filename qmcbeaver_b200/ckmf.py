"""Reader for QMcBeaver's ``.ckmf`` input files (the parts the walker path
needs) and the mapping of their flags onto the library's run parameters.

The file is a whitespace-token stream, read section by section exactly as
QMCInput::read does (QMcBeaver/src/QMCInput.cpp:26-52):

* ``&flags``: key / value token pairs up to ``&``; a key token starting with
  ``#`` comments out the rest of its line (QMCFlags::read_flags,
  QMcBeaver/src/QMCFlags.cpp:190-885).
* ``&geometry``: ``atoms`` records ``label Z x y z``, labels First-upper
  (QMcBeaver/src/QMCMolecule.cpp:83-113).
* ``&basis``: per atom ``label nfunc maxgauss`` then per function
  ``ngauss type`` and ``ngauss`` (exponent, coefficient) pairs
  (QMcBeaver/src/QMCBasisFunctionCoefficients.cpp:84-127).
* ``&wavefunction``: ``norbitals`` x ``nbasisfunc`` coefficients (twice,
  each after a three-word title, for ``unrestricted``), the alpha and beta
  occupations of every determinant and the CI coefficients, optionally
  constrained (``c <index> <factor>``), closed by ``&``
  (QMcBeaver/src/QMCWavefunction.cpp:311-472).
* ``&Jastrow``: two-body blocks (``ParticleTypes:`` ... ``Constants:``) up
  to the first block that is not two-body (QMcBeaver/src/
  QMCCorrelationFunctionParameters.cpp:59-279), linked up/down parameters
  (QMcBeaver/src/QMCJastrowParameters.cpp:708-900); three-body blocks are
  detected and reported, not evaluated.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import desc as D
from .system import BasisFunction, Cambridge2, MolecularSystem, Pade
from .threebody import ThreeBody


class CkmfError(ValueError):
    pass


class _Tokens:
    """Whitespace tokens with their line numbers."""

    def __init__(self, text: str):
        self.tok: List[Tuple[str, int]] = []
        for ln, line in enumerate(text.splitlines()):
            for t in line.split():
                self.tok.append((t, ln))
        self.i = 0

    def eof(self) -> bool:
        return self.i >= len(self.tok)

    def peek(self) -> str:
        return self.tok[self.i][0] if self.i < len(self.tok) else ""

    def next(self) -> str:
        if self.i >= len(self.tok):
            raise CkmfError("unexpected end of input")
        t = self.tok[self.i][0]
        self.i += 1
        return t

    def skip_line(self) -> None:
        ln = self.tok[self.i - 1][1]
        while self.i < len(self.tok) and self.tok[self.i][1] == ln:
            self.i += 1

    def seek(self, marker: str, start: int = 0) -> bool:
        for j in range(start, len(self.tok)):
            if self.tok[j][0] == marker:
                self.i = j + 1
                return True
        return False

    def numbers(self) -> List[float]:
        """Numeric tokens up to the first token that does not start like a
        number (Array1D::read, QMcBeaver/include/Array1D.h:664-689)."""
        out = []
        while not self.eof() and (self.peek()[0].isdigit() or self.peek()[0] in "+-."):
            out.append(float(self.next()))
        return out


def first_upper(s: str) -> str:
    """StringManipulation::toFirstUpperRestLower."""
    return s[:1].upper() + s[1:].lower()


@dataclasses.dataclass
class CorrelationBlock:
    p1: str
    p2: str
    kind: str
    n_params: List[int]
    params: List[float]
    n_consts: List[int]
    consts: List[float]

    def function(self, a_diag: float = -1e-5):
        """The correlation function object of this block, or None for type
        None (QMCCorrelationFunctionFactory, QMcBeaver/src/
        QMCCorrelationFunctionFactory.cpp:21-60)."""
        if self.kind == "None":
            return None
        bp = np.cumsum([0] + self.n_params[:-1]).tolist()
        bc = np.cumsum([0] + self.n_consts[:-1]).tolist()
        if self.kind == "FixedCuspPade":
            # numerator [0, constants of type 0, parameters of type 0],
            # denominator [1, constants of type 1, parameters of type 1]
            # (FixedCuspPadeCorrelationFunction::initializeParameters,
            # QMcBeaver/src/FixedCuspPadeCorrelationFunction.cpp:15-69)
            if len(self.n_params) > 2 or len(self.n_consts) > 2:
                raise CkmfError("FixedCuspPade takes at most two parameter and constant types")
            nnc = len(self.consts) if len(bc) <= 1 else bc[1]
            nnp = len(self.params) if len(bp) <= 1 else bp[1]
            num = [0.0] + list(self.consts[:nnc]) + list(self.params[:nnp])
            den = [1.0] + list(self.consts[nnc:]) + list(self.params[nnp:])
            return Pade(num=num, den=den)
        if self.kind == "Pade":
            # numerator [0, parameters of type 0], denominator [1, the rest]
            # (PadeCorrelationFunction::initializeParameters,
            # QMcBeaver/src/PadeCorrelationFunction.cpp:15-52)
            if len(self.n_params) != 2:
                raise CkmfError("Pade takes two parameter types")
            b1 = bp[1]
            return Pade(num=[0.0] + list(self.params[:b1]), den=[1.0] + list(self.params[b1:]))
        if self.kind == "Cambridge2":
            if len(self.consts) < 2:
                raise CkmfError("Cambridge2 needs the constants gamma and C")
            if len(self.n_params) != 2 or len(self.params) < 2:
                raise CkmfError("Cambridge2 needs two parameter types, L and alpha")
            return Cambridge2.from_parameters(self.params, self.consts, a_diag)
        raise CkmfError(f"correlation function type {self.kind!r} is not supported")


@dataclasses.dataclass
class ThreeBodyBlock:
    """One three-body block (QMCThreeBodyCorrelationFunctionParameters::read,
    QMcBeaver/src/QMCThreeBodyCorrelationFunctionParameters.cpp:48-277)."""
    nucleus: str
    p2: str
    p3: str
    kind: str
    nen: int
    nee: int
    params: List[float]
    C: int
    cutoff: float

    def function(self, rep_ne: bool, rep_ee: bool) -> Optional[ThreeBody]:
        if self.kind == "None":
            return None
        if self.kind != "Cambridge":
            raise CkmfError(f"three-body function type {self.kind!r} is not supported")
        if self.nen < 3 or self.nee < 3:
            raise CkmfError("three-body functions need NeN, Nee >= 3")
        return ThreeBody.from_input(self.params, self.nen, self.nee, self.C, self.cutoff, rep_ne, rep_ee)


@dataclasses.dataclass
class CkmfInput:
    flags: Dict[str, str]
    labels: List[str]
    Z: np.ndarray
    coords: np.ndarray
    basis: List[List[BasisFunction]]
    orbitals: np.ndarray                # (norbitals [x2 unrestricted], nbasis)
    alpha_occupation: np.ndarray        # (ndet, norbitals)
    beta_occupation: np.ndarray
    ci_coeffs: np.ndarray
    jastrow: List[CorrelationBlock]
    three_body: List[ThreeBodyBlock]
    path: str = ""

    @property
    def three_body_blocks(self) -> int:
        """Three-body blocks in use (type other than None)."""
        return sum(1 for b in self.three_body if b.kind != "None")

    # ------------------------------------------------------------- flags
    def flag(self, key: str, default=None, kind=str):
        v = self.flags.get(key)
        if v is None:
            return default
        return kind(v)

    @property
    def n_determinants(self) -> int:
        return self.alpha_occupation.shape[0]

    @property
    def n_alpha(self) -> int:
        return int(self.alpha_occupation[0].sum())

    @property
    def n_beta(self) -> int:
        return int(self.beta_occupation[0].sum())

    # ------------------------------------------------------------ system
    def to_system(self, replace_cusps: Optional[bool] = None, three_body: Optional[bool] = None,
                  name: Optional[str] = None) -> MolecularSystem:
        """The Slater-Jastrow system of this input (one or several determinants).

        replace_cusps: None follows ``replace_electron_nucleus_cusps`` (on by
        default in the reference); True / False overrides it.  three_body:
        None / True evaluates the input's three-body blocks (the reference
        evaluates every block present, whatever use_three_body_jastrow says),
        False leaves them out."""
        if self.flag("trial_function_type", "restricted") not in ("restricted", "unrestricted"):
            raise CkmfError("only restricted / unrestricted trial functions are read")
        if replace_cusps is None:
            replace_cusps = self.flag("replace_electron_nucleus_cusps", 1, int) == 1
        na, nb = self.n_alpha, self.n_beta
        if nb > na:
            raise CkmfError("more beta than alpha electrons")
        a_occ = np.nonzero(self.alpha_occupation[0])[0]
        b_occ = np.nonzero(self.beta_occupation[0])[0]
        det_a = det_b = ci = None
        if self.n_determinants > 1:
            det_a = np.array([np.nonzero(r)[0] for r in self.alpha_occupation])
            det_b = np.array([np.nonzero(r)[0] for r in self.beta_occupation]).reshape(self.n_determinants, nb)
            if det_a.ndim != 2 or det_a.shape[1] != na:
                raise CkmfError("every determinant must occupy the same number of orbitals per spin")
            ci = np.asarray(self.ci_coeffs, np.float64)
        a_diag = self.flag("a_diag", -1e-5, float)
        link = self.flag("link_Jastrow_parameters", 1, int) == 1
        ee_anti = ee_up = ee_dn = None
        en_up: Dict[str, object] = {}
        en_dn: Dict[str, object] = {}
        types = list(dict.fromkeys(self.labels))
        for b in self.jastrow:
            f = b.function(a_diag)
            if b.p1 == "Electron_up":
                if b.p2 == "Electron_up":
                    if na < 2:
                        raise CkmfError("Electron_up-Electron_up block with fewer than two up electrons")
                    ee_up = f
                elif b.p2 == "Electron_down":
                    if na < 1 or nb < 1:
                        raise CkmfError("Electron_up-Electron_down block without both spins")
                    ee_anti = f
                elif b.p2 in types:
                    en_up[b.p2] = f
            else:
                if b.p2 == "Electron_down":
                    if nb < 2:
                        raise CkmfError("Electron_down-Electron_down block with fewer than two down electrons")
                    ee_dn = f
                elif b.p2 in types:
                    if nb < 1:
                        raise CkmfError("Electron_down-nucleus block without down electrons")
                    en_dn[b.p2] = f
        if link:
            if na > 1 and nb > 1:
                ee_dn = ee_up
            if nb > 0:
                en_dn = dict(en_up)
        en_up = {k: v for k, v in en_up.items() if v is not None}
        en_dn = {k: v for k, v in en_dn.items() if v is not None}
        tb = self._three_body(types, na, nb) if three_body is not False else {}
        return MolecularSystem(
            labels=list(self.labels), Z=np.asarray(self.Z, float), coords=np.asarray(self.coords, float),
            basis=self.basis, mo=np.asarray(self.orbitals, float), n_alpha=na, n_beta=nb,
            alpha_occ=a_occ, beta_occ=b_occ, ee_anti=ee_anti, ee_para_up=ee_up, ee_para_dn=ee_dn,
            en_up=en_up, en_dn=en_dn, name=name or self.path, det_alpha=det_a, det_beta=det_b, ci_coeffs=ci,
            replace_cusps=bool(replace_cusps), three_body=tb)

    def _three_body(self, types: List[str], na: int, nb: int) -> Dict[str, tuple]:
        """Per nucleus type (up-down, up-up, down-down) three-body functions,
        linked as link_NEE_Jastrows says (default 2: every pair kind takes the
        up-down function) (QMcBeaver/src/QMCJastrowParameters.cpp:911-1066)."""
        rep_ne = self.flag("reproduce_NE_with_NEE_jastrow", 0, int) == 1
        rep_ee = self.flag("reproduce_EE_with_NEE_jastrow", 0, int) == 1
        link = self.flag("link_NEE_Jastrows", 2, int)
        tb = {l: [None, None, None] for l in types}
        for b in self.three_body:
            if b.nucleus not in tb:
                continue
            f = b.function(rep_ne, rep_ee)
            if b.p2 == "Electron_up" and b.p3 == "Electron_down":
                tb[b.nucleus][0] = f
            elif b.p2 == "Electron_up" and b.p3 == "Electron_up":
                if na < 2:
                    raise CkmfError("Electron_up-Electron_up three-body block with fewer than two up electrons")
                tb[b.nucleus][1] = f
            elif b.p2 == "Electron_down" and b.p3 == "Electron_down":
                if nb < 2:
                    raise CkmfError("Electron_down-Electron_down three-body block with fewer than two down electrons")
                tb[b.nucleus][2] = f
        if na > 1 and nb > 1:
            for l in types:
                if link == 1:
                    tb[l][2] = tb[l][1]
                elif link == 2:
                    tb[l][1] = tb[l][0]
                    tb[l][2] = tb[l][0]
        return {l: tuple(v) for l, v in tb.items() if any(x is not None for x in v)}

    def run_params(self, **overrides) -> D.RunParams:
        """The library's run parameters for this input's flags
        (QMCFlags defaults, QMcBeaver/src/QMCFlags.cpp:24-185)."""
        f = self.flag
        run_type = {"variational": D.QMCB_VMC, "diffusion": D.QMCB_DMC}
        sampling = {"no_importance_sampling": D.QMCB_NO_IMPORTANCE_SAMPLING,
                    "importance_sampling": D.QMCB_IMPORTANCE_SAMPLING,
                    "umrigar93_importance_sampling": D.QMCB_UMRIGAR93_IMPORTANCE_SAMPLING}
        qf = {"none": D.QMCB_QF_NONE, "umrigar93_equalelectrons": D.QMCB_QF_UMRIGAR93_EQUAL,
              "umrigar93_unequalelectrons": D.QMCB_QF_UMRIGAR93_UNEQUAL}
        emod = {"none": D.QMCB_EMOD_NONE, "umrigar93": D.QMCB_EMOD_UMRIGAR93,
                "modified_umrigar93": D.QMCB_EMOD_MODIFIED_UMRIGAR93}
        rw = {"simple_symmetric": D.QMCB_RW_SIMPLE_SYMMETRIC, "simple_asymmetric": D.QMCB_RW_SIMPLE_ASYMMETRIC,
              "umrigar93_probability_weighted": D.QMCB_RW_UMRIGAR93_PROBABILITY_WEIGHTED}
        ecut = {"none": D.QMCB_ECUT_NONE, "umrigar93": D.QMCB_ECUT_UMRIGAR93,
                "bdjm-push88": D.QMCB_ECUT_BDJM_PUSH88}

        def pick(name, table, key, default):
            if name in overrides:
                return overrides[name]
            v = f(key, default)
            if v not in table:
                raise CkmfError(f"{key} {v!r} is not supported by the walker path")
            return table[v]

        ecut_input = pick("energy_cutoff", ecut, "energy_cutoff_type", "umrigar93")
        ecut_run = ecut_input if "energy_cutoff" in overrides else D.QMCB_ECUT_NONE
        kw = dict(
            run_type=pick("run_type", run_type, "run_type", "variational"),
            sampling=pick("sampling", sampling, "sampling_method", "umrigar93_importance_sampling"),
            qf_modification=pick("qf_modification", qf, "QF_modification_type", "umrigar93_unequalelectrons"),
            energy_modification=pick("energy_modification", emod, "energy_modification_type", "umrigar93"),
            reweighting=pick("reweighting", rw, "walker_reweighting_method", "umrigar93_probability_weighted"),
            # the reference reads energy_cutoff_type but never applies it
            # (QMCWalkerData::getModifiedLocalEnergy has no caller): an
            # input's value is checked, and the run has no cutoff
            energy_cutoff=ecut_run,
            dynamic_time_step=1,  # the reference updates dt_effective as it runs
            dt=f("dt", 0.01, float),
            energy_trial=f("energy", 0.0, float),
            energy_estimated=f("energy", 0.0, float),
            energy_original=f("energy", 0.0, float),
            branching_threshold=f("branching_threshold", 2.0, float),
            fusion_threshold=f("fusion_threshold", 0.45, float),
            old_walker_acceptance=f("old_walker_acceptance_parameter", 50, int),
            population_control=f("population_control_parameter", 1.0, float),
            rel_cutoff=f("rel_cutoff", 100.0, float),
            limit_branching=f("limit_branching", 1, int),
            target_walkers=f("number_of_walkers", 100, int),
            # QMCWalker::reweight_walker deletes walkers by fixed rules after
            # every reweight; iteration 0 follows the equilibration steps
            walker_deletion=1,
            equilibration_steps=f("equilibration_steps", 2000, int),
        )
        kw.update(overrides)
        return D.run_params(**kw)


def _read_flags(t: _Tokens) -> Dict[str, str]:
    flags: Dict[str, str] = {}
    if not t.seek("&flags"):
        raise CkmfError("no &flags section")
    while not t.eof():
        k = t.next()
        if k == "&":
            break
        if k.startswith("#"):
            t.skip_line()
            continue
        flags[k] = t.next()
    return flags


def _read_geometry(t: _Tokens, natoms: int):
    if not t.seek("&geometry"):
        raise CkmfError("no &geometry section")
    labels, Z, xyz = [], [], []
    for i in range(natoms):
        l = first_upper(t.next())
        if l == "&":
            raise CkmfError(f"&geometry ended after {i} of {natoms} atoms")
        labels.append(l)
        Z.append(float(t.next()))
        xyz.append([float(t.next()) for _ in range(3)])
    return labels, np.asarray(Z), np.asarray(xyz, float).reshape(-1, 3)


def _read_basis(t: _Tokens, natoms: int):
    if not t.seek("&basis"):
        raise CkmfError("no &basis section")
    basis = []
    for _ in range(natoms):
        label = first_upper(t.next())
        if not ("A" <= label[:1] <= "Z"):
            raise CkmfError(f"&basis: invalid atom label {label!r}")
        nf, _maxg = int(t.next()), int(t.next())
        if nf <= 0:
            raise CkmfError(f"&basis: atom {label} with {nf} functions")
        fs = []
        for _ in range(nf):
            ng = int(t.next())
            typ = t.next().lower()
            ex, co = [], []
            for _ in range(ng):
                ex.append(float(t.next()))
                co.append(float(t.next()))
            fs.append(BasisFunction(type=typ, exponents=np.asarray(ex), coefficients=np.asarray(co)))
            fs[-1].powers  # validates the type string
        basis.append(fs)
    return basis


def _read_wavefunction(t: _Tokens, norb: int, nbasis: int, ndet: int, kind: str):
    if not t.seek("&wavefunction"):
        raise CkmfError("no &wavefunction section")
    if kind not in ("restricted", "unrestricted"):
        raise CkmfError(f"trial_function_type {kind!r} is not supported")
    blocks = 1 if kind == "restricted" else 2
    rows = []
    for b in range(blocks):
        if blocks == 2:
            for _ in range(3):
                t.next()   # "Alpha/Beta Molecular Orbitals"
        for _ in range(norb):
            rows.append([float(t.next()) for _ in range(nbasis)])
    final = norb * blocks
    aocc = np.zeros((ndet, final), np.int64)
    bocc = np.zeros((ndet, final), np.int64)
    t.next(); t.next()   # "Alpha Occupation"
    for i in range(ndet):
        for j in range(norb):
            aocc[i, j] = int(t.next())
    t.next(); t.next()   # "Beta Occupation"
    for i in range(ndet):
        for j in range(final - norb, final):
            bocc[i, j] = int(t.next())
    t.next(); t.next()   # "CI Coeffs"
    ci = np.zeros(ndet)
    constraint = [-1] * ndet
    factor = [1.0] * ndet
    for i in range(ndet):
        tok = t.next()
        if "c" in tok:
            c = int(t.next())
            factor[i] = float(t.next())
            constraint[i] = c if constraint[c] == -1 else constraint[c]
        else:
            ci[i] = float(tok)
    for i in range(ndet):
        if constraint[i] != -1:
            ci[i] = factor[i] * ci[constraint[i]]
    if t.next() != "&":
        raise CkmfError("&wavefunction section not closed by '&'")
    ne = int(aocc[0].sum() + bocc[0].sum())
    for i in range(1, ndet):
        if int(aocc[i].sum() + bocc[i].sum()) != ne:
            raise CkmfError(f"determinant {i + 1} has a different electron count")
    return np.asarray(rows, float), aocc, bocc, ci


def _read_jastrow(t: _Tokens):
    blocks: List[CorrelationBlock] = []
    if not t.seek("&Jastrow"):
        raise CkmfError("no &Jastrow section")
    while t.peek() == "ParticleTypes:":
        start = t.i
        t.next()
        p1, p2 = first_upper(t.next()), first_upper(t.next())
        if t.peek() != "CorrelationFunctionType:":
            # a three-body block (``threeBodyCorrelationFunctionType:``)
            # ends the two-body list
            t.i = start
            break
        t.next()
        kind = t.next()
        t.next()
        npt = int(t.next())
        t.next()
        nparams = [int(t.next()) for _ in range(npt)]
        t.next()
        params = t.numbers()
        total = sum(nparams)
        params = (params + [0.0] * total)[:total]
        t.next()
        nct = int(t.next())
        t.next()
        nconsts = [int(t.next()) for _ in range(nct)]
        t.next()
        consts = t.numbers()
        if len(consts) != sum(nconsts):
            raise CkmfError(f"({p1},{p2}): {len(consts)} constants, {sum(nconsts)} expected")
        if p1 == "Electron_up" or (p2 != "Electron_up" and p1 == "Electron_down"):
            a, b = p1, p2
        elif p2 in ("Electron_up", "Electron_down"):
            a, b = p2, p1
        else:
            raise CkmfError(f"two non-electron particles ({p1}, {p2}) in one correlation function")
        blocks.append(CorrelationBlock(a, b, kind, nparams, params, nconsts, consts))
    three: List[ThreeBodyBlock] = []
    while t.peek() == "ParticleTypes:":
        t.next()
        p1, p2, p3 = first_upper(t.next()), first_upper(t.next()), first_upper(t.next())
        if t.next() != "threeBodyCorrelationFunctionType:":
            raise CkmfError(f"({p1},{p2},{p3}): expected a three-body block")
        kind = t.next()
        t.next()
        npt = int(t.next())
        if npt != 2:
            raise CkmfError("three-body blocks have two parameter types (NeN, Nee)")
        t.next()
        nen, nee = int(t.next()), int(t.next())
        t.next()
        params = t.numbers()
        t.next()
        C = int(float(t.next()))
        t.next()
        cutoff = float(t.next())
        three.append(ThreeBodyBlock(p1, p2, p3, kind, nen, nee, params, C, cutoff))
    return blocks, three


def read_ckmf(path: str, text: Optional[str] = None) -> CkmfInput:
    """Parses a QMcBeaver input file (or its text)."""
    if text is None:
        with open(path) as fh:
            text = fh.read()
    t = _Tokens(text)
    flags = _read_flags(t)
    natoms = int(flags.get("atoms", "0"))
    labels, Z, xyz = _read_geometry(_Tokens(text), natoms)
    if "&pseudopotential" in text.split():
        raise CkmfError("pseudopotentials are not evaluated by the walker path")
    basis = _read_basis(_Tokens(text), natoms)
    nbasis = sum(len(fs) for fs in basis)
    if int(flags.get("nbasisfunc", nbasis)) != nbasis:
        raise CkmfError("nbasisfunc does not match the &basis section")
    orb, aocc, bocc, ci = _read_wavefunction(_Tokens(text), int(flags["norbitals"]), nbasis,
                                             int(flags.get("ndeterminants", "1")),
                                             flags.get("trial_function_type", "restricted"))
    charge = int(flags.get("charge", "0"))
    ne = int(aocc[0].sum() + bocc[0].sum())
    if abs(Z.sum() - (ne + charge)) > 1e-9:
        raise CkmfError(f"nuclear charge {Z.sum()} != electrons {ne} + charge {charge}")
    jas, three = _read_jastrow(_Tokens(text))
    return CkmfInput(flags=flags, labels=labels, Z=Z, coords=xyz, basis=basis, orbitals=orb,
                     alpha_occupation=aocc, beta_occupation=bocc, ci_coeffs=ci, jastrow=jas,
                     three_body=three, path=path)


def patch_flags(text: str, updates: Dict[str, object]) -> str:
    """The input text with the value of each flag in `updates` replaced (or
    the flag added at the end of ``&flags``); every other line is kept."""
    lines = text.splitlines()
    try:
        start = next(i for i, l in enumerate(lines) if l.split()[:1] == ["&flags"])
    except StopIteration:
        raise CkmfError("no &flags section")
    todo = dict(updates)
    i = start + 1
    end = None
    while i < len(lines):
        toks = lines[i].split()
        if not toks:
            i += 1
            continue
        if toks[0] == "&":
            end = i
            break
        if toks[0].startswith("#"):
            i += 1
            continue
        key = toks[0]
        # the value is the next token: on this line or the next non-empty one
        if len(toks) > 1:
            if key in todo:
                lines[i] = f"{key} {todo.pop(key)}"
            i += 1
            continue
        j = i + 1
        while j < len(lines) and not lines[j].split():
            j += 1
        if key in todo:
            lines[j] = f" {todo.pop(key)}"
        i = j + 1
    if end is None:
        raise CkmfError("&flags section not closed")
    add = []
    for k, v in todo.items():
        add += [k, f" {v}"]
    lines[end:end] = add
    return "\n".join(lines) + "\n"


def strip_three_body(text: str) -> str:
    """The input text without its three-body Jastrow blocks.  The reference
    reads every such block after the two-body ones and switches the
    three-body Jastrow on whenever one is used, whatever
    ``use_three_body_jastrow`` says (QMcBeaver/src/QMCJastrowParameters.cpp:
    911-1066), so leaving it out of an evaluation means leaving the blocks
    out of the text."""
    lines = text.splitlines()
    out: List[str] = []
    in_jastrow = False
    skipping = False
    for l in lines:
        toks = l.split()
        if toks[:1] == ["&Jastrow"]:
            in_jastrow = not in_jastrow
            skipping = False
        elif in_jastrow and toks[:1] == ["ParticleTypes:"]:
            skipping = len(toks) >= 4
        if not skipping:
            out.append(l)
    return "\n".join(out) + "\n"
