"""Cambridge three-body (electron-electron-nucleus) Jastrow functions.

For a nucleus I and two electrons at distances r1, r2 from it and r12 from
each other, with L the function's inverse cutoff and the scaled distances
x1 = L r1, x2 = L r2, x12 = L r12,

    U = (x1 - 1)^C (x2 - 1)^C  sum_{l,m < NeN, n < Nee} c_lmn x1^l x2^m x12^n

inside x1, x2 < 1 (zero outside); CambridgeThreeBodyCorrelationFunction,
QMcBeaver/src/CambridgeThreeBodyCorrelationFunction.cpp.

The input lists all NeN^2 Nee coefficients in ascending-power order; the
reference multiplies them by a dependency matrix that imposes the l <-> m
symmetry and the electron-electron and electron-nucleus no-cusp conditions
(QMCThreeBodyCorrelationFunctionParameters::read / makeParamDepMatrix /
gaussianParamDepMatrix, QMcBeaver/src/QMCThreeBodyCorrelationFunctionParameters.cpp:
48-277, 833-1425).  This module restates that construction, so the
coefficient tables handed to the library are the ones the reference
evaluates.
"""
from __future__ import annotations

import dataclasses
from typing import List, Sequence, Tuple

import numpy as np


def _map(nen: int, nee: int, l: int, m: int, n: int) -> int:
    return l * nen * nee + m * nee + n


def file_order(nen: int, nee: int) -> List[int]:
    """Coefficient index of every input parameter: ascending maximum power,
    symmetric (l, m) / (m, l) pairs next to each other
    (QMcBeaver/src/QMCThreeBodyCorrelationFunctionParameters.cpp:175-205)."""
    out: List[int] = []
    for p in range(max(nen, nee)):
        for n in range(nee):
            for l in range(nen):
                for m in range(l + 1):
                    if (l == p or m == p or n == p) and (l <= p and m <= p and n <= p):
                        out.append(_map(nen, nee, l, m, n))
                        if l != m:
                            out.append(_map(nen, nee, m, l, n))
    if len(out) != nen * nen * nee:
        raise ValueError("three-body parameter ordering does not cover every term")
    return out


def _manual_dependencies(nen: int, nee: int, C: int, rep_ne: bool, rep_ee: bool):
    """makeParamDepMatrix without the Gaussian elimination path
    (QMcBeaver/src/QMCThreeBodyCorrelationFunctionParameters.cpp:1081-1425)."""
    T = nen * nen * nee
    mp = lambda l, m, n: _map(nen, nee, l, m, n)
    free = np.zeros(T, bool)
    for l in range(nen):
        for m in range(nen):
            for n in range(nee):
                f = True
                if m > l:
                    f = False
                elif l > 0 and m == 0 and n == 0:
                    if not rep_ne:
                        f = False
                elif l == 0 and n > 1:
                    if not rep_ee:
                        f = False
                elif m == 0 and n == 1:
                    f = False
                elif l == nen - 1 and n == 1:
                    f = False
                elif l == 0 and n == 0:
                    f = False
                elif l < nen and m == 1 and n == 0:
                    f = False
                elif l == nen - 2 and m == 1 and n == 2:
                    f = False
                elif l == nen - 1 and m == 1 and n > 1:
                    f = False
                free[mp(l, m, n)] = f
    P = np.eye(T)
    for l in range(nen - 1):
        for m in range(l + 1, nen):
            for n in range(nee):
                P[mp(l, m, n), mp(l, m, n)] = 0.0
    P[1, 1] = 0.0
    P[nen * nee + 1, nen * nee + 1] = 0.0
    for k in range(2, 2 * nen - 1):
        if k < nen:
            li, mi = k, 0
        else:
            li, mi = nen - 1, k - (nen - 1)
        dep = li * nen * nee + mi * nee + 1
        P[dep, dep] = 0.0
        if k % 2 == 0:
            i1 = k * nen * nee // 2 + k * nee // 2 + 1
            if dep != i1:
                P[dep, i1] = -1.0 if li == mi else -0.5
        for l in range(nen):
            for m in range(l):
                if l + m == k:
                    i1 = l * nen * nee + m * nee + 1
                    if dep != i1:
                        P[dep, i1] = -2.0 if li == mi else -1.0
    shift = 1.0
    P[0, 0] = 0.0
    P[0, nen * nee] = shift / C
    P[nen * nee + nee, nen * nee + nee] = 0.0
    P[nen * nee + nee, nen * nee] = C / shift
    for k in range(2, nen + nee - 1):
        if k < nen:
            li, ni = k, 0
        elif k == nen:
            li, ni = k - 2, 2
        else:
            li, ni = nen - 1, k - (nen - 1)
        dep = li * nen * nee + nee + ni
        P[dep, dep] = 0.0
        if k < nee:
            i1, i2 = k, nen * nee + k
            P[dep, i1] = C / shift
            if dep != i2:
                P[dep, i2] = -1.0
        for l in range(1, nen):
            for n in range(nee):
                if l + n == k:
                    i1 = l * nen * nee + n
                    i2 = l * nen * nee + nee + n
                    P[dep, i1] = C / shift
                    if dep != i2:
                        P[dep, i2] = -1.0
    if not rep_ne:
        for l in range(1, nen):
            P[l * nen * nee, l * nen * nee] = 0.0
    if not rep_ee:
        for n in range(2, nee):
            P[n, n] = 0.0
    # substitute until no definition uses a dependent parameter
    for _ in range(101):
        good = True
        for l in range(nen):
            for m in range(l + 1):
                for n in range(nee):
                    i1 = mp(l, m, n)
                    if free[i1]:
                        if abs(P[i1, i1] - 1.0) > 1e-10 or np.any(np.abs(np.delete(P[i1], i1)) > 1e-10):
                            raise ValueError(f"three-body parameter {l}{m}{n} should be free")
                        continue
                    if abs(P[i1, i1]) > 1e-10:
                        raise ValueError(f"three-body parameter {l}{m}{n} should be dependent")
                    for i in range(T):
                        if i != i1 and abs(P[i, i1]) > 1e-10:
                            good = False
                            P[i, :] += P[i, i1] * P[i1, :]
                            P[i, i1] = 0.0
                    for a in range(nen):
                        for b in range(nen):
                            for c in range(nee):
                                i2 = mp(a, b, c)
                                if not free[i2] and abs(P[i1, i2]) > 1e-10:
                                    good = False
                                    P[i1, :] += P[i1, i2] * P[i2, :]
                                    P[i1, i2] = 0.0
        if good:
            break
    else:
        raise ValueError("three-body parameter dependencies are circular")
    for l in range(nen - 1):
        for m in range(l + 1, nen):
            for n in range(nee):
                P[mp(l, m, n), :] = P[mp(m, l, n), :]
    return P, free


def constraint_matrix(nen: int, nee: int, C: int, rep_ne: bool, rep_ee: bool) -> np.ndarray:
    """Rows of the linear constraints on the coefficients (l, m, n order):
    electron-electron no-cusp (equation 24 of Drummond, Towler, Needs, PRB 70,
    235119 (2004)), electron-nucleus no-cusp (equation 27), l <-> m symmetry,
    and without reproduce_*_with_NEE_jastrow the terms the two-body Jastrow
    already carries set to zero (the system gaussianParamDepMatrix builds,
    QMcBeaver/src/QMCThreeBodyCorrelationFunctionParameters.cpp:833-935)."""
    nn, ne = nen - 1, nee - 1
    T = nen * nen * nee
    mp = lambda l, m, n: _map(nen, nee, l, m, n)
    ncon = nee * nen * (nen - 1) // 2 + 2 * nn + 1 + nn + ne + 1
    if not rep_ne:
        ncon += nn
    if not rep_ee:
        ncon += ne
    A = np.zeros((ncon, T))
    num = nen * (nen - 1) // 2
    for l in range(nen):
        for m in range(nen):
            for n in range(nee):
                idx = mp(l, m, n)
                if n == 1:
                    A[l + m, idx] = 1.0                      # electron-electron cusp
                k0 = 2 * nn + 1
                if l == 0:
                    A[m + n + k0, idx] = C                   # electron-nucleus cusp
                if l == 1:
                    A[m + n + k0, idx] = -1.0
                k0 += nn + ne + 1
                if l > m:
                    A[l * (l - 1) // 2 + m + n * num + k0, idx] = -1.0   # l <-> m symmetry
                if l < m:
                    A[m * (m - 1) // 2 + l + n * num + k0, idx] = 1.0
                k0 += nee * num
                if not rep_ee:
                    if l == 0 and m == 0 and n > 0:
                        A[n - 1 + k0, idx] = 1.0
                    k0 += ne
                if not rep_ne:
                    if l > 0 and m == 0 and n == 0:
                        A[l - 1 + k0, idx] = 1.0
                    k0 += nn
    return A


def _gaussian_dependencies(nen: int, nee: int, C: int, rep_ne: bool, rep_ee: bool):
    """gaussianParamDepMatrix (QMcBeaver/src/QMCThreeBodyCorrelationFunctionParameters.cpp:
    833-1079): the symmetry and no-cusp constraints as rows of a linear
    system, solved for a chosen set of dependent coefficients by
    Gauss-Jordan elimination (Array2D::rref(int), QMcBeaver/include/Array2D.h:
    1780-1908).  The reduced system, and so the dependencies, are unique for
    the chosen set."""
    if nen != nee:
        # the reference sizes this system with Nee * NeN * Nee variables
        raise ValueError("reproduce_*_with_NEE_jastrow needs NeN == Nee")
    nn = nen - 1
    T = nen * nen * nee
    mp = lambda l, m, n: _map(nen, nee, l, m, n)
    A = constraint_matrix(nen, nee, C, rep_ne, rep_ee)
    ncon = A.shape[0]
    pivot_row = {}   # dependent column -> its constraint row

    def rref(t: int) -> None:
        if t in pivot_row:
            return
        used = set(pivot_row.values())
        best = None
        for r in range(ncon - 1, -1, -1):
            if abs(A[r, t]) >= 1e-10 and r not in used:
                best = r
                break
        if best is None:
            raise ValueError(f"three-body constraints cannot make coefficient {t} dependent")
        scale = A[best, t]
        if abs(scale - 1.0) > 1e-10:
            A[best, :] /= scale
        A[best, t] = 1.0
        for r in range(ncon):
            sc = A[r, t]
            if r == best or abs(sc) < 1e-10:
                continue
            A[r, :] -= A[best, :] * sc
            A[r, np.abs(A[r]) < 1e-10] = 0.0
            A[r, t] = 0.0
        pivot_row[t] = best

    if not rep_ne:
        for l in range(1, nen):
            rref(mp(l, 0, 0))
    if not rep_ee:
        for n in range(1, nee):
            rref(mp(0, 0, n))
    rref(mp(0, 0, 1))
    rref(mp(1, 0, 1))
    rref(mp(nn, nn, 1))
    rref(mp(nn, nn - 1, 1))
    for n in range(nee):
        for l in range(nen):
            for m in range(nen):
                if l < m:
                    rref(mp(l, m, n))
    if nen == 3 and nee == 3:
        for t in [(1, 0, 0), (2, 0, 0), (2, 0, 2), (2, 0, 1), (1, 1, 0), (1, 0, 2), (0, 1, 2)]:
            rref(mp(*t))
    elif nen == 4 and nee == 4:
        for t in [(1, 1, 0), (1, 0, 0), (0, 1, 0), (2, 0, 0), (3, 0, 0), (1, 1, 0), (3, 0, 1), (2, 0, 1),
                  (3, 0, 2), (3, 0, 3), (2, 0, 2)]:
            rref(mp(*t))
    # (the reference only warns when a constraint is left unused, as for
    # NeN = Nee = 4 where one constraint is implied by the others)
    A[np.abs(A) < 1e-100] = 0.0
    P = np.eye(T)
    free = np.ones(T, bool)
    for j, r in pivot_row.items():
        free[j] = False
        P[j, :] = np.where(np.abs(A[r]) > 1e-50, -A[r], 0.0)
        P[j, j] = 0.0
    return P, free


def dependency_matrix(nen: int, nee: int, C: int, rep_ne: bool, rep_ee: bool):
    """(P, free): coefficients = P @ input coefficients (in (l, m, n) order)."""
    if rep_ne and rep_ee:
        return _gaussian_dependencies(nen, nee, C, rep_ne, rep_ee)
    return _manual_dependencies(nen, nee, C, rep_ne, rep_ee)


@dataclasses.dataclass
class ThreeBody:
    nen: int
    nee: int
    C: int
    cutoff: float           # L: distances are scaled by it; the function lives inside 1 / L
    coeffs: np.ndarray      # [nen * nen * nee], index l * nen * nee + m * nee + n

    @staticmethod
    def from_input(params: Sequence[float], nen: int, nee: int, C: int, cutoff: float, rep_ne: bool = False,
                   rep_ee: bool = False) -> "ThreeBody":
        """The coefficients the reference evaluates for one input block."""
        T = nen * nen * nee
        total = np.zeros(T)
        fp = list(params) + [0.0] * T
        for k, idx in enumerate(file_order(nen, nee)):
            total[idx] = float(fp[k])
        P, _ = dependency_matrix(nen, nee, C, rep_ne, rep_ee)
        c = P @ total
        tb = ThreeBody(nen=nen, nee=nee, C=int(C), cutoff=float(cutoff), coeffs=c)
        tb.check()
        return tb

    def input_parameters(self) -> List[float]:
        """The coefficients in input order (they already satisfy the
        constraints, so reading them back reproduces them)."""
        return [float(self.coeffs[i]) for i in file_order(self.nen, self.nee)]

    def check(self, tol: float = 1e-10) -> None:
        """QMCThreeBodyCorrelationFunctionParameters::checkCuspAndSymmetry
        (QMcBeaver/src/QMCThreeBodyCorrelationFunctionParameters.cpp:692-831)."""
        nen, nee, c = self.nen, self.nee, self.coeffs
        mp = lambda l, m, n: _map(nen, nee, l, m, n)
        for l in range(nen - 1):
            for m in range(l + 1, nen):
                for n in range(nee):
                    d = c[mp(l, m, n)] - c[mp(m, l, n)]
                    if abs(c[mp(l, m, n)]) > tol:
                        d /= c[mp(l, m, n)]
                    if abs(d) > tol:
                        raise ValueError("three-body coefficients are not symmetric")
        # the sums are checked relative to their terms: the elimination's
        # rounding is proportional to them (the reference checks 1e-10
        # absolute, which its own rounding can pass or fail by a hair)
        for k in range(2 * nen - 1):
            t = [c[mp(l, m, 1)] for l in range(nen) for m in range(nen) if l + m == k]
            if abs(sum(t)) > tol * max(1.0, sum(abs(x) for x in t)):
                raise ValueError("three-body electron-electron cusp condition not satisfied")
        for k in range(nen + nee - 1):
            t = [self.C * c[mp(0, m, n)] - c[mp(1, m, n)] for m in range(nen) for n in range(nee) if m + n == k]
            if abs(sum(t)) > tol * max(1.0, sum(abs(x) for x in t)):
                raise ValueError("three-body electron-nucleus cusp condition not satisfied")

    def evaluate(self, r1v: np.ndarray, r2v: np.ndarray):
        """U, grad_1 U, grad_2 U, lap_1 U + lap_2 U for electrons at r1v, r2v
        relative to the nucleus (direct formulas, for tests)."""
        L = self.cutoff
        r1, r2 = np.linalg.norm(r1v), np.linalg.norm(r2v)
        d12 = r1v - r2v
        r12 = np.linalg.norm(d12)
        x1, x2, x12 = r1 * L, r2 * L, r12 * L
        if x1 - 1 > 0 or x2 - 1 > 0:
            return 0.0, np.zeros(3), np.zeros(3), 0.0
        c = self.coeffs.reshape(self.nen, self.nen, self.nee)
        l = np.arange(self.nen)[:, None, None]
        m = np.arange(self.nen)[None, :, None]
        n = np.arange(self.nee)[None, None, :]

        def pw(x, k):
            return np.where(k >= 0, np.power(x, np.maximum(k, 0)), 0.0)

        P = np.sum(c * pw(x1, l) * pw(x2, m) * pw(x12, n))
        Pl = np.sum(c * l * pw(x1, l - 1) * pw(x2, m) * pw(x12, n))
        Pm = np.sum(c * m * pw(x1, l) * pw(x2, m - 1) * pw(x12, n))
        Pn = np.sum(c * n * pw(x1, l) * pw(x2, m) * pw(x12, n - 1))
        Pll = np.sum(c * l * (l - 1) * pw(x1, l - 2) * pw(x2, m) * pw(x12, n))
        Pmm = np.sum(c * m * (m - 1) * pw(x1, l) * pw(x2, m - 2) * pw(x12, n))
        Pnn = np.sum(c * n * (n - 1) * pw(x1, l) * pw(x2, m) * pw(x12, n - 2))
        Pln = np.sum(c * l * n * pw(x1, l - 1) * pw(x2, m) * pw(x12, n - 1))
        Pmn = np.sum(c * m * n * pw(x1, l) * pw(x2, m - 1) * pw(x12, n - 1))
        C = self.C
        f1, f2 = (x1 - 1) ** C, (x2 - 1) ** C
        f1p, f2p = C * (x1 - 1) ** (C - 1), C * (x2 - 1) ** (C - 1)
        f1pp, f2pp = C * (C - 1) * (x1 - 1) ** (C - 2), C * (C - 1) * (x2 - 1) ** (C - 2)
        U = f1 * f2 * P
        U1 = (f1p * P + f1 * Pl) * f2          # dU/dx1
        U2 = (f2p * P + f2 * Pm) * f1
        U12 = f1 * f2 * Pn
        U11 = (f1pp * P + 2 * f1p * Pl + f1 * Pll) * f2
        U22 = (f2pp * P + 2 * f2p * Pm + f2 * Pmm) * f1
        U1212 = f1 * f2 * Pnn
        U1_12 = (f1p * Pn + f1 * Pln) * f2
        U2_12 = (f2p * Pn + f2 * Pmn) * f1
        u1, u2, u12 = r1v / r1, r2v / r2, d12 / r12
        g1 = L * (U1 * u1 + U12 * u12)
        g2 = L * (U2 * u2 - U12 * u12)
        lap = L * L * (U11 + 2 / x1 * U1 + U22 + 2 / x2 * U2 + 2 * (U1212 + 2 / x12 * U12)
                       + 2 * np.dot(u1, u12) * U1_12 - 2 * np.dot(u2, u12) * U2_12)
        return float(U), g1, g2, float(lap)


def random_three_body(rng: np.random.Generator, nen: int = 4, nee: int = 4, C: int = 3, cutoff: float = 0.3,
                      scale: float = 1.0, rep_ne: bool = True, rep_ee: bool = True) -> ThreeBody:
    """Random coefficients satisfying every constraint (the shape of the
    reference's inputs: NeN = Nee = 4, C = 3, cutoff 0.26 to 0.3).  The
    elimination leaves one electron-electron condition to the input for
    NeN = 4 (its inputs satisfy it), so the random draw is projected onto
    the null space of all constraint rows first."""
    T = nen * nen * nee
    x = rng.normal(0.0, scale, T)
    A = constraint_matrix(nen, nee, C, rep_ne, rep_ee)
    x = x - np.linalg.pinv(A) @ (A @ x)
    fo = file_order(nen, nee)
    return ThreeBody.from_input([float(x[i]) for i in fo], nen, nee, C, cutoff, rep_ne, rep_ee)
