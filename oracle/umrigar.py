"""Umrigar93 importance-sampling move (C. J. Umrigar, M. P. Nightingale,
K. J. Runge, J. Chem. Phys. 99, 2865 (1993)) restated on the CPU.

TEST INFRASTRUCTURE ONLY (the oracle): tests use it to check the device
move; nothing in the product imports it.

Follows QMCWalker::moveElectronsUmrigar93ImportanceSampling and
QMCWalker::calculateReverseGreensFunctionUmrigar93ImportanceSampling
(QMcBeaver/src/QMCWalker.cpp:400-586, 783-926).  Per electron, with A the
nearest nucleus, d = |x - A|, z the unit vector from A to x and v the
modified drift:
  v_z = z.v, v_rho = |v - v_z z| along the unit vector rho,
  z' = max(d + v_z tau, 0), rho' = 2 v_rho tau z' / (d + z'),
  zeta = sqrt(Z_A^2 + 1/tau),
  P_s = 0.5 erfc((d + v_z tau) / sqrt(2 tau)) clipped to [0, 1], P_g = 1 - P_s,
  G(y) = P_g (2 pi tau)^-3/2 exp(-|y - A - rho' rho - z' z|^2 / 2 tau)
       + P_s / pi zeta^3 exp(-2 zeta |y - A|).
A single-electron move (one_e_per_iter) multiplies the one-electron G of
every electron: the moved one at its new position, the others at their own.
"""
import math
from typing import Sequence, Tuple

import numpy as np


def frame(coords: np.ndarray, Z: Sequence[float], x: Sequence[float], v: Sequence[float], tau: float):
    """(A, c, zeta, P_g, P_s) of an electron at x with modified drift v
    (QMcBeaver/src/QMCWalker.cpp:421-490).  The nearest nucleus is the first
    of the smallest distance (QMCMolecule::findClosestNucleusIndex)."""
    x = np.asarray(x, float)
    v = np.asarray(v, float)
    d2 = ((coords - x) ** 2).sum(axis=1)
    a = int(np.argmin(d2))
    A = coords[a]
    d = math.sqrt(d2[a])
    zu = (x - A) / d
    zc = float(zu @ v)
    rad = v - zc * zu
    rc = math.sqrt(float(rad @ rad))
    if rc > 1e-15:
        rad = rad / rc
    zC = max(d + zc * tau, 0.0)
    rC = 2.0 * rc * tau * zC / (d + zC)
    zeta = math.sqrt(Z[a] * Z[a] + 1.0 / tau)
    ps = min(max(0.5 * math.erfc((d + zc * tau) / math.sqrt(2.0 * tau)), 0.0), 1.0)
    return A, A + rC * rad + zC * zu, zeta, 1.0 - ps, ps


def log_gf(F, y: Sequence[float], tau: float) -> float:
    """ln of the one-electron transition density of frame F at y
    (QMcBeaver/src/QMCWalker.cpp:540-583)."""
    A, c, zeta, pg, ps = F
    y = np.asarray(y, float)
    d1 = float(((y - c) ** 2).sum())
    d2 = float(((y - A) ** 2).sum())
    lg = math.log(pg) - 1.5 * math.log(2 * math.pi * tau) - d1 / (2 * tau) if pg > 0 else -math.inf
    ls = math.log(ps / math.pi) + 3 * math.log(zeta) - 2 * zeta * math.sqrt(d2) if ps > 0 else -math.inf
    m = max(lg, ls)
    if m == -math.inf:
        return m
    return m + math.log(math.exp(lg - m) + math.exp(ls - m))


def log_forward(coords, Z, R: np.ndarray, mg: np.ndarray, e: int, rn: Sequence[float], tau: float) -> float:
    """ln G(R -> R') of moving electron e of R (modified drift mg) to rn."""
    tot = 0.0
    for i in range(R.shape[0]):
        F = frame(coords, Z, R[i], mg[i], tau)
        tot += log_gf(F, rn if i == e else R[i], tau)
    return tot


def log_reverse(coords, Z, Rn: np.ndarray, mgn: np.ndarray, e: int, ro: Sequence[float], tau: float) -> float:
    """ln G(R' -> R): frames of the new positions Rn with their modified drift
    mgn, density at the old positions (electron e was at ro)
    (QMcBeaver/src/QMCWalker.cpp:783-926)."""
    tot = 0.0
    for i in range(Rn.shape[0]):
        F = frame(coords, Z, Rn[i], mgn[i], tau)
        tot += log_gf(F, ro if i == e else Rn[i], tau)
    return tot


def propose(F, u: Sequence[float], tau: float) -> Tuple[np.ndarray, bool]:
    """A draw from the frame's density from uniforms u[0..5] in (0, 1]:
    u[0] < P_g picks the Gaussian (Box-Muller on u[1..4]); otherwise the
    radius is a Gamma(3) variate over 2 zeta, -ln(u1 u2 u3) / (2 zeta) (the
    law Random::randomDistribution1 samples by rejection), and the direction
    is uniform on the sphere (phi = 2 pi u4, cos theta = 1 - 2 u5).
    Returns (position, gaussian?)."""
    A, c, zeta, pg, ps = F
    if u[0] < pg:
        r1 = math.sqrt(-2.0 * math.log(u[1]))
        r2 = math.sqrt(-2.0 * math.log(u[3]))
        g = np.array([r1 * math.cos(2 * math.pi * u[2]), r1 * math.sin(2 * math.pi * u[2]),
                      r2 * math.cos(2 * math.pi * u[4])])
        return c + math.sqrt(tau) * g, True
    r = -math.log(u[1] * u[2] * u[3]) / (2.0 * zeta)
    phi, theta = 2 * math.pi * u[4], math.acos(1.0 - 2.0 * u[5])
    return A + r * np.array([math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta)]), False
