"""First-order (linear) optics of the supported element subset, used only to
match generated beams to a ring: the one-turn matrix gives the periodic Twiss
parameters and dispersion at the start of the line (the role of elegant's
``matched_to_cell`` in bunched_beam, bunched_beam.c:427).  Particle tracking
never uses these matrices.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .lattice import Lattice


def element_matrix(e) -> np.ndarray:
    """6x6 first-order transfer matrix in (x, xp, y, yp, s, delta)."""
    m = np.eye(6)
    L = e.length
    t = e.type
    if t in ("DRIF", "EDRIFT", "KSEXT", "CSRDRIFT", "RFCA"):
        m[0, 1] = m[2, 3] = L
        return m
    if t == "KQUAD":
        k = e.get("K1") * (1 + e.get("FSE"))
        for plane, kk in ((0, k), (2, -k)):
            if kk > 0:
                r = math.sqrt(kk)
                c, s = math.cos(r * L), math.sin(r * L)
                m[plane:plane + 2, plane:plane + 2] = [[c, s / r], [-r * s, c]]
            elif kk < 0:
                r = math.sqrt(-kk)
                c, s = math.cosh(r * L), math.sinh(r * L)
                m[plane:plane + 2, plane:plane + 2] = [[c, s / r], [r * s, c]]
            else:
                m[plane, plane + 1] = L
        return m
    if t in ("CSBEND", "CSRCSBEND"):
        ang = e.get("ANGLE")
        if ang == 0:
            m[0, 1] = m[2, 3] = L
            return m
        rho = L / ang
        c, s = math.cos(ang), math.sin(ang)
        m[0:2, 0:2] = [[c, rho * s], [-s / rho, c]]
        m[0, 5] = rho * (1 - c)
        m[1, 5] = s
        m[4, 0] = s
        m[4, 1] = rho * (1 - c)
        m[4, 5] = rho * (ang - s)
        m[2, 3] = L
        return m
    return m


def line_matrix(lattice: Lattice) -> np.ndarray:
    m = np.eye(6)
    for e in lattice.elements:
        m = element_matrix(e) @ m
    return m


@dataclass
class Twiss:
    beta_x: float
    alpha_x: float
    beta_y: float
    alpha_y: float
    eta_x: float = 0.0
    etap_x: float = 0.0
    tune_x: float = 0.0
    tune_y: float = 0.0


def periodic_twiss(lattice: Lattice) -> Twiss:
    """Periodic solution of the one-turn matrix (raises if unstable)."""
    m = line_matrix(lattice)
    out = []
    for p in (0, 2):
        a = m[p:p + 2, p:p + 2]
        cmu = 0.5 * (a[0, 0] + a[1, 1])
        if abs(cmu) >= 1:
            raise ValueError(f"linear motion in plane {p // 2} is unstable (cos mu = {cmu})")
        smu = math.copysign(math.sqrt(1 - cmu * cmu), a[0, 1])
        beta = a[0, 1] / smu
        alpha = (a[0, 0] - a[1, 1]) / (2 * smu)
        tune = math.acos(cmu) / (2 * math.pi)
        out.append((beta, alpha, tune))
    d = np.linalg.solve(np.eye(2) - m[0:2, 0:2], m[0:2, 5])
    return Twiss(out[0][0], out[0][1], out[1][0], out[1][1], float(d[0]), float(d[1]), out[0][2], out[1][2])
