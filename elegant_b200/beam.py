"""Seeded synthetic bunches (the role of elegant's &bunched_beam,
bunched_beam.c:427 and generate_bunch.c:557).

elegant draws its Gaussians from the toolkit's RNG streams, which are not in
the reference tree, so beams here come from numpy's PCG64 with an explicit
seed; every consumer (the CUDA engine, the CPU oracles) is handed the same
coordinates, so parity never depends on the generator.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

ME_MEV = 0.51099895000  # electron rest energy, MeV (CODATA 2018)


def p_central_from_momentum_mev(p_mev: float) -> float:
    """beta*gamma for an electron of momentum p (MeV/c), as run_setup's p_central_mev."""
    return p_mev / ME_MEV


@dataclass
class Beam:
    """Particles as an (n, 6) FP64 array in elegant's order (x, xp, y, yp, s, delta) plus int64 IDs."""

    coords: np.ndarray
    ids: np.ndarray

    def __post_init__(self):
        self.coords = np.ascontiguousarray(self.coords, dtype=np.float64)
        self.ids = np.ascontiguousarray(self.ids, dtype=np.int64)
        if self.coords.ndim != 2 or self.coords.shape[1] != 6:
            raise ValueError("coords must be (n, 6)")
        if self.ids.shape != (self.coords.shape[0],):
            raise ValueError("ids must be (n,)")

    @property
    def n(self) -> int:
        return self.coords.shape[0]

    def columns(self) -> list[np.ndarray]:
        return [np.ascontiguousarray(self.coords[:, i]) for i in range(6)]

    def copy(self) -> "Beam":
        return Beam(self.coords.copy(), self.ids.copy())


def gaussian_beam(n: int, seed: int, emit_x: float, emit_y: float, beta_x: float, alpha_x: float, beta_y: float,
                  alpha_y: float, sigma_s: float, sigma_delta: float, eta_x: float = 0.0, etap_x: float = 0.0,
                  chirp: float = 0.0, centred: bool = True, first_id: int = 1) -> Beam:
    """6-D Gaussian bunch matched to the given Twiss parameters.

    Transverse: u = sqrt(eps*beta) g1, u' = sqrt(eps/beta) (g2 - alpha g1) per
    plane, plus dispersion (eta, eta') times delta.  Longitudinal: s ~ N(0,
    sigma_s), delta ~ N(0, sigma_delta) + chirp * s (elegant's
    momentum_chirp, dp/p per metre).  ``centred`` removes the sample means.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((n, 6))
    if centred and n > 1:
        g -= g.mean(axis=0)
    c = np.empty((n, 6))
    for p, (eps, beta, alpha) in enumerate(((emit_x, beta_x, alpha_x), (emit_y, beta_y, alpha_y))):
        c[:, 2 * p] = math.sqrt(eps * beta) * g[:, 2 * p]
        c[:, 2 * p + 1] = math.sqrt(eps / beta) * (g[:, 2 * p + 1] - alpha * g[:, 2 * p])
    c[:, 4] = sigma_s * g[:, 4]
    c[:, 5] = sigma_delta * g[:, 5] + chirp * c[:, 4]
    c[:, 0] += eta_x * c[:, 5]
    c[:, 1] += etap_x * c[:, 5]
    return Beam(c, np.arange(first_id, first_id + n, dtype=np.int64))
