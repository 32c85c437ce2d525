"""Named synthetic workloads with the shapes of the benchmark cases.

- ``fodo_ring``: 3 GeV electrons, 8 FODO cells (DRIF 0.5, KQUAD 0.3 m
  K1=+1.2 N_KICKS=8, DRIF 0.5, 2x CSBEND 1 m 2pi/16 N_KICKS=8, KQUAD -1.2,
  KSEXT 0.2 m K2=+/-5 alternating, 20 mm circular MAXAMP), one zero-length
  RFCA (1 MV, harmonic 100, phase 180 deg: above transition, no net loss).
- ``ring_beam``: 6-D Gaussian, emit 1 nm per plane at the periodic Twiss and
  dispersion of the ring, sigma_delta 1e-3, sigma_s 3 mm, centred.
- ``ensemble``: instances of the ring with seeded quadrupole offsets (50 um
  rms in x and y), quadrupole and sextupole relative strength errors (1e-3,
  1e-2 rms), Gaussians cut at 3 sigma (elegant &error default cutoff), and
  per-instance particle counts uniform in [500, 4000].
- ``chicane``: 1 GeV, four CSRCSBEND (0.5 m, +/-0.05 rad, N_KICKS=20,
  BINS=600, SG_HALFWIDTH=2) with CSRDRIFT 5 m, 1 m, 5 m; 1 nC.
"""
from __future__ import annotations

import math

import numpy as np

from .beam import Beam, gaussian_beam, p_central_from_momentum_mev
from .lattice import Element, Lattice
from .optics import periodic_twiss

C_MKS = 2.99792458e8


def fodo_cell(index: int, ksext: float = 5.0) -> list[Element]:
    ang = 2 * math.pi / 16
    k2 = ksext if index % 2 == 0 else -ksext
    return [
        Element("MA", "MAXAMP", {"X_MAX": 0.02, "Y_MAX": 0.02, "ELLIPTICAL": 1}),
        Element("D1", "DRIF", {"L": 0.5}),
        Element("QF", "KQUAD", {"L": 0.3, "K1": 1.2, "N_KICKS": 8}),
        Element("D2", "DRIF", {"L": 0.5}),
        Element("B1", "CSBEND", {"L": 1.0, "ANGLE": ang, "N_KICKS": 8}),
        Element("B2", "CSBEND", {"L": 1.0, "ANGLE": ang, "N_KICKS": 8}),
        Element("QD", "KQUAD", {"L": 0.3, "K1": -1.2, "N_KICKS": 8}),
        Element("SF" if index % 2 == 0 else "SD", "KSEXT", {"L": 0.2, "K2": k2}),
    ]


RING_P_MEV = 3000.0


def ring_p_central() -> float:
    return p_central_from_momentum_mev(RING_P_MEV)


def fodo_ring(n_cells: int = 8, rf: bool = True, volt: float = 1e6, harmonic: int = 100,
              phase: float = 180.0) -> Lattice:
    els = []
    for c in range(n_cells):
        els += fodo_cell(c)
    if rf:
        circumference = sum(e.length for e in els)
        p = ring_p_central()
        beta = p / math.sqrt(p * p + 1)
        freq = harmonic * C_MKS * beta / circumference
        els.append(Element("RF", "RFCA", {"L": 0.0, "VOLT": volt, "FREQ": freq, "PHASE": phase}))
    return Lattice(els)


def radiating_ring(isr: bool = False, volt: float = 4e6, edge_angle: float = 0.0) -> Lattice:
    """The FODO ring with SYNCH_RAD (and ISR) on its quadrupoles, sextupoles
    and dipoles, and an RF cavity whose voltage and phase replace the energy
    radiated per turn: U0 = C_gamma E^4 / rho (C_gamma = 8.8463e-5 m/GeV^3),
    phase = 180 - asin(U0 / V) degrees (above transition).  edge_angle sets
    E1 = E2 on the dipoles (edge focusing and the edge radiation terms)."""
    base = fodo_ring(rf=False)
    bend = next(e for e in base.elements if e.type == "CSBEND")
    rho = bend.params["L"] / bend.params["ANGLE"]
    e_gev = ring_p_central() * 0.51099895e-3
    u0_mev = 8.8463e-5 * e_gev ** 4 / rho * 1e3
    phase = 180.0 - math.degrees(math.asin(u0_mev / (volt / 1e6)))
    extra = {"SYNCH_RAD": 1}
    if isr:
        extra["ISR"] = 1
    els = []
    for e in fodo_ring(volt=volt, phase=phase).elements:
        if e.type in ("KQUAD", "KSEXT", "CSBEND"):
            params = dict(e.params, **extra)
            if e.type == "CSBEND" and edge_angle:
                params.update(E1=edge_angle, E2=edge_angle)
            e = Element(e.name, e.type, params)
        els.append(e)
    return Lattice(els)


def ring_beam(n: int = 10000, seed: int = 12345, lattice: Lattice | None = None, first_id: int = 1,
              twiss=None) -> Beam:
    """twiss: matched optics to use instead of the periodic solution of the
    lattice (fixture-generated beams pass the values they were made with, so
    that the libm elementary functions of another host cannot move a bit)."""
    tw = twiss or periodic_twiss(lattice or fodo_ring(rf=False))
    return gaussian_beam(n, seed, 1e-9, 1e-9, tw.beta_x, tw.alpha_x, tw.beta_y, tw.alpha_y, 3e-3, 1e-3,
                         eta_x=tw.eta_x, etap_x=tw.etap_x, first_id=first_id)


def _cut_gaussian(rng: np.random.Generator, n: int, sigma: float, cutoff: float = 3.0) -> np.ndarray:
    out = rng.standard_normal(n)
    bad = np.abs(out) > cutoff
    while bad.any():
        out[bad] = rng.standard_normal(int(bad.sum()))
        bad = np.abs(out) > cutoff
    return out * sigma


def ensemble(n_instances: int = 512, seed: int = 2024, n_min: int = 500, n_max: int = 4000,
             lattice: Lattice | None = None, twiss=None):
    """Returns (lattice, beam, offsets, overrides) for a batched error ensemble.

    overrides: list of (element_index, parameter_name, values[n_instances]);
    twiss: as for ring_beam.
    """
    lat = lattice or fodo_ring()
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = rng.integers(n_min, n_max + 1, size=n_instances)
    offsets = np.zeros(n_instances + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(counts)
    overrides = []
    for i, e in enumerate(lat.elements):
        if e.type == "KQUAD":
            overrides.append((i, "DX", _cut_gaussian(rng, n_instances, 50e-6)))
            overrides.append((i, "DY", _cut_gaussian(rng, n_instances, 50e-6)))
            overrides.append((i, "FSE", _cut_gaussian(rng, n_instances, 1e-3)))
        elif e.type == "KSEXT":
            overrides.append((i, "FSE", _cut_gaussian(rng, n_instances, 1e-2)))
    tw = twiss or periodic_twiss(Lattice([e for e in lat.elements if e.type != "RFCA"]))
    parts = []
    next_id = 1
    for i in range(n_instances):
        b = gaussian_beam(int(counts[i]), seed * 7919 + i, 1e-9, 1e-9, tw.beta_x, tw.alpha_x, tw.beta_y,
                          tw.alpha_y, 3e-3, 1e-3, eta_x=tw.eta_x, etap_x=tw.etap_x, first_id=next_id)
        next_id += int(counts[i])
        parts.append(b)
    beam = Beam(np.concatenate([b.coords for b in parts]), np.concatenate([b.ids for b in parts]))
    return lat, beam, offsets, overrides


CHICANE_P_MEV = 1000.0


def chicane(bins: int = 600, n_kicks: int = 20, sg_halfwidth: int = 2, charge: float = 1e-9,
            stupakov: bool = False, drift: dict | None = None) -> Lattice:
    """Four-dipole chicane with CSR (CSRCSBEND L=0.5 m, angle +-0.05, CSRDRIFT
    5/1/5 m).  stupakov: CSRDRIFT USE_STUPAKOV=1 instead of mode 0; drift:
    extra CSRDRIFT parameters (N_KICKS, DZ, CSR)."""
    b = {"L": 0.5, "N_KICKS": n_kicks, "BINS": bins, "SG_HALFWIDTH": sg_halfwidth}
    d = dict(drift or {})
    if stupakov:
        d["USE_STUPAKOV"] = 1
    return Lattice([
        Element("Q", "CHARGE", {"TOTAL": charge}),
        Element("B1", "CSRCSBEND", dict(b, ANGLE=0.05)),
        Element("D1", "CSRDRIFT", dict(d, L=5.0)),
        Element("B2", "CSRCSBEND", dict(b, ANGLE=-0.05)),
        Element("D2", "CSRDRIFT", dict(d, L=1.0)),
        Element("B3", "CSRCSBEND", dict(b, ANGLE=-0.05)),
        Element("D3", "CSRDRIFT", dict(d, L=5.0)),
        Element("B4", "CSRCSBEND", dict(b, ANGLE=0.05)),
    ])


def chicane_beam(n: int = 1_000_000, seed: int = 777, chirp: float = -10.0, sigma_z: float = 1e-3,
                 sigma_delta: float = 1e-4, emit_n: float = 1e-6, beta: float = 10.0) -> Beam:
    p = p_central_from_momentum_mev(CHICANE_P_MEV)
    eps = emit_n / p
    return gaussian_beam(n, seed, eps, eps, beta, 0.0, beta, 0.0, sigma_z, sigma_delta, chirp=chirp)
