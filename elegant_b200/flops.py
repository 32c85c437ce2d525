"""Algorithmic FP64 operation count per particle-turn, for the roofline.

The count follows the element maps as the reference writes them
(multipole.c, csbend.c, simple_rfca.c, matrix.c, limit_amplitudes.c): every
+, -, *, / and sqrt counts 1, comparisons and sign flips 0, and every call
of an elementary function (sin, cos, asin, tan) counts a fixed
ELEMENTARY_WEIGHT = 20 operations, whatever implementation evaluates it --
the order of a double-precision polynomial kernel plus its argument
reduction.  So the figure depends on the lattice and the reference's
formulas only: making the engine's own sin/cos/asin cheaper, or its
divisions and square roots (each a short Newton sequence on the FP64 pipe),
does not move it.  The ncu pipe counters in profiles/ give the hardware
view (FP64 pipe busy, issue slots busy) beside it.
"""
from __future__ import annotations

from .lattice import Lattice

ELEMENTARY_WEIGHT = 20

M2S = 9            # convertMomentaToSlopes: (1+d)^2 - qx^2 - qy^2, sqrt, 2 divisions
APERTURE_IN = 7    # checkMultAperture, elliptical: x+dx, y+dy, 2 div, 2 mul, add
APERTURE_AFTER = 5  # elimit_amplitudes: 2 mul, 2 div, add
DRIFT_SUB = 11     # kick-integrator drift substep: x, y (2 each), s (7)
BEND_DRIFT_ARITH = 27  # integrate_csbend_ordn drift substep without its elementary functions
BEND_DRIFT_CALLS = 4   # asin(QX/f), sin and cos of (ds/rho0 + phi), cos(phi)
BEND_KICK = 14         # its kick: (1 + X/rho0), two products and divisions, the (1+d) round trip
EDGE_ARITH, EDGE_CALLS = 8, 1   # edge focusing: tan(E - psi/(1+d)) and the products
RFCA_ARITH, RFCA_CALLS = 44, 1  # energy kick sin(omega t + phase) and the slope update


def _nsub(order: int) -> int:
    return {2: 2, 4: 4, 6: 8}[order]


def element_counts(e, has_aperture: bool) -> tuple[int, int]:
    """(arithmetic operations, elementary-function calls) of one element."""
    t = e.type
    ap_after = APERTURE_AFTER if has_aperture else 0
    if t == "DRIF":
        order = int(e.get("ORDER")) or 2
        return (11 if order >= 2 else 6) + ap_after, 0
    if t == "EDRIFT":
        return 11 + ap_after, 0
    if t in ("KQUAD", "KSEXT"):
        integ = int(e.get("INTEGRATION_ORDER"))
        n_kicks = int(e.get("N_KICKS"))
        n_slices = int(e.get("N_SLICES"))
        if n_kicks > 0:
            n_slices = max(1, -(-n_kicks // integ)) if integ > 2 else n_kicks
        nsub = _nsub(integ)
        kick = 4 if t == "KQUAD" else 10
        if t == "KSEXT":
            kick += 4 * ((e.get("K1") != 0) + (e.get("J1") != 0))
        per_slice = (APERTURE_IN if has_aperture else 2) + nsub * DRIFT_SUB + (nsub - 1) * (kick + M2S + 4 + M2S)
        mis = 26 if (e.get("DX") or e.get("DY") or e.get("DZ")) else 0
        return 20 + n_slices * per_slice + (APERTURE_IN if has_aperture else 2) + M2S + 1 + mis + ap_after, 0
    if t == "CSBEND":
        nsub = _nsub(int(e.get("INTEGRATION_ORDER")))
        n_slices = int(e.get("N_SLICES"))
        per_slice = (5 if has_aperture else 0) + nsub * BEND_DRIFT_ARITH + (nsub - 1) * BEND_KICK
        n_edges = (e.get("EDGE1_EFFECTS") != 0) + (e.get("EDGE2_EFFECTS") != 0)
        entry, canon, tail = 23, 9 + 9, 5 + 15 + 30
        arith = entry + canon + n_slices * per_slice + tail + EDGE_ARITH * n_edges + ap_after
        return arith, n_slices * nsub * BEND_DRIFT_CALLS + EDGE_CALLS * n_edges
    if t == "RFCA":
        return RFCA_ARITH + ap_after, RFCA_CALLS
    if t == "MAXAMP":
        return ap_after, 0
    return 0, 0


def counts_per_particle_turn(lattice: Lattice) -> tuple[int, int]:
    arith = calls = 0
    has_ap = any(e.type == "MAXAMP" for e in lattice.elements)
    for e in lattice.elements:
        a, c = element_counts(e, has_ap)
        arith += a
        calls += c
    return arith, calls


def flops_per_particle_turn(lattice: Lattice) -> int:
    arith, calls = counts_per_particle_turn(lattice)
    return arith + ELEMENTARY_WEIGHT * calls
