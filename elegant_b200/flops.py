"""Algorithmic FP64 operation count per particle-turn, for the roofline.

Counted from the element maps as the reference writes them (multipole.c,
csbend.c, simple_rfca.c, matrix.c, limit_amplitudes.c): every +, -, *, /,
sqrt counts 1, an fma counts 2, comparisons and sign flips count 0.  The
elementary functions count the operations of their implementations in
elegant_b200/csrc/b2e_math.h (asin on |x| <= 2^-6: 10, on |x| <= 1/8: 24;
sin or cos kernel on |x| <= 2^-4: 10 / 13, on |x| <= pi/4: 22 / 27; a pi/2
reduction: 7).  A bend's substep angle decides which sin/cos kernel its
drift takes; its sin(phi) = p_x / p is taken to be below 2^-6 (stored beams).  Division and sqrt are one
operation here although the FP64 pipe executes each as a short Newton
sequence, so the achieved fraction of the DGEMM peak understates pipe
occupancy; the ncu pipe counters in profiles/ give that directly.
"""
from __future__ import annotations

from .lattice import Lattice

ASIN_TINY = 10
ASIN_SMALL = 24
SIN_KERNEL = 22
COS_KERNEL = 27
SIN_SMALL = 10
COS_SMALL = 13
# largest |drift fraction| of the kick integrators: order 2, 4 (Forest-Ruth), 6 (taken as 1)
MAX_DRIFT_FRAC = {2: 0.5, 4: 1.0 / (2.0 * (2.0 - 2.0 ** (1.0 / 3.0))), 6: 1.0}
REDUCTION = 7
TAN = REDUCTION + SIN_KERNEL + COS_KERNEL + 1

M2S = 9            # convertMomentaToSlopes: (1+d)^2 - qx^2 - qy^2, sqrt, 2 divisions
APERTURE_IN = 7    # checkMultAperture, elliptical: x+dx, y+dy, 2 div, 2 mul, add
APERTURE_AFTER = 5  # elimit_amplitudes: 2 mul, 2 div, add
DRIFT_SUB = 11     # kick-integrator drift substep: x, y (2 each), s (7)


def _nsub(order: int) -> int:
    return {2: 2, 4: 4, 6: 8}[order]


def element_flops(e, has_aperture: bool) -> int:
    t = e.type
    ap_after = APERTURE_AFTER if has_aperture else 0
    if t == "DRIF":
        order = int(e.get("ORDER")) or 2
        return (11 if order >= 2 else 6) + ap_after
    if t == "EDRIFT":
        return 11 + ap_after
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
        return 20 + n_slices * per_slice + (APERTURE_IN if has_aperture else 2) + M2S + 1 + mis + ap_after
    if t == "CSBEND":
        integ = int(e.get("INTEGRATION_ORDER"))
        nsub = _nsub(integ)
        n_slices = int(e.get("N_SLICES"))
        angle = abs(float(e.get("ANGLE"))) / max(n_slices, 1) * MAX_DRIFT_FRAC.get(integ, 1.0)
        small = angle + 0.01 <= 2.0 ** -4  # substep angle plus a particle angle within the short kernels
        sn, cs = (SIN_SMALL, COS_SMALL) if small else (SIN_KERNEL, COS_KERNEL)
        drift = 4 + 1 + 2 + ASIN_TINY + 2 + sn + cs + 1 + cs + 1 + 6 + 2 + 3 + 1 + 4
        kick = 10 + 4
        per_slice = (5 if has_aperture else 0) + nsub * drift + (nsub - 1) * kick
        edges = (8 + TAN) * ((e.get("EDGE1_EFFECTS") != 0) + (e.get("EDGE2_EFFECTS") != 0))
        entry, canon, tail = 23, 9 + 9, 5 + 15 + 30
        return entry + canon + n_slices * per_slice + tail + edges + ap_after
    if t == "RFCA":
        return 10 + (2 + REDUCTION + SIN_KERNEL + 3) + 2 + 23 + 4 + ap_after
    if t == "MAXAMP":
        return ap_after
    return 0


def flops_per_particle_turn(lattice: Lattice) -> int:
    total, has_ap = 0, any(e.type == "MAXAMP" for e in lattice.elements)
    seen_ap = False
    for e in lattice.elements:
        seen_ap = seen_ap or e.type == "MAXAMP"
        total += element_flops(e, seen_ap or has_ap)
    return total
