"""elegant's momentum-aperture scan (momentumAperture.c:456-657, output_mode
0, fiducialize 0 or 1) restated one trial at a time, on the CPU oracles: the
check for elegant_b200.momentum_aperture, which runs all trials of a
refinement level at once.  Test infrastructure only."""
import math

import numpy as np

from elegant_b200 import Element, Lattice
from elegant_b200.beam import Beam
from elegant_b200.momentum_aperture import select_elements, wedge_lattice
from reforacle import with_fiducial


def _with_wedge(wl: Lattice, wedge_index: int, x0: float, y0: float, delta: float) -> Lattice:
    els = list(wl.elements)
    e = els[wedge_index]
    els[wedge_index] = Element(e.name, e.type, dict(e.params, DX=x0, DY=y0, DP=delta))
    return Lattice(els)


def fiducial_time(oracle, lattice, p_central):
    """fiducialize = 1 (momentumAperture.c:385-410): the on-momentum particle
    from the origin, one pass, FIRST_BEAM_IS_FIDUCIAL; its RFCA fiducial time
    (the lattice has one RFCA).  Trials then keep it, given as T_REFERENCE."""
    assert sum(e.type == "RFCA" for e in lattice.elements) == 1
    _, n_left, _ = oracle.track(lattice, np.zeros((1, 6)), np.array([1]), p_central, 1)[:3]
    assert n_left == 1, "Fiducial particle lost"
    return oracle.last_fiducial_t0()


def serial_momentum_aperture(oracle, lattice, p_central, n_passes, x_initial=1e-5, y_initial=1e-5,
                             delta_negative_limit=-0.10, delta_positive_limit=0.10, delta_step_size=0.0025,
                             splits=1, steps_back=1, split_step_divisor=10, fiducialize=False, **select):
    """Per selected element and side: (deltaSurvived, deltaLost,
    lostOnPass), each trial one oracle run of one particle."""
    locs = select_elements(lattice, **select)
    wl, wedges = wedge_lattice(lattice, locs, 0 if n_passes == 1 else 1)
    t0 = fiducial_time(oracle, lattice, p_central) if fiducialize else None
    out = []
    for k, _ in enumerate(locs):
        row = []
        for side in (0, 1):
            sign = -1 if side == 0 else 1
            delta_start = 0.0
            delta_lost = sign * 1.7976931348623157e308 / 2
            interval = delta_step_size * sign
            limit = delta_negative_limit if side == 0 else delta_positive_limit
            survived, lost_on_pass = 0.0, -1
            for split in range(splits + 1):
                delta = delta_start
                while abs(delta) <= abs(limit):
                    lat = _with_wedge(wl, wedges[k], x_initial, y_initial, delta)
                    if t0 is not None:
                        lat = with_fiducial(lat, t0)
                    rows, n_left, _ = oracle.track(lat, np.zeros((1, 6)), np.array([1]), p_central, n_passes)[:3]
                    if n_left == 0:
                        lost_on_pass = int(rows[0, 7])
                        delta_lost = delta
                        break
                    survived = delta
                    delta += interval
                delta_start = survived - steps_back * interval
                interval /= split_step_divisor
                delta_start += interval
                limit = delta_lost
                if (delta_start < 0 and sign == 1) or (delta_start > 0 and sign == -1):
                    delta_start = 0
            row.append((survived, delta_lost if abs(delta_lost) < 1e300 else None, lost_on_pass))
        out.append(row)
    return out


def oracle_trials(oracle):
    """track_trials for elegant_b200.momentum_aperture on a CPU oracle: each
    instance (its set of overrides) in its own run.  An instance of two rows
    is (fiducial particle, trial): the fiducial's one-pass run gives the RFCA
    fiducial time, and the trial runs alone with it as T_REFERENCE."""
    def run(wl, offsets, overrides, beam, p_central, n_passes):
        n = beam.n
        lost = np.full(n, -1, dtype=np.int32)
        coords = np.zeros((n, 6))
        t0 = None
        for t in range(len(offsets) - 1):
            els = list(wl.elements)
            for (ie, name, values) in overrides:
                if values[t] != 0:
                    e = els[ie]
                    els[ie] = Element(e.name, e.type, dict(e.params, **{name: float(values[t])}))
            lat = Lattice(els)
            r = offsets[t + 1] - 1  # the trial's row
            if offsets[t + 1] - offsets[t] == 2:
                if t0 is None:
                    t0 = fiducial_time(oracle, wl, p_central)
                lat = with_fiducial(lat, t0)
            rows, n_left, _ = oracle.track(lat, beam.coords[r:r + 1], beam.ids[r:r + 1], p_central, n_passes)[:3]
            coords[r] = rows[0, :6]
            if n_left == 0:
                lost[r] = int(rows[0, 7])
        return lost, coords, math.nan
    return run
