"""elegant's momentum-aperture scan (momentumAperture.c:456-657, output_mode
0, fiducialize 0) restated one trial at a time, on the CPU oracles: the check
for elegant_b200.momentum_aperture, which runs all trials of a refinement
level at once.  Test infrastructure only."""
import math

import numpy as np

from elegant_b200 import Element, Lattice
from elegant_b200.beam import Beam
from elegant_b200.momentum_aperture import select_elements, wedge_lattice


def _with_wedge(wl: Lattice, wedge_index: int, x0: float, y0: float, delta: float) -> Lattice:
    els = list(wl.elements)
    e = els[wedge_index]
    els[wedge_index] = Element(e.name, e.type, dict(e.params, DX=x0, DY=y0, DP=delta))
    return Lattice(els)


def serial_momentum_aperture(oracle, lattice, p_central, n_passes, x_initial=1e-5, y_initial=1e-5,
                             delta_negative_limit=-0.10, delta_positive_limit=0.10, delta_step_size=0.0025,
                             splits=1, steps_back=1, split_step_divisor=10, **select):
    """Per selected element and side: (deltaSurvived, deltaLost,
    lostOnPass), each trial one oracle run of one particle."""
    locs = select_elements(lattice, **select)
    wl, wedges = wedge_lattice(lattice, locs, 0 if n_passes == 1 else 1)
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
    instance (one particle, one set of overrides) in its own run."""
    def run(wl, offsets, overrides, beam, p_central, n_passes):
        n = beam.n
        lost = np.full(n, -1, dtype=np.int32)
        coords = np.zeros((n, 6))
        for t in range(n):
            els = list(wl.elements)
            for (ie, name, values) in overrides:
                if values[t] != 0:
                    e = els[ie]
                    els[ie] = Element(e.name, e.type, dict(e.params, **{name: float(values[t])}))
            rows, n_left, _ = oracle.track(Lattice(els), beam.coords[t:t + 1], beam.ids[t:t + 1], p_central,
                                           n_passes)[:3]
            coords[t] = rows[0, :6]
            if n_left == 0:
                lost[t] = int(rows[0, 7])
        return lost, coords, math.nan
    return run
