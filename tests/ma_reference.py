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


def serial_local_acceptance(oracle, lattice, p_central, n_passes, x_initial=1e-5, y_initial=1e-5,
                            delta_negative_limit=-0.10, delta_positive_limit=0.10, delta_negative_start=0.0,
                            delta_positive_start=0.0, delta_step_size=0.0025, **select):
    """&momentum_aperture output_mode 2 (multiparticleLocalMomentumAcceptance,
    momentumAperture.c:840-1100) restated one particle per oracle run: the
    grid of :864-866 and :823-827, the offset at the selected element's
    entrance on the firing pass (:801-833), the one-pass fiducial run's RF
    phase for every particle (:899-913), the nearest loss per side
    (:1053-1082) and one grid step back (:1090-1093).  Per selected element:
    ((deltaNegative, nearest negative loss or None), (deltaPositive, ...))."""
    span = (delta_positive_limit - delta_positive_start) + (delta_negative_start - delta_negative_limit)
    n_delta = int(span / delta_step_size + 1)
    step = span / (n_delta - 1)
    cut = int((delta_negative_start - delta_negative_limit) / step + 0.5)
    locs = select_elements(lattice, **select)
    fire = 0 if n_passes == 1 else 1
    t0 = fiducial_time(oracle, lattice, p_central) if any(e.type == "RFCA" for e in lattice.elements) else None
    big = 1.7976931348623157e308
    out = []
    for i in locs:
        lost = [-big, big]
        found = [False, False]
        for idelta in range(n_delta):
            delta = delta_negative_limit + idelta * step if idelta < cut else \
                delta_positive_start + (idelta - cut) * step
            els = list(lattice.elements)
            els.insert(i, Element("WEDGE", "MALIGN", {"DX": x_initial, "DY": y_initial, "DP": delta,
                                                      "ON_PASS": fire}))
            lat = Lattice(els)
            if t0 is not None:
                lat = with_fiducial(lat, t0)
            _, n_left, _ = oracle.track(lat, np.zeros((1, 6)), np.array([1]), p_central, n_passes)[:3]
            if n_left == 0:
                side = 1 if delta >= 0 else 0
                if not found[side] or (delta < lost[side] if side else delta > lost[side]):
                    found[side], lost[side] = True, delta
        out.append(((lost[0] + step, lost[0] if found[0] else None),
                    (lost[1] - step, lost[1] if found[1] else None)))
    return out


def oracle_instances(oracle):
    """track_trials for elegant_b200.momentum_aperture.local_momentum_acceptance
    on a CPU oracle: each instance (its overrides applied) in its own run;
    its first row is the fiducial particle, whose one-pass run gives the RFCA
    fiducial time the other rows keep as T_REFERENCE."""
    def run(wl, offsets, overrides, beam, p_central, n_passes):
        lost = np.full(beam.n, -1, dtype=np.int32)
        coords = np.zeros((beam.n, 6))
        has_rf = any(e.type == "RFCA" for e in wl.elements)
        t0 = fiducial_time(oracle, wl, p_central) if has_rf else None
        for t in range(len(offsets) - 1):
            els = list(wl.elements)
            for (ie, name, values) in overrides:
                e = els[ie]
                els[ie] = Element(e.name, e.type, dict(e.params, **{name: float(values[t])}))
            lat = Lattice(els)
            if t0 is not None:
                lat = with_fiducial(lat, t0)
            a, b = offsets[t] + 1, offsets[t + 1]
            rows, n_left, _ = oracle.track(lat, beam.coords[a:b], beam.ids[a:b], p_central, n_passes)[:3]
            pos = {int(pid): k for k, pid in enumerate(beam.ids[a:b])}
            for j, r in enumerate(rows):
                k = a + pos[int(r[6])]
                coords[k] = r[:6]
                if j >= n_left:  # survivors first, then the lost rows with their pass
                    lost[k] = int(r[7])
        return lost, coords, math.nan
    return run


def serial_scan_with_tunes(run_trial, lattice, n_passes, forbid, x_initial=1e-5, y_initial=1e-5,
                           delta_negative_limit=-0.10, delta_positive_limit=0.10, delta_step_size=0.0025,
                           splits=1, steps_back=1, split_step_divisor=10, **select):
    """The reference's scan (momentumAperture.c:456-657) with its tune logic
    (:515-603): run_trial(lattice with the wedge, n_passes) -> (lost,
    lost_on_pass, tunes or None).  With forbid, a zero-delta trial gives the
    nominal tunes; a surviving trial without tunes, or with another integer
    part of twice a tune, counts as lost (loss pass -1).  The last survivor's
    tunes are kept (0 before any survivor, -1 when none were found).  Per
    selected element and side: (deltaSurvived, deltaLost or None,
    lostOnPass, nux, nuy)."""
    locs = select_elements(lattice, **select)
    wl, wedges = wedge_lattice(lattice, locs, 0 if n_passes == 1 else 1)
    out = []
    for k, _ in enumerate(locs):
        nominal = None
        if forbid:
            lost, _, nominal = run_trial(_with_wedge(wl, wedges[k], x_initial, y_initial, 0.0), n_passes)
            assert not lost and nominal is not None, "Fiducial particle tune is undefined"
        row = []
        for side in (0, 1):
            sign = -1 if side == 0 else 1
            delta_start = 0.0
            delta_lost = sign * 1.7976931348623157e308 / 2
            interval = delta_step_size * sign
            limit = delta_negative_limit if side == 0 else delta_positive_limit
            survived, lost_on_pass, nu = 0.0, -1, (0.0, 0.0)
            for split in range(splits + 1):
                delta = delta_start
                while abs(delta) <= abs(limit):
                    lost, lp, tunes = run_trial(_with_wedge(wl, wedges[k], x_initial, y_initial, delta), n_passes)
                    t = tunes if tunes is not None else (-1.0, -1.0)
                    if not lost and forbid and (not all(0 <= v <= 1 for v in t) or
                                                int(2 * t[0]) != int(2 * nominal[0]) or
                                                int(2 * t[1]) != int(2 * nominal[1])):
                        lost, lp = True, -1
                    if lost:
                        lost_on_pass, delta_lost = lp, delta
                        break
                    survived, nu = delta, t
                    delta += interval
                delta_start = survived - steps_back * interval
                interval /= split_step_divisor
                delta_start += interval
                limit = delta_lost
                if (delta_start < 0 and sign == 1) or (delta_start > 0 and sign == -1):
                    delta_start = 0
            row.append((survived, delta_lost if abs(delta_lost) < 1e300 else None, lost_on_pass, nu[0], nu[1]))
        out.append(row)
    return out


def synthetic_tunes(dp: float):
    """Stand-in tunes of a surviving trial with momentum offset dp, for
    testing the tune bookkeeping on the CPU: x near the half integer with a
    large chromaticity, y far from it."""
    return ((0.455 + 30.0 * dp) % 1.0, 0.277 + 5.0 * dp)


def oracle_trials_with_tunes(oracle):
    """oracle_trials plus stand-in tunes (synthetic_tunes of the instance's
    wedge offset) for every surviving row, -1 for lost rows."""
    base = oracle_trials(oracle)

    def run(wl, offsets, overrides, beam, p_central, n_passes):
        lost, coords, effort = base(wl, offsets, overrides, beam, p_central, n_passes)
        dps = np.zeros(len(offsets) - 1)
        for (_, name, values) in overrides:
            if name == "DP":
                dps += np.asarray(values)
        nux = np.full(beam.n, -1.0)
        nuy = np.full(beam.n, -1.0)
        for t in range(len(offsets) - 1):
            for r in range(offsets[t], offsets[t + 1]):
                if lost[r] < 0:
                    nux[r], nuy[r] = synthetic_tunes(dps[t])
        return lost, coords, effort, (nux, nuy)
    return run


def oracle_run_trial(oracle, p_central):
    """run_trial for serial_scan_with_tunes on a CPU oracle with
    synthetic_tunes of the wedge's DP."""
    def run(lat, n_passes):
        dp = sum(e.params.get("DP", 0.0) for e in lat.elements if e.type == "MALIGN")  # one wedge is set
        rows, n_left, _ = oracle.track(lat, np.zeros((1, 6)), np.array([1]), p_central, n_passes)[:3]
        if n_left == 0:
            return True, int(rows[0, 7]), None
        return False, -1, synthetic_tunes(dp)
    return run
