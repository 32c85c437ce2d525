"""Momentum-aperture search (elegant's &momentum_aperture, output_mode 0,
momentumAperture.c:243-700) on the batched engine.

The reference, for every selected element and each sign of the momentum
offset, tracks one particle at a time: the particle starts on the design
orbit (zero coordinates), and when it reaches the element after the selected
one on pass 1 (pass 0 for a one-pass run) a tracking "wedge" offsets it by
(x_initial, y_initial, delta) through offset_beam (momentumAperture.c:34-45).
Each scan steps delta from its start by delta_step_size until a particle is
lost; each of the `splits` refinements restarts steps_back steps behind the
last survivor with a step split_step_divisor times smaller, up to the first
loss (:540-657).  Every run is its own fiducial beam (fiducialize = 0:
delete_phase_references before each run).

Particle fates are independent, so each refinement level is one engine run
holding every trial of every element and side at once: one ensemble instance
per trial (so that each trial's RF phase reference comes from that particle
alone, as in the reference), a MALIGN element after every selected element
carrying the wedge (ON_PASS = the firing pass; per-instance overrides set DX,
DY and DP on the trial's own element and leave the others at zero, where
offset_beam changes nothing).  The deltas come from the same repeated
additions, so the first loss of each scan, the last survivor before it and
the next level's start are the reference's, bit for bit.

fiducialize = 1 (:385-410, :527, :560-566): one on-momentum particle from
the origin is tracked first and sets the RF phase references, which every
trial then keeps.  Batched: each instance carries that fiducial particle as
its first row and the trial as its second; the engine takes the phase
reference from the first row alone (fiducial_particles = 1), and the wedge
acts on the trial's particle ID only (MALIGN START_PID = END_PID), so the
fiducial row runs the reference's fiducial run (one pass) in every
instance.  A fiducial particle lost on that pass stops the search, as in
the reference.

output_mode 1 (one row per element and side, :141-160, :715-731) is a layout
of the same results (elegant_b200.sdds.write_momentum_aperture).

output_mode 2 (multiparticleLocalMomentumAcceptance, :840-1120, Pelegant
only) tracks a fixed grid of deltas at every selected element in one beam
and takes, per element and side, the lost delta nearest zero, one step back:
local_momentum_acceptance.

Tunes (:569-603, determineTunesFromTrackingData :1125-1162): the reference
records every trial's x, x', y, y' at the wedge from the firing pass on and,
for a particle that survives more than two recorded turns, takes its tunes
by NAFF with adjustTuneHalfPlane; the last survivor's tunes are the nuxLost /
nuyLost columns.  Here the engine records the turns at the end of each pass
(record_tbt; the same turns, so the same tunes up to NAFF's resolution) and
the NAFF kernel gives the tunes.  forbid_resonance_crossing (:515-538,
:569-590): the tunes of a zero-delta trial at each element are the nominal
ones, and a trial whose tunes cannot be found, or whose integer part of
twice a tune differs from the nominal one, counts as lost; for such a
trial the reference reports its final coordinates and whatever loss pass
its coordinate array held from an earlier trial (reported here as -1).
The NAFF kernel takes 4 to 8192 turns: with three recorded turns (4
passes) the reference finds tunes and this module reports -1.

Not built: include patterns with wildcards other than '*' and '?'.
"""
from __future__ import annotations

import fnmatch
import math

import numpy as np

from .beam import Beam
from .lattice import Element, Lattice
from .track import Tracker

WEDGE = "MA_WEDGE"


def wedge_lattice(lattice: Lattice, locations, fire_on_pass: int) -> tuple[Lattice, list[int]]:
    """The lattice with a zero MALIGN wedge where each selected element's
    wedge fires: before the element that follows it, or before the first
    selected element for the line's last element (momentumAperture.c:517-518).
    Returns it and the wedges' element indices, in the order of locations."""
    last = len(lattice.elements) - 1
    before = {}  # element index -> selected elements whose wedge goes just before it
    for i in locations:
        before.setdefault(i + 1 if i < last else locations[0], []).append(i)
    els, at = [], {}
    for i, e in enumerate(lattice.elements):
        for src in before.get(i, []):
            at[src] = len(els)
            els.append(Element(f"{WEDGE}{src}", "MALIGN", {"ON_PASS": fire_on_pass}))
        els.append(e)
    return Lattice(els), [at[i] for i in locations]


def select_elements(lattice: Lattice, s_start=0.0, s_end=math.inf, include_name_pattern=None,
                    include_type_pattern=None, skip_elements=0, process_elements=2 ** 31 - 1):
    """Element indices in the reference's order and selection
    (momentumAperture.c:282-300): end position in [s_start, s_end), name and
    type patterns, the first skip_elements matches skipped, at most
    process_elements."""
    out, z, skip = [], 0.0, skip_elements
    for i, e in enumerate(lattice.elements):
        z += e.length
        if not (len(out) < process_elements and z < s_end):
            break
        if z >= s_start and (include_name_pattern is None or fnmatch.fnmatchcase(e.name, include_name_pattern)) and \
                (include_type_pattern is None or fnmatch.fnmatchcase(e.type, include_type_pattern)):
            if skip > 0:
                skip -= 1
                continue
            out.append(i)
    return out


def scan_deltas(start: float, interval: float, limit: float) -> list[float]:
    """The deltas one scan tries: start, start + interval, ... while
    |delta| <= |limit| (repeated additions, momentumAperture.c:543-643)."""
    out, d = [], start
    while abs(d) <= abs(limit):
        out.append(d)
        d += interval
        if len(out) > 10_000_000:
            raise ValueError("momentum aperture scan does not end")
    return out


def momentum_aperture(lattice: Lattice, p_central: float, n_passes: int, x_initial=1e-5, y_initial=1e-5,
                      delta_negative_limit=-0.10, delta_positive_limit=0.10, delta_negative_start=0.0,
                      delta_positive_start=0.0, delta_step_size=0.0025, splits=1, steps_back=1,
                      split_step_divisor=10, s_start=0.0, s_end=math.inf, include_name_pattern=None,
                      include_type_pattern=None, skip_elements=0, process_elements=2 ** 31 - 1,
                      soft_failure=False, fiducialize=False, forbid_resonance_crossing=False, device=0,
                      compact_every=0, track_trials=None):
    """Returns one dict per selected element: name, type, s (its end),
    index, occurrence (1-based among the elements of its name), and per side
    ('negative', 'positive'): delta (last survivor),
    found (a loss was found), lost_on_pass, x_lost, y_lost, s_lost (end of
    the element of the loss), delta_when_lost (the particle's delta there),
    delta_lost (the first lost trial's offset), nux and nuy (the last
    survivor's tunes: 0 without a survivor, -1 when none were found).  Also
    returns the number of particle-turns tracked.  track_trials(lattice,
    offsets, overrides, beam, p_central, n_passes) -> (lost_pass, coords at
    the end or at loss, effort[, (nux, nuy)]), rows in beam order, replaces
    the engine (used to check the batching against a CPU tracker); with
    fiducialize the beam has two rows per instance, the fiducial particle
    first; without the tunes item every trial's tunes are -1."""
    if delta_negative_limit >= 0 or delta_positive_limit <= 0 or delta_negative_start > 0 or \
            delta_positive_start < 0 or delta_step_size <= 0 or splits < 0 or s_start >= s_end:
        raise ValueError("momentum_aperture: invalid limits, starts, step, splits or s range "
                         "(momentumAperture.c:80-101)")
    locs = select_elements(lattice, s_start, s_end, include_name_pattern, include_type_pattern, skip_elements,
                           process_elements)
    if not locs:
        raise ValueError("no elements found between s_start and s_end for momentum aperture computation")
    fire = 0 if n_passes == 1 else 1
    # turns recorded from the firing pass on; tunes when more than two (momentumAperture.c:568)
    n_turns = n_passes - fire
    tune_window = None
    if n_turns > 2:
        collective = any(e.type in ("CSRCSBEND", "CSRDRIFT") for e in lattice.elements)
        if 4 <= n_turns <= 8192 and compact_every == 0 and not collective:
            tune_window = (fire + 1, n_turns)
        elif forbid_resonance_crossing:
            raise ValueError("forbid_resonance_crossing needs 4 to 8192 recorded turns (n_passes 5 to 8193), "
                             "no compact_every and no CSR elements")
    wl, wedges = wedge_lattice(lattice, locs, fire)
    z_end = np.cumsum([e.length for e in lattice.elements])
    wl_end = np.cumsum([e.length for e in wl.elements])
    limits = (delta_negative_limit, delta_positive_limit)
    starts = (delta_negative_start, delta_positive_start)
    # per (location, side) scan state, as in the reference's loop variables
    st = []
    for k, _ in enumerate(locs):
        for side in (0, 1):
            sign = -1 if side == 0 else 1
            st.append({"k": k, "side": side, "sign": sign, "start": starts[side], "interval": delta_step_size * sign,
                       "limit": limits[side], "lost": sign * 1.7976931348623157e308 / 2, "survived": 0.0,
                       "survivor": False, "loser": False, "lost_on_pass": -1, "x_lost": 0.0, "y_lost": 0.0,
                       "s_lost": 0.0, "delta_lost_at": 0.0, "active": True, "nux": 0.0, "nuy": 0.0})
    effort = 0.0
    nominal = None
    if forbid_resonance_crossing and tune_window is not None:
        # the nominal tunes: a zero-delta trial at each element (momentumAperture.c:515-538)
        lp, _, _, eff, tunes = _track_trials(wl, wedges, st, [(2 * k, 0.0) for k in range(len(locs))], p_central,
                                             n_passes, x_initial, y_initial, device, 0, track_trials, fiducialize,
                                             tune_window)
        effort += eff
        nominal = list(zip(*tunes)) if tunes is not None else None
        if nominal is None or (lp >= 0).any() or not all(_tunes_found(nu) for nu in nominal):
            raise RuntimeError("Fiducial particle tune is undefined. (momentumAperture.c:529-533)")
    for split in range(splits + 1):
        trials = []  # (scan index, delta)
        for j, s in enumerate(st):
            if s["active"]:
                trials += [(j, d) for d in scan_deltas(s["start"], s["interval"], s["limit"])]
        if trials:
            lost_pass, c, lost_elem, eff, tunes = _track_trials(wl, wedges, st, trials, p_central, n_passes,
                                                                x_initial, y_initial, device, compact_every,
                                                                track_trials, fiducialize, tune_window)
            effort += eff
            x_l, y_l, s_fin, dpl = c[:, 0], c[:, 2], c[:, 4], c[:, 5]
            done = set()
            for t, (j, d) in enumerate(trials):
                if j in done:
                    continue
                s = st[j]
                nu = (float(tunes[0][t]), float(tunes[1][t])) if tunes is not None else (-1.0, -1.0)
                if lost_pass[t] >= 0:
                    s.update(lost_on_pass=int(lost_pass[t]), x_lost=float(x_l[t]), y_lost=float(y_l[t]),
                             delta_lost_at=float(dpl[t]), loser=True,
                             s_lost=float(wl_end[lost_elem[t]]) if lost_elem[t] >= 0 else 0.0)
                    s["lost"] = d
                    done.add(j)
                elif nominal is not None and _crosses(nu, nominal[s["k"]]):
                    # counted as lost with its final coordinates (momentumAperture.c:569-612)
                    s.update(lost_on_pass=-1, x_lost=float(x_l[t]), y_lost=float(y_l[t]),
                             delta_lost_at=(float(dpl[t]) - p_central) / p_central, loser=True,
                             s_lost=float(s_fin[t]))
                    s["lost"] = d
                    done.add(j)
                else:
                    s["survived"] = d
                    s["survivor"] = True
                    s["nux"], s["nuy"] = nu
        for s in st:
            if not s["active"]:
                continue
            stop = False
            if split == 0:
                if not s["survivor"]:
                    if not soft_failure:
                        raise RuntimeError(f"No survivor found for initial scan for element index {locs[s['k']]}")
                    s["survived"], s["survivor"], stop = 0.0, True, True
                if not s["loser"]:
                    if not soft_failure:
                        raise RuntimeError(f"No loss found for initial scan for element index {locs[s['k']]}")
                    s["loser"], stop = True, True
            s["start"] = s["survived"] - steps_back * s["interval"]
            s["interval"] /= split_step_divisor
            s["start"] += s["interval"]
            s["limit"] = s["lost"]
            if (s["start"] < 0 and s["sign"] == 1) or (s["start"] > 0 and s["sign"] == -1):
                s["start"] = 0
            if stop:
                s["active"] = False
    out = []
    for k, i in enumerate(locs):
        e = lattice.elements[i]
        occurrence = sum(1 for f in lattice.elements[:i + 1] if f.name == e.name)
        row = {"index": i, "name": e.name, "type": e.type, "s": float(z_end[i]), "occurrence": occurrence}
        for side, label in ((0, "negative"), (1, "positive")):
            s = st[2 * k + side]
            row[label] = {"delta": s["survived"], "found": s["loser"], "lost_on_pass": s["lost_on_pass"],
                          "x_lost": s["x_lost"], "y_lost": s["y_lost"], "s_lost": s["s_lost"],
                          "delta_when_lost": s["delta_lost_at"],
                          "delta_lost": s["lost"] if s["loser"] and abs(s["lost"]) < 1e300 else None,
                          "nux": s["nux"], "nuy": s["nuy"]}
        out.append(row)
    return out, effort


def _tunes_found(nu) -> bool:
    return all(0.0 <= v <= 1.0 for v in nu)


def _crosses(nu, nominal) -> bool:
    """forbid_resonance_crossing's test (momentumAperture.c:569-590): no tunes,
    or a different integer part of twice either tune (C truncation)."""
    if not _tunes_found(nu):
        return True
    return int(2 * nu[0]) != int(2 * nominal[0]) or int(2 * nu[1]) != int(2 * nominal[1])


def _track_trials(wl, wedges, st, trials, p_central, n_passes, x_initial, y_initial, device, compact_every,
                  track_trials=None, fiducialize=False, tune_window=None):
    """One engine run, one instance per trial: the trial's particle alone, or
    (fiducialize) the fiducial particle, ID 2t+1, then the trial's, ID 2t+2.
    Returns the trials' loss passes, coordinates (at the end or at the
    loss, n x 6), loss elements, the effort and, with tune_window = (first
    record, records), the trials' tunes (nux, nuy) from the turn-by-turn
    records (None when the tracker gives none)."""
    n = len(trials)
    per = 2 if fiducialize else 1
    coords = np.zeros((per * n, 6))
    ids = np.arange(1, per * n + 1, dtype=np.int64)
    offsets = np.arange(0, per * n + 1, per, dtype=np.int64)
    trial_id = ids[per - 1::per].astype(np.float64)
    overrides = []
    for w_k, wi in enumerate(wedges):
        dx = np.zeros(n)
        dy = np.zeros(n)
        dp = np.zeros(n)
        pid = np.full(n, -1.0)
        for t, (j, d) in enumerate(trials):
            if st[j]["k"] == w_k:
                dx[t], dy[t], dp[t] = x_initial, y_initial, d
                pid[t] = trial_id[t]
        overrides += [(wi, "DX", dx), (wi, "DY", dy), (wi, "DP", dp)]
        if fiducialize:
            overrides += [(wi, "START_PID", pid), (wi, "END_PID", pid)]
    beam = Beam(coords, ids)
    tunes = None
    if track_trials is not None:
        got = track_trials(wl, offsets, overrides, beam, p_central, n_passes)
        lost_pass, c, effort = got[:3]
        if tune_window is not None and len(got) > 3:
            tunes = (np.asarray(got[3][0], dtype=np.float64), np.asarray(got[3][1], dtype=np.float64))
        lost_elem = np.full(per * n, -1)
    else:
        with Tracker(wl, p_central, n_passes, device=device, compact_every=compact_every,
                     fiducial_particles=1 if fiducialize else 0, record_tbt=tune_window is not None) as t:
            t.load_ensemble(offsets, overrides)
            res = t.track(beam)
            if tune_window is not None:
                nu = t.tbt_tunes(*tune_window)  # rows in upload order: no compaction with record_tbt
                tunes = (nu["nux"], nu["nuy"])
        order = np.argsort(res.ids)
        lost_pass, c, lost_elem, effort = res.lost_pass[order], res.coords[order], res.lost_element[order], res.effort
    if fiducialize:
        # the reference's fiducial run is one pass (momentumAperture.c:396-404)
        if (lost_pass[0::2] == 0).any():
            raise RuntimeError("Fiducial particle lost. Don't know what to do. (momentumAperture.c:400-404)")
        lost_pass, c, lost_elem = lost_pass[1::2], c[1::2], lost_elem[1::2]
        if tunes is not None:
            tunes = (tunes[0][1::2], tunes[1][1::2])
    return lost_pass, c, lost_elem, effort, tunes


def _has_wildcards(pattern: str) -> bool:
    return any(c in pattern for c in "*?[")


def acceptance_grid(delta_negative_limit: float, delta_positive_limit: float, delta_negative_start: float,
                    delta_positive_start: float, delta_step_size: float):
    """output_mode 2's delta grid (momentumAperture.c:864-866, :823-827):
    n_delta points over both sides, the step that spans them exactly, the
    index where the positive side starts, and the delta of each index, all
    with the reference's operations (C's truncation to long included)."""
    span = (delta_positive_limit - delta_positive_start) + (delta_negative_start - delta_negative_limit)
    n_delta = int(span / delta_step_size + 1)
    if n_delta < 2:
        raise ValueError("momentum_aperture: the delta grid needs two points or more")
    step = span / (n_delta - 1)
    cutover = int((delta_negative_start - delta_negative_limit) / step + 0.5)
    deltas = [delta_negative_limit + i * step if i < cutover else delta_positive_start + (i - cutover) * step
              for i in range(n_delta)]
    return n_delta, step, cutover, deltas


def omni_wedge_lattice(lattice: Lattice, locations, fire_on_pass: int, n_delta: int, x_initial: float,
                       y_initial: float) -> tuple[Lattice, list[int]]:
    """The lattice with a MALIGN wedge at the entrance of each selected
    element, where the omni wedge of output_mode 2 acts (do_tracking.c:839-844
    calls it before the element; momentumOffsetFunctionOmni,
    momentumAperture.c:801-833): on the firing pass it offsets by (x_initial,
    y_initial, delta) the particles whose ID falls in the element's block of
    n_delta IDs.  Returns it and the wedges' element indices."""
    at_loc = {i: k for k, i in enumerate(locations)}
    els, wedges = [], []
    for i, e in enumerate(lattice.elements):
        if i in at_loc:
            k = at_loc[i]
            wedges.append(len(els))
            els.append(Element(f"{WEDGE}{i}", "MALIGN", {"ON_PASS": fire_on_pass, "DX": x_initial, "DY": y_initial,
                                                         "START_PID": k * n_delta,
                                                         "END_PID": k * n_delta + n_delta - 1}))
        els.append(e)
    return Lattice(els), wedges


def local_momentum_acceptance(lattice: Lattice, p_central: float, n_passes: int, x_initial=1e-5, y_initial=1e-5,
                              delta_negative_limit=-0.10, delta_positive_limit=0.10, delta_negative_start=0.0,
                              delta_positive_start=0.0, delta_step_size=0.0025, s_start=0.0, s_end=math.inf,
                              include_name_pattern=None, include_type_pattern=None, skip_elements=0,
                              process_elements=2 ** 31 - 1, starting_coord=None, device=0, compact_every=0,
                              track_trials=None):
    """&momentum_aperture output_mode 2 (multiparticleLocalMomentumAcceptance,
    momentumAperture.c:840-1120) on the batched engine.

    The reference tracks one fiducial particle for one pass
    (FIRST_BEAM_IS_FIDUCIAL, :899-913), then one beam holding, for each of
    the n_elem selected elements and each of the grid's n_delta deltas, a
    particle with ID ie*n_delta + idelta starting at starting_coord (zero by
    default); on pass 1 (pass 0 for a one-pass run) the particles of element
    ie are offset by (x_initial, y_initial, delta) as they enter it.  Every
    lost particle then bounds its element's side: the lost delta nearest
    zero (delta >= 0 is the positive side, :1069-1081), and the reported
    limit is one grid step back from it (:1090-1093); a side without a loss
    reports +-DBL_MAX.

    Batched: one ensemble instance per grid delta, holding the fiducial
    particle first (the engine takes the RF phase reference from it alone,
    fiducial_particles = 1; its ID lies outside every wedge's block) and then
    one particle per selected element; the wedges carry the instance's delta
    as a per-instance DP override.  Every instance's fiducial row runs the
    same first pass as the reference's fiducial run.

    Returns one dict per selected element: index, name, type, s (its end),
    occurrence, and per side ('negative', 'positive'): delta (the reported
    limit), found, delta_lost (the nearest lost delta, None if none); and the
    particle-turns tracked.  track_trials(lattice, offsets, overrides, beam,
    p_central, n_passes) -> (lost_pass, coords, effort), rows in beam order,
    replaces the engine."""
    if delta_negative_limit >= 0 or delta_positive_limit <= 0 or delta_negative_start > 0 or \
            delta_positive_start < 0 or delta_step_size <= 0 or s_start >= s_end or \
            abs(delta_negative_limit - delta_negative_start) <= delta_step_size / 2 or \
            delta_positive_limit - delta_positive_start <= delta_step_size / 2:
        raise ValueError("momentum_aperture: invalid limits, starts, step or s range (momentumAperture.c:80-101)")
    if include_name_pattern is not None and _has_wildcards(include_name_pattern):
        raise ValueError("Can't have wildcards in name pattern for output_mode=2")
    if include_type_pattern is not None:
        raise ValueError("Can't used include_type_pattern for output_mode=2")
    locs = select_elements(lattice, s_start, s_end, include_name_pattern, None, skip_elements, process_elements)
    if not locs:
        raise ValueError("no elements found between s_start and s_end for momentum aperture computation")
    n_delta, step, cutover, deltas = acceptance_grid(delta_negative_limit, delta_positive_limit,
                                                     delta_negative_start, delta_positive_start, delta_step_size)
    n_elem = len(locs)
    n_total = n_elem * n_delta
    fire = 0 if n_passes == 1 else 1
    wl, wedges = omni_wedge_lattice(lattice, locs, fire, n_delta, x_initial, y_initial)

    per = n_elem + 1
    start = np.zeros(6) if starting_coord is None else np.asarray(starting_coord, dtype=np.float64)[:6]
    coords = np.tile(start, (per * n_delta, 1))
    ids = np.empty(per * n_delta, dtype=np.int64)
    for idelta in range(n_delta):
        ids[idelta * per] = n_total + idelta  # the fiducial particle: outside every wedge's ID block
        ids[idelta * per + 1:(idelta + 1) * per] = np.arange(n_elem, dtype=np.int64) * n_delta + idelta
    offsets = np.arange(0, per * n_delta + 1, per, dtype=np.int64)
    dp = np.asarray(deltas, dtype=np.float64)
    overrides = [(wi, "DP", dp) for wi in wedges]
    beam = Beam(coords, ids)
    if track_trials is not None:
        lost_pass, _, effort = track_trials(wl, offsets, overrides, beam, p_central, n_passes)
        lost_pass = np.asarray(lost_pass)
        out_ids = ids
    else:
        with Tracker(wl, p_central, n_passes, device=device, compact_every=compact_every,
                     fiducial_particles=1) as t:
            t.load_ensemble(offsets, overrides)
            res = t.track(beam)
        lost_pass, out_ids, effort = res.lost_pass, res.ids, res.effort

    fid = out_ids >= n_total
    if (lost_pass[fid] == 0).any():
        # the reference's fiducial run is one pass (momentumAperture.c:907-913)
        raise RuntimeError("Fiducial particle lost. Don't know what to do. (momentumAperture.c:907-913)")
    big = 1.7976931348623157e308
    lost_at = [[-big, big] for _ in range(n_elem)]  # deltaLost[side][ie] (:1041-1044)
    found = [[False, False] for _ in range(n_elem)]
    for pid, lp in zip(out_ids[~fid], lost_pass[~fid]):
        if lp < 0:
            continue
        idelta = int(pid) % n_delta
        ie = (int(pid) - idelta) // n_delta
        d = deltas[idelta]
        side = 1 if d >= 0 else 0
        if not found[ie][side] or (d < lost_at[ie][side] if side else d > lost_at[ie][side]):
            found[ie][side] = True
            lost_at[ie][side] = d
    z_end = np.cumsum([e.length for e in lattice.elements])
    out = []
    for k, i in enumerate(locs):
        e = lattice.elements[i]
        occurrence = sum(1 for f in lattice.elements[:i + 1] if f.name == e.name)
        row = {"index": i, "name": e.name, "type": e.type, "s": float(z_end[i]), "occurrence": occurrence}
        for side, label in ((0, "negative"), (1, "positive")):
            lost = lost_at[k][side]
            row[label] = {"delta": lost + step if side == 0 else lost - step, "found": found[k][side],
                          "delta_lost": lost if found[k][side] else None}
        out.append(row)
    return out, effort
