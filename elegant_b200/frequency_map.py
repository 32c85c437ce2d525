"""Frequency map analysis (elegant's &frequency_map, frequencyMap.c:130-320)
on the batched engine.

The reference tracks every grid point (x, y, delta) by itself, one turn per
do_tracking call, recording x, x', y, y' each turn, and takes its tunes with
computeTunesFromTracking (twiss.cc:3799-4032: NAFF of the four signals, then
adjustTuneHalfPlane); with include_changes it goes on from the last
coordinates for a second window and reports the tune change and the
diffusion log10(dnux^2 + dnuy^2).  The RF phase reference comes from one turn
of the reference particle beforehand (frequencyMap.c:180-195).

Here all grid points are one engine run: row 0 of the beam is the reference
particle and the only one that sets the RF phase reference
(fiducial_particles = 1); every pass records the coordinates on the device
(record_tbt); the tunes of both windows come from the NAFF kernel
(b2e_tbt_tunes).  The second window continues the same run for another
turns - 1 passes from the first window's last coordinates, as the
reference's second call does.
"""
from __future__ import annotations

import math

import numpy as np

from .beam import Beam
from .track import Tracker


def grid(xmin, xmax, ymin, ymax, nx, ny, delta_min=0.0, delta_max=0.0, ndelta=1, quadratic_spacing=False):
    """Grid points in the reference's order and arithmetic
    (frequencyMap.c:197-227): delta outermost, then x, then y."""
    dx = dy = 0.0
    if not quadratic_spacing:
        if nx > 1:
            dx = (xmax - xmin) / (nx - 1)
        if ny > 1:
            dy = (ymax - ymin) / (ny - 1)
    ddelta = (delta_max - delta_min) / (ndelta - 1) if ndelta > 1 else 0.0
    pts = []
    for idelta in range(ndelta):
        delta = delta_min + idelta * ddelta
        for ix in range(nx):
            x = xmin + (xmax - xmin) * math.sqrt((ix + 1.0) / nx) if quadratic_spacing else xmin + ix * dx
            for iy in range(ny):
                y = ymin + (ymax - ymin) * math.sqrt((iy + 1.0) / ny) if quadratic_spacing else ymin + iy * dy
                pts.append((x, y, delta))
    return pts


def frequency_map(lattice, p_central, n_passes, xmin=-0.1, xmax=0.1, ymin=1e-6, ymax=0.1, delta_min=0.0,
                  delta_max=0.0, nx=20, ny=21, ndelta=1, include_changes=False, quadratic_spacing=False,
                  full_grid_output=False, reference_coord=None, device=0):
    """Returns rows (dicts) in the reference's output order: x, y, delta,
    nux, nuy, s (path length per turn), and with include_changes dnux, dnuy,
    dnu, dx, dy, diffusion, diffusionRate.  Points whose tunes cannot be
    found (lost, or outside [0, 1]) are left out unless full_grid_output
    (then their tunes are -1)."""
    turns = n_passes // 2 if include_changes else n_passes
    if turns < 4:
        raise ValueError("frequency_map needs at least 4 turns per window")
    ref = np.zeros(6) if reference_coord is None else np.asarray(reference_coord, dtype=np.float64)
    pts = grid(xmin, xmax, ymin, ymax, nx, ny, delta_min, delta_max, ndelta, quadratic_spacing)
    n = len(pts) + 1
    coords = np.tile(ref, (n, 1))
    for k, (x, y, d) in enumerate(pts):
        # computeTunesFromTracking adds y, then x, then delta (twiss.cc:3853-3855)
        coords[k + 1, 2] += y
        coords[k + 1, 0] += x
        coords[k + 1, 5] += d
    ids = np.arange(1, n + 1, dtype=np.int64)
    with Tracker(lattice, p_central, turns - 1, device=device, record_tbt=True, fiducial_particles=1) as t:
        res = t.track(Beam(coords, ids))
        first = t.tbt_tunes(0, turns)
        s_turn = res.coords[:, 4] / turns  # endingCoord[4] / turns (frequencyMap.c:253)
        second = None
        if include_changes:
            t.continue_tracking()  # from the first window's last coordinates (frequencyMap.c:272-281)
            second = t.tbt_tunes(0, turns)
    rows = []
    for k, (x, y, d) in enumerate(pts):
        i = k + 1
        nux, nuy = first["nux"][i], first["nuy"][i]
        bad = not (0 <= nux <= 1 and 0 <= nuy <= 1)
        if bad:
            nux = nuy = -1.0
            if not full_grid_output:
                continue
        row = {"x": x, "y": y, "delta": d, "nux": nux, "nuy": nuy, "s": float(s_turn[i])}
        if include_changes:
            nux2, nuy2, ax2, ay2 = second["nux"][i], second["nuy"][i], second["ax"][i], second["ay"][i]
            diffusion = 0.0
            if bad:
                nux2, nuy2, ax2, ay2 = nux, nuy, first["ax"][i], first["ay"][i]
            elif not (0 <= nux2 <= 1 and 0 <= nuy2 <= 1):
                if not full_grid_output:
                    continue
                nux2, nuy2, ax2, ay2 = nux, nuy, first["ax"][i], first["ay"][i]
            else:
                diffusion = math.log10((nux2 - nux) ** 2 + (nuy2 - nuy) ** 2)
            row.update(dnux=abs(nux2 - nux), dnuy=abs(nuy2 - nuy),
                       dnu=math.sqrt((nux2 - nux) ** 2 + (nuy2 - nuy) ** 2),
                       dx=abs(first["ax"][i] - ax2), dy=abs(first["ay"][i] - ay2), diffusion=diffusion,
                       diffusionRate=0.0 if diffusion == 0 else diffusion / 2 - math.log10(turns))
        rows.append(row)
    return rows
