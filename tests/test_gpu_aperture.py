"""Dynamic-aperture search (many-particle mode) on the GPU against the
reference's serial scan (aperture_search.c:296-570) restated here over the
reference's own tracking code (oracle/_ref, shared maths)."""
import numpy as np
import pytest

from elegant_b200 import Element, Lattice, workloads as w
from elegant_b200.aperture import find_aperture_mp, scan_points

pytestmark = pytest.mark.gpu


def serial_scan(ref, lat, p0, n_passes, xmin, xmax, ymin, ymax, nx, ny):
    """The reference's loop: per round, the not-yet-found rows' next point,
    tracked together; a survivor ends its row's scan."""
    ys, xl, xr = scan_points(xmin, xmax, ymin, ymax, nx, ny)
    out = {}
    for side, xs in (("left", xl), ("right", xr)):
        found = {}
        k = 0
        todo = list(range(len(ys)))
        while todo and k < len(xs):
            c = np.zeros((len(todo), 6))
            c[:, 0] = xs[k]
            c[:, 2] = [ys[iy] for iy in todo]
            rows, nl, _, _ = ref.track(lat, c, np.arange(1, len(todo) + 1), p0, n_passes)
            alive_ids = {int(r[6]) for r in rows[:nl]}
            for j, iy in enumerate(todo):
                if j + 1 in alive_ids:
                    found[iy] = xs[k]
            todo = [iy for iy in todo if iy not in found]
            k += 1
        out[side] = found
    left = [(out["left"][iy], ys[iy]) for iy in range(len(ys)) if iy in out["left"]]
    right = [(out["right"][iy], ys[iy]) for iy in range(len(ys)) if iy in out["right"]]
    return left + right[::-1]


def test_many_particle_aperture_matches_serial_scan(ref_b2e):
    lat, p0 = w.fodo_ring(), w.ring_p_central()
    args = dict(xmin=-0.03, xmax=0.03, ymin=0.0, ymax=0.02, nx=13, ny=5)
    (res,), effort = find_aperture_mp(lat, p0, 25, compact_every=3, **args)
    ref = serial_scan(ref_b2e, lat, p0, 25, **args)
    assert res["boundary"] == ref
    assert 0 < res["survivors"] < res["points"]


def test_aperture_ensemble_of_lattices():
    """Several error seeds scanned in one run equal the same seeds scanned one
    at a time."""
    lat, _, _, overrides = w.ensemble(n_instances=3, n_min=10, n_max=20, seed=41)
    args = dict(xmin=-0.025, xmax=0.025, ymin=0.0, ymax=0.015, nx=11, ny=4)
    together, _ = find_aperture_mp(lat, w.ring_p_central(), 15, overrides=overrides, n_instances=3, **args)
    for i in range(3):
        els = []
        for j, e in enumerate(lat.elements):
            params = dict(e.params)
            for (ie, name, vals) in overrides:
                if ie == j:
                    params[name] = float(vals[i])
            els.append(Element(e.name, e.type, params))
        (alone,), _ = find_aperture_mp(Lattice(els), w.ring_p_central(), 15, **args)
        assert together[i]["boundary"] == alone["boundary"]
        assert np.array_equal(together[i]["alive"], alone["alive"])
