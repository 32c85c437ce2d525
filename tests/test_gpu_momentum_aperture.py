"""Momentum aperture on the device: every refinement level is one engine run
of one-particle instances with MALIGN wedges; each element's last surviving
offset, first lost offset and loss pass equal elegant's serial scan on its
own code (oracle/_ref), which tracks one particle per run."""
import numpy as np
import pytest

from elegant_b200 import Element, Lattice, Tracker, workloads as w
from elegant_b200.momentum_aperture import momentum_aperture
from ma_reference import serial_momentum_aperture
from reforacle import by_id

pytestmark = pytest.mark.gpu
P0 = w.ring_p_central()


@pytest.mark.parametrize("passes", [1, 40])
def test_momentum_aperture_matches_serial_scan(ref_b2e, passes):
    lat = w.fodo_ring()
    kw = dict(include_type_pattern="K*", process_elements=6, delta_step_size=0.0015, splits=2)
    serial = serial_momentum_aperture(ref_b2e, lat, P0, passes, **kw)
    rows, effort = momentum_aperture(lat, P0, passes, **kw)
    assert effort > 0 and len(rows) == 6
    for row, s in zip(rows, serial):
        for side, label in ((0, "negative"), (1, "positive")):
            got = row[label]
            assert (got["delta"], got["delta_lost"], got["lost_on_pass"]) == s[side], (row["name"], label)


@pytest.mark.parametrize("passes", [1, 40])
def test_fiducialized_momentum_aperture_matches_serial_scan(ref_b2e, passes):
    """fiducialize = 1 on the device (a fiducial row per instance,
    fiducial_particles = 1, the wedge on the trial's ID) against the serial
    scan with one fiducial particle's phase for all trials."""
    from test_momentum_aperture import mid_rf_ring
    lat = mid_rf_ring() if passes == 1 else w.fodo_ring()
    kw = dict(include_type_pattern="K*", process_elements=4, delta_step_size=0.0015, splits=2)
    serial = serial_momentum_aperture(ref_b2e, lat, P0, passes, fiducialize=True, **kw)
    rows, effort = momentum_aperture(lat, P0, passes, fiducialize=True, **kw)
    assert effort > 0 and len(rows) == 4
    for row, s in zip(rows, serial):
        for side, label in ((0, "negative"), (1, "positive")):
            got = row[label]
            assert (got["delta"], got["delta_lost"], got["lost_on_pass"]) == s[side], (row["name"], label)


def test_malign_element_bit_exact(ref_b2e):
    """MALIGN (offset_beam) on one pass and on every pass, with a particle-ID
    window, through the ring: equal to the reference driver."""
    base = w.fodo_ring()
    els = list(base.elements)
    els.insert(5, Element("M1", "MALIGN", {"DX": 1e-4, "DYP": -2e-5, "DZ": 0.01, "DP": 1e-3, "ON_PASS": 1}))
    els.insert(20, Element("M2", "MALIGN", {"DT": 1e-12, "DE": -2e-4, "START_PID": 10, "END_PID": 400}))
    lat = Lattice(els)
    beam = w.ring_beam(1000, seed=44)
    with Tracker(lat, P0, 20) as t:
        res = t.track(beam)
    rows, nl, _, _ = ref_b2e.track(lat, beam.coords, beam.ids, P0, 20)
    ref_c, ref_ids, ref_loss = by_id(rows)
    order = np.argsort(res.ids)
    assert res.n_left == nl
    alive = ref_loss < 0
    assert np.array_equal(res.coords[order][alive], ref_c[alive])


@pytest.mark.parametrize("passes", [1, 40])
def test_local_acceptance_matches_serial_restatement(ref_b2e, passes):
    """output_mode 2 on the device (one instance per grid delta, a fiducial
    row first, the wedges on each element's ID block) against one reference
    run per particle with the fiducial particle's RF phase."""
    from elegant_b200.momentum_aperture import local_momentum_acceptance
    from ma_reference import serial_local_acceptance
    from test_momentum_aperture import mid_rf_ring
    lat = mid_rf_ring() if passes == 1 else w.fodo_ring()
    kw = dict(process_elements=8, delta_step_size=0.0005, delta_negative_limit=-0.02, delta_positive_limit=0.02)
    serial = serial_local_acceptance(ref_b2e, lat, P0, passes, **kw)
    rows, effort = local_momentum_acceptance(lat, P0, passes, **kw)
    assert effort > 0 and len(rows) == len(serial) == 8
    for row, s in zip(rows, serial):
        for side, label in ((0, "negative"), (1, "positive")):
            assert (row[label]["delta"], row[label]["delta_lost"]) == s[side], (row["name"], label)


def _engine_run_trial(n_passes_window_first=2):
    """run_trial for ma_reference.serial_scan_with_tunes on the engine: one
    particle per run, its tunes from the turns recorded after the firing
    pass (records 2..n_passes)."""
    from elegant_b200.beam import Beam

    def run(lat, n_passes):
        with Tracker(lat, P0, n_passes, record_tbt=True) as t:
            res = t.track(Beam(np.zeros((1, 6)), np.array([1], dtype=np.int64)))
            if res.lost_pass[0] >= 0:
                return True, int(res.lost_pass[0]), None
            nu = t.tbt_tunes(n_passes_window_first, n_passes - 1)
        v = (float(nu["nux"][0]), float(nu["nuy"][0]))
        return False, -1, v if all(0 <= x <= 1 for x in v) else None
    return run


@pytest.mark.parametrize("forbid", [False, True])
def test_momentum_aperture_tunes_match_serial_scan(forbid):
    """The last survivor's tunes (nuxLost/nuyLost) and forbid_resonance_crossing
    (momentumAperture.c:515-603) in the batched search against the
    reference's scan run one trial at a time on the engine with the same
    turn-by-turn NAFF; horizontal tune near the half integer (0.545)."""
    from ma_reference import serial_scan_with_tunes
    lat = w.fodo_ring()
    kw = dict(include_type_pattern="K*", process_elements=3, delta_step_size=0.0015, splits=1)
    serial = serial_scan_with_tunes(_engine_run_trial(), lat, 64, forbid, **kw)
    rows, _ = momentum_aperture(lat, P0, 64, forbid_resonance_crossing=forbid, **kw)
    for row, s in zip(rows, serial):
        for side, label in ((0, "negative"), (1, "positive")):
            got = row[label]
            assert (got["delta"], got["delta_lost"], got["lost_on_pass"], got["nux"], got["nuy"]) == s[side], \
                (row["name"], label)
            # the linear optics give the tunes folded into [0, 0.5] (0.455, 0.277); NAFF with
            # adjustTuneHalfPlane unfolds them (0.545, 0.723 on momentum)
            assert abs(min(got["nux"], 1 - got["nux"]) - 0.455) < 0.06
            assert abs(min(got["nuy"], 1 - got["nuy"]) - 0.277) < 0.06
