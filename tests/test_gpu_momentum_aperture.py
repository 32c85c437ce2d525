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
