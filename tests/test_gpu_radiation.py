"""Synchrotron radiation on the device.

SYNCH_RAD is deterministic: the ring with radiating quadrupoles, sextupoles
and dipoles (edges included) equals elegant's own code bit for bit.  ISR
deviates come from the counter-based generator shared with the C
restatement, addressed by particle ID, pass, element, slice and step, so the
device equals the restatement bit for bit and does not depend on how the
particles are launched or compacted (the reference's own serial generator is
compared in distribution on the CPU, tests/test_radiation.py)."""
import numpy as np
import pytest

from elegant_b200 import Element, Lattice, Tracker, workloads as w
from elegant_b200._native import EngineError
from reforacle import PortOracle, by_id

pytestmark = pytest.mark.gpu
P0 = w.ring_p_central()


def _check_equal(res, rows, nl):
    ref_c, ref_ids, ref_loss = by_id(rows)
    order = np.argsort(res.ids)
    assert res.n_left == nl
    assert np.array_equal(res.ids[order], ref_ids)
    alive = ref_loss < 0
    assert np.array_equal(res.lost_pass[order] < 0, alive)
    c = res.coords[order]
    bad = c[alive] != ref_c[alive]
    assert not bad.any(), f"{bad.sum()} coordinates differ, max {np.abs(c[alive] - ref_c[alive]).max()}"


@pytest.mark.parametrize("edge", [0.0, 0.04])
def test_synch_rad_ring_bit_exact(ref_b2e, edge):
    lat = w.radiating_ring(edge_angle=edge)
    beam = w.ring_beam(2000, seed=41)
    with Tracker(lat, P0, 100) as t:
        res = t.track(beam)
    rows, nl, _, _ = ref_b2e.track(lat, beam.coords, beam.ids, P0, 100)
    assert nl > 1500
    _check_equal(res, rows, nl)


def test_isr_matches_the_restatement_bit_for_bit():
    lat = w.radiating_ring(isr=True)
    beam = w.ring_beam(500, seed=42)
    with Tracker(lat, P0, 25, isr_seed=99) as t:
        res = t.track(beam)
    port = PortOracle("b2e")
    port.set_isr(99, 3.0)
    rows, nl, _ = port.track(lat, beam.coords, beam.ids, P0, 25)[:3]
    port.set_isr(0)
    _check_equal(res, rows, nl)


def test_isr_independent_of_launch_shape_and_compaction():
    lat = w.radiating_ring(isr=True)
    beam = w.ring_beam(3000, seed=43)
    out = []
    for kw in ({}, {"passes_per_launch": 3}, {"compact_every": 4}):
        with Tracker(lat, P0, 30, isr_seed=5, **kw) as t:
            r = t.track(beam)
        order = np.argsort(r.ids)
        out.append((r.coords[order], r.lost_pass[order]))
    for c, lp in out[1:]:
        assert np.array_equal(lp, out[0][1])
        alive = lp < 0
        assert np.array_equal(c[alive], out[0][0][alive])
    with Tracker(lat, P0, 30, isr_seed=6) as t:
        r = t.track(beam)
    assert not np.array_equal(r.coords[np.argsort(r.ids)][:, 5], out[0][0][:, 5])


@pytest.mark.parametrize("typ, params", [
    ("KQUAD", {"L": 0.3, "K1": 1.0, "ISR": 1, "ISR1PART": 0}),
    ("CSRCSBEND", {"L": 0.5, "ANGLE": 0.05, "BINS": 100, "SYNCH_RAD": 1}),
])
def test_unsupported_radiation_options_are_rejected(typ, params):
    lat = Lattice([Element("D", "DRIF", {"L": 1.0}), Element("X", typ, params)])
    with pytest.raises(EngineError) as e:
        Tracker(lat, P0, 1)
    assert e.value.code == -2
