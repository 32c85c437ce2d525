"""GPU parity of the CSR step (CSRCSBEND + CSRDRIFT) against elegant's own
track_through_csbendCSR / track_through_driftCSR (oracle/_ref, shared maths):
bit-identical final coordinates and bit-identical per-kick wake arrays."""
import numpy as np
import pytest

from elegant_b200 import Element, Lattice, Tracker, workloads as w
from reforacle import by_id

pytestmark = pytest.mark.gpu
P0 = 1000 / 0.51099895


def run_both(ref, lat, beam):
    with Tracker(lat, P0, 1) as t:
        res = t.track(beam)
        wakes = t.csr_wakes(10_000_000)
    rows, nl, _, ref_wakes = ref.track(lat, beam.coords, beam.ids, P0, 1, capture_wakes=True)
    return res, wakes, rows, nl, ref_wakes


def check(res, wakes, rows, nl, ref_wakes):
    ref_c, ref_ids, ref_loss = by_id(rows)
    order = np.argsort(res.ids)
    assert res.n_left == nl
    assert np.array_equal(res.ids[order], ref_ids)
    assert wakes.shape == ref_wakes.shape and wakes.size > 0
    bad = np.flatnonzero(wakes != ref_wakes)
    assert bad.size == 0, f"{bad.size} wake values differ, first at {bad[:5]}"
    c = res.coords[order]
    alive = ref_loss < 0
    diff = c[alive] != ref_c[alive]
    assert not diff.any(), f"{diff.sum()} coordinates differ, max {np.abs(c[alive] - ref_c[alive]).max()}"


@pytest.mark.parametrize("bins,kicks,sg", [(200, 6, 2), (120, 4, 0), (300, 5, 3)])
def test_chicane_bit_exact(ref_b2e, bins, kicks, sg):
    lat = w.chicane(bins=bins, n_kicks=kicks, sg_halfwidth=sg)
    beam = w.chicane_beam(20000, seed=bins)
    check(*run_both(ref_b2e, lat, beam))


def test_chicane_steady_state_and_plain_sum(ref_b2e):
    lat = w.chicane(bins=150, n_kicks=4)
    els = []
    for i, e in enumerate(lat.elements):
        if e.type == "CSRCSBEND":
            extra = {"STEADY_STATE": 1} if i % 2 else {"TRAPAZOID_INTEGRATION": 0}
            e = Element(e.name, e.type, dict(e.params, **extra))
        els.append(e)
    beam = w.chicane_beam(15000, seed=4)
    check(*run_both(ref_b2e, Lattice(els), beam))


def test_chicane_csrdrift_multiple_kicks(ref_b2e):
    lat = w.chicane(bins=100, n_kicks=3)
    els = [Element(e.name, e.type, dict(e.params, N_KICKS=4)) if e.type == "CSRDRIFT" else e for e in lat.elements]
    beam = w.chicane_beam(8000, seed=9)
    check(*run_both(ref_b2e, Lattice(els), beam))


def test_chicane_without_charge_is_plain_tracking(ref_b2e):
    lat = w.chicane(bins=100, n_kicks=3, charge=0.0)
    beam = w.chicane_beam(5000, seed=2)
    check(*run_both(ref_b2e, lat, beam))
