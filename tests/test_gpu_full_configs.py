"""Parity at the full sizes of the benchmark cases, against elegant's own
tracking code run on the same inputs (tests/golden/make_full_configs.py ran
oracle/_ref and stored digests, the glibc ring coordinates and the per-pass
ensemble history).

- ring: 10,000 particles x 1,000 turns: survivors bit-identical to the
  reference with the shared elementary functions; against the reference
  with glibc's, every coordinate inside the ring's own one-ulp sensitivity
  envelope and the identical (ID, loss pass) set.
- edge: 2,000 particles around the ring's dynamic aperture x 1,000 turns:
  the loss set equal to both references'.
- chicane: 1,000,000 particles, BINS=600, 80 dipole kicks: coordinates and
  every per-kick wake array bit-identical.
- ensemble: 32 full-size instances x 1,000 turns: every instance's survivors
  and losses bit-identical, the per-pass history equal to the moments of the
  reference's own particles.
- train: bunches of 0.5 M and 4 M particles tracked together, each
  bit-identical (coordinates and wakes) to the reference's run of that bunch.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_full_configs as fc  # noqa: E402

from elegant_b200 import Tracker, workloads as w  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fixture():
    return fc.load_fixture()


def _lost(res):
    return fc.lost_pairs(res.ids, res.lost_pass)


def test_full_ring_1000_turns(fixture):
    g = fixture["ring"]
    lat, beam = fc.ring_inputs(fc.twiss_from(g["twiss"]))
    assert fc.digest_beam(beam.coords, beam.ids) == g["input"], "input beam differs from the fixture's"
    with Tracker(lat, w.ring_p_central(), g["turns"]) as t:
        res = t.track(beam)
    # shared elementary functions: bit for bit
    assert res.n_left == g["b2e"]["n_left"] and res.effort == g["b2e"]["effort"]
    assert _lost(res) == g["b2e"]["lost"]
    assert fc.digest_survivors(res.coords, res.ids, res.lost_pass) == g["b2e"]["survivors"]
    # glibc's elementary functions: the same losses, coordinates inside the
    # growth of a one-ulp change of x under the reference itself
    ref = np.load(fc.RING_LIBM)
    assert _lost(res) == g["libm"]["lost"]
    order = np.argsort(res.ids)
    assert np.array_equal(res.ids[order], ref["ids"])
    alive = (res.lost_pass[order] < 0) & (ref["lost_pass"] < 0)
    diff = fc._rel(ref["coords"][alive], res.coords[order][alive])
    envelope = np.asarray(g["libm"]["envelope"])
    assert (diff <= 20 * envelope + 1e-15).all(), (diff, envelope)


def test_ring_dynamic_aperture_edge_1000_turns(fixture):
    """2,000 particles around the dynamic-aperture boundary, 1,000 turns:
    losses spread over the whole run; the (ID, loss pass) set equals both the
    shared-maths and the glibc reference's (which here agree with each other
    and with glibc after a one-ulp change of x), survivors bit-identical to
    the shared-maths reference."""
    g = fixture["edge"]
    lat, beam = fc.edge_inputs()
    assert fc.digest_beam(beam.coords, beam.ids) == g["input"]
    with Tracker(lat, w.ring_p_central(), g["turns"]) as t:
        res = t.track(beam)
    lost = _lost(res)
    assert len(lost) > 1000 and sum(p > 100 for _, p in lost) > 50
    ref = np.load(fc.EDGE_LOSSES)
    assert lost == ref["b2e"].tolist() == ref["libm"].tolist()
    assert fc.digest_lost(res.ids, res.lost_pass) == g["b2e"]["lost"] == g["libm"]["lost"]
    assert res.n_left == g["b2e"]["n_left"] and res.effort == g["b2e"]["effort"]
    assert fc.digest_survivors(res.coords, res.ids, res.lost_pass) == g["b2e"]["survivors"]


def test_full_chicane_1m_particles(fixture):
    g = fixture["chicane"]
    lat, beam = fc.chicane_inputs()
    assert fc.digest_beam(beam.coords, beam.ids) == g["input"]
    with Tracker(lat, fc.CHICANE_P0, 1) as t:
        res = t.track(beam)
        wakes = t.csr_wakes(g["kicks"] * g["bins"] + 1)
    assert res.n_left == g["n_left"] and _lost(res) == g["lost"]
    wk = wakes.reshape(-1, g["bins"])
    assert wk.shape[0] == g["kicks"]
    bad = [k for k in range(g["kicks"]) if fc.digest_array(wk[k]) != g["wakes"][k]]
    assert not bad, f"wake arrays of kicks {bad[:10]} differ"
    assert fc.digest_survivors(res.coords, res.ids, res.lost_pass) == g["survivors"]


def test_full_ensemble_32_instances_1000_turns(fixture):
    g = fixture["ensemble"]
    lat, beam, offsets, overrides = fc.ensemble_inputs(fc.twiss_from(fixture["ring"]["twiss"]))
    assert fc.digest_beam(beam.coords, beam.ids) == g["input"]
    assert [int(x) for x in offsets] == g["offsets"]
    with Tracker(lat, w.ring_p_central(), fc.RING_TURNS, record_history=True) as t:
        t.load_ensemble(offsets, overrides)
        res = t.track(beam)
        hist = t.history()
    for i, gi in enumerate(g["instances"]):
        sl = slice(offsets[i], offsets[i + 1])
        c, ids, lp = res.coords[sl], res.ids[sl], res.lost_pass[sl]
        assert int((lp < 0).sum()) == gi["n_left"], i
        assert fc.digest_lost(ids, lp) == gi["lost"], i
        assert fc.digest_survivors(c, ids, lp) == gi["survivors"], i
    h = np.load(fc.ENSEMBLE_HISTORY)
    assert np.array_equal(hist["survivors"], h["survivors"])
    keep, ref = h["passes"], h["moments"]  # ref: [instance][kept pass][cx, cy, ex, ey]
    for k, key in enumerate(("cx", "cy", "ex", "ey")):
        np.testing.assert_allclose(hist[key][:, keep], ref[:, :, k], rtol=1e-10, atol=1e-18, err_msg=key)


def test_full_train_half_and_four_million(fixture):
    g = fixture["train"]
    lat, beam, offsets = fc.train_inputs()
    assert fc.digest_beam(beam.coords, beam.ids) == g["input"]
    with Tracker(lat, fc.CHICANE_P0, 1) as t:
        t.load_ensemble(offsets, [])
        res = t.track(beam)
        wakes = t.csr_wakes(80 * 2 * 600 + 1)
    nb = len(offsets) - 1
    wk = wakes.reshape(-1, nb, 600)
    for b, gb in enumerate(g["bunches"]):
        sl = slice(offsets[b], offsets[b + 1])
        c, ids, lp = res.coords[sl], res.ids[sl], res.lost_pass[sl]
        assert int((lp < 0).sum()) == gb["n_left"], b
        assert fc.lost_pairs(ids, lp) == gb["lost"], b
        bad = [k for k in range(wk.shape[0]) if fc.digest_array(wk[k, b]) != gb["wakes"][k]]
        assert not bad and wk.shape[0] == len(gb["wakes"]), (b, bad[:10])
        assert fc.digest_survivors(c, ids, lp) == gb["survivors"], b
