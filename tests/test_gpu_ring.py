"""GPU parity of the fused ring kernel against the reference's own tracking
code (oracle/_ref, built with the engine's elementary functions).

Bar: bit-identical final coordinates for every surviving particle and an
identical set of (particle ID, loss pass) for lost ones.
"""
import numpy as np
import pytest

from elegant_b200 import Element, Lattice, Tracker, workloads as w
from elegant_b200.beam import Beam
from reforacle import by_id

pytestmark = pytest.mark.gpu


def gpu_track(lat, beam, p, passes, **kw):
    with Tracker(lat, p, passes, **kw) as t:
        return t.track(beam)


def assert_parity(res, rows, n_left):
    ref_c, ref_ids, ref_loss = by_id(rows)
    order = np.argsort(res.ids)
    c, ids, lp = res.coords[order], res.ids[order], res.lost_pass[order]
    assert np.array_equal(ids, ref_ids)
    assert res.n_left == n_left
    ref_lost = {(int(i), int(l)) for i, l in zip(ref_ids, ref_loss) if l >= 0}
    gpu_lost = {(int(i), int(l)) for i, l in zip(ids, lp) if l >= 0}
    assert gpu_lost == ref_lost
    alive = lp < 0
    diff = c[alive] != ref_c[alive]
    assert not diff.any(), f"{diff.sum()} coordinates differ; max abs {np.abs(c[alive]-ref_c[alive]).max()}"


def test_ring_bit_exact_100_turns(ref_b2e):
    lat = w.fodo_ring()
    beam = w.ring_beam(256, seed=11)
    res = gpu_track(lat, beam, w.ring_p_central(), 100)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 100)
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_bit_exact_1000_turns(ref_b2e):
    """The single-ring workload's 1,000 turns: every survivor coordinate
    bit-identical to the reference's own tracking (shared elementary
    functions) and the same (ID, loss turn) set, on a sample of its beam."""
    lat = w.fodo_ring()
    full = w.ring_beam(10000, seed=12345)
    idx = np.linspace(0, 9999, 160).astype(int)
    beam = Beam(full.coords[idx], full.ids[idx])
    res = gpu_track(lat, beam, w.ring_p_central(), 1000)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 1000)
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_losses_match(ref_b2e):
    """Large-amplitude and off-momentum particles hit the 20 mm aperture,
    the slope limit and the sextupole dynamic aperture."""
    lat = w.fodo_ring()
    rng = np.random.default_rng(3)
    n = 300
    c = np.zeros((n, 6))
    c[:, 0] = rng.uniform(-0.022, 0.022, n)
    c[:, 1] = rng.uniform(-3e-3, 3e-3, n)
    c[:, 2] = rng.uniform(-0.015, 0.015, n)
    c[:, 3] = rng.uniform(-2e-3, 2e-3, n)
    c[:, 4] = rng.normal(0, 5e-3, n)
    c[:, 5] = rng.uniform(-0.03, 0.03, n)
    beam = Beam(c, np.arange(1, n + 1))
    res = gpu_track(lat, beam, w.ring_p_central(), 40)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 40)
    assert nl < n, "test beam should lose particles"
    assert_parity(res, rows, nl)


@pytest.mark.parametrize("exponents", [(2, 2), (4, 6), (8, 2), (10, 4)])
def test_ring_aperture_around_quarter_axes(ref_b2e, exponents):
    """Particles at, just inside and just outside a quarter of the half-axes
    (where the aperture tests stop dividing) and near the edge, for
    elliptical and super-elliptical MAXAMP apertures."""
    xe, ye = exponents
    els = [Element(e.name, e.type, dict(e.params, EXPONENT=xe, YEXPONENT=ye)) if e.type == "MAXAMP" else e
           for e in w.fodo_ring().elements]
    lat = Lattice(els)
    q = 0.25 * 0.02
    edge = [q, np.nextafter(q, 1), np.nextafter(q, 0), 0.0195, 0.02, 0.0201]
    rng = np.random.default_rng(11)
    rows = [(sx * a, sy * b) for a in edge for b in edge for sx in (1, -1) for sy in (1, -1)]
    rows += [tuple(v) for v in rng.uniform(-0.021, 0.021, (200, 2))]
    n = len(rows)
    c = np.zeros((n, 6))
    c[:, 0] = [r[0] for r in rows]
    c[:, 2] = [r[1] for r in rows]
    c[:, 1] = rng.uniform(-2e-4, 2e-4, n)
    c[:, 3] = rng.uniform(-2e-4, 2e-4, n)
    beam = Beam(c, np.arange(1, n + 1))
    res = gpu_track(lat, beam, w.ring_p_central(), 5)
    ref_rows, nl, _, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 5)
    assert 0 < nl < n
    assert_parity(res, ref_rows, nl)


def test_ring_misaligned_and_tilted(ref_b2e):
    lat = w.fodo_ring()
    els = []
    for i, e in enumerate(lat.elements):
        if e.type == "KQUAD":
            e = Element(e.name, e.type, dict(e.params, DX=3e-4 * ((i % 3) - 1), DY=-2e-4, FSE=1e-3 * (i % 2)))
        if e.type == "KSEXT" and i % 3 == 0:
            e = Element(e.name, e.type, dict(e.params, TILT=0.01, DX=1e-4))
        els.append(e)
    lat2 = Lattice(els)
    beam = w.ring_beam(128, seed=4)
    res = gpu_track(lat2, beam, w.ring_p_central(), 30)
    rows, nl, _, _ = ref_b2e.track(lat2, beam.coords, beam.ids, w.ring_p_central(), 30)
    assert_parity(res, rows, nl)


def test_continuation_equals_single_run():
    lat = w.fodo_ring()
    beam = w.ring_beam(200, seed=9)
    one = gpu_track(lat, beam, w.ring_p_central(), 60)
    with Tracker(lat, w.ring_p_central(), 30) as t:
        t.track(beam)  # uploads and tracks passes 0..29
        eff2 = t.continue_tracking()
        two = t.download()
    assert np.array_equal(one.coords, two.coords)
    assert np.array_equal(one.lost_pass, two.lost_pass)


def test_passes_per_launch_invariance():
    lat = w.fodo_ring()
    beam = w.ring_beam(200, seed=2)
    a = gpu_track(lat, beam, w.ring_p_central(), 25)
    b = gpu_track(lat, beam, w.ring_p_central(), 25, passes_per_launch=4)
    assert np.array_equal(a.coords, b.coords)
    assert np.array_equal(a.lost_pass, b.lost_pass)


def test_empty_and_single_particle(ref_b2e):
    lat = w.fodo_ring()
    empty = Beam(np.zeros((0, 6)), np.zeros(0, dtype=np.int64))
    res = gpu_track(lat, empty, w.ring_p_central(), 3)
    assert res.n_left == 0 and res.effort == 0
    one = w.ring_beam(1, seed=1)
    res = gpu_track(lat, one, w.ring_p_central(), 20)
    rows, nl, _, _ = ref_b2e.track(lat, one.coords, one.ids, w.ring_p_central(), 20)
    assert_parity(res, rows, nl)


def test_ensemble_matches_per_instance_reference(ref_b2e):
    lat, beam, offsets, overrides = w.ensemble(n_instances=6, n_min=40, n_max=90, seed=5)
    with Tracker(lat, w.ring_p_central(), 15) as t:
        t.load_ensemble(offsets, overrides)
        res = t.track(beam)
    for i in range(6):
        sl = slice(offsets[i], offsets[i + 1])
        els = []
        for j, e in enumerate(lat.elements):
            params = dict(e.params)
            for (ie, name, vals) in overrides:
                if ie == j:
                    params[name] = float(vals[i])
            els.append(Element(e.name, e.type, params))
        rows, nl, _, _ = ref_b2e.track(Lattice(els), beam.coords[sl], beam.ids[sl], w.ring_p_central(), 15)
        sub = type(res)(res.coords[sl], res.ids[sl], res.lost_pass[sl], res.lost_element[sl],
                        int((res.lost_pass[sl] < 0).sum()), 0.0)
        assert_parity(sub, rows, nl)


def _lossy_beam(n, seed):
    rng = np.random.default_rng(seed)
    c = np.zeros((n, 6))
    c[:, 0] = rng.uniform(-0.022, 0.022, n)
    c[:, 1] = rng.uniform(-3e-3, 3e-3, n)
    c[:, 2] = rng.uniform(-0.015, 0.015, n)
    c[:, 3] = rng.uniform(-2e-3, 2e-3, n)
    c[:, 4] = rng.normal(0, 5e-3, n)
    c[:, 5] = rng.uniform(-0.03, 0.03, n)
    return Beam(c, np.arange(1, n + 1))


@pytest.mark.parametrize("history", [False, True])
def test_kernel_variants_identical(history):
    """Every variant the autotuner may pick (occupancy target x warp barrier
    level) gives identical coordinates and losses, with and without history."""
    lat = w.fodo_ring()
    beam = _lossy_beam(700, seed=21)
    ref = gpu_track(lat, beam, w.ring_p_central(), 12, ring_variant=1)
    assert (ref.lost_pass >= 0).any() and (ref.lost_pass < 0).any()
    for v in range(1, 18):
        r = gpu_track(lat, beam, w.ring_p_central(), 12, ring_variant=v, record_history=history)
        assert np.array_equal(r.coords, ref.coords), v
        assert np.array_equal(r.lost_pass, ref.lost_pass), v
        assert np.array_equal(r.lost_element, ref.lost_element), v


def test_autotuner_picks_a_variant():
    lat = w.fodo_ring()
    beam = w.ring_beam(20000, seed=8)
    with Tracker(lat, w.ring_p_central(), 3) as t:
        t.track(beam)
        chosen, ms = t.ring_tuning()
    assert 1 <= chosen <= 17
    assert len(ms) == 17 and all(m > 0 for m in ms)


def _moments(coords, alive):
    """Survivors, centroids and rms emittances as rms_emittance
    (final_props.c:844-880) forms them: sqrt(<dx^2><dx'^2> - <dx dx'>^2)."""
    c = coords[alive]
    n = len(c)
    if n == 0:
        return n, 0.0, 0.0, 0.0, 0.0
    m = c[:, :4].mean(axis=0)
    d = c[:, :4] - m
    ex = np.sqrt(max((d[:, 0] ** 2).mean() * (d[:, 1] ** 2).mean() - (d[:, 0] * d[:, 1]).mean() ** 2, 0.0))
    ey = np.sqrt(max((d[:, 2] ** 2).mean() * (d[:, 3] ** 2).mean() - (d[:, 2] * d[:, 3]).mean() ** 2, 0.0))
    return n, m[0], m[2], ex, ey


def test_ensemble_history_matches_per_pass_moments():
    """The per-pass history equals the moments of the coordinates downloaded
    after each pass, per instance; recording it leaves the tracking unchanged."""
    lat, beam, offsets, overrides = w.ensemble(n_instances=5, n_min=150, n_max=400, seed=9)
    # instance 2 gets a large-amplitude beam so that it loses particles
    lossy = _lossy_beam(int(offsets[3] - offsets[2]), seed=4)
    beam.coords[offsets[2]:offsets[3]] = lossy.coords
    passes = 6
    with Tracker(lat, w.ring_p_central(), passes, record_history=True) as t:
        t.load_ensemble(offsets, overrides)
        res = t.track(beam)
        hist = t.history()
    assert hist["ex"].shape == (5, passes)
    with Tracker(lat, w.ring_p_central(), passes) as t:
        t.load_ensemble(offsets, overrides)
        plain = t.track(beam)
    assert np.array_equal(res.coords, plain.coords)
    assert np.array_equal(res.lost_pass, plain.lost_pass)

    with Tracker(lat, w.ring_p_central(), 1, record_history=True) as t:
        t.load_ensemble(offsets, overrides)
        t.upload(beam)
        expected = np.zeros((5, passes, 5))
        for j in range(passes):
            t.continue_tracking()
            r = t.download()
            order = np.argsort(r.ids)
            coords, lost = r.coords[order], r.lost_pass[order]
            for i in range(5):
                sl = slice(offsets[i], offsets[i + 1])
                expected[i, j] = _moments(coords[sl], lost[sl] < 0)
        stepped = t.history()
    assert (expected[2, :, 0] < expected[2, 0, 0]).any() or expected[2, 0, 0] < offsets[3] - offsets[2]
    for h in (hist, stepped):
        assert np.array_equal(h["survivors"], expected[:, :, 0].astype(np.int64))
        for k, col in (("cx", 1), ("cy", 2), ("ex", 3), ("ey", 4)):
            np.testing.assert_allclose(h[k], expected[:, :, col], rtol=1e-10, atol=1e-18)
    assert np.array_equal(stepped["ex"], hist["ex"])


@pytest.mark.parametrize("ensemble", [False, True])
def test_compaction_gives_the_same_particles(ensemble):
    """Moving each instance's survivors to the front every few passes (rows
    reordered, launches over survivors only) changes no particle's result."""
    if ensemble:
        lat, beam, offsets, overrides = w.ensemble(n_instances=4, n_min=200, n_max=500, seed=12)
        lossy = _lossy_beam(int(offsets[2] - offsets[1]), seed=6)
        beam.coords[offsets[1]:offsets[2]] = lossy.coords
    else:
        lat, beam = w.fodo_ring(), _lossy_beam(900, seed=17)

    def run(**kw):
        with Tracker(lat, w.ring_p_central(), 30, **kw) as t:
            if ensemble:
                t.load_ensemble(offsets, overrides)
            return t.track(beam)

    plain, comp = run(), run(compact_every=3)
    assert (plain.lost_pass >= 0).sum() > 50
    assert comp.effort == plain.effort and comp.n_left == plain.n_left
    o1, o2 = np.argsort(plain.ids), np.argsort(comp.ids)
    assert np.array_equal(plain.ids[o1], comp.ids[o2])
    assert np.array_equal(plain.lost_pass[o1], comp.lost_pass[o2])
    assert np.array_equal(plain.lost_element[o1], comp.lost_element[o2])
    alive = plain.lost_pass[o1] < 0
    assert np.array_equal(plain.coords[o1][alive], comp.coords[o2][alive])
    if ensemble:  # every particle stays inside its own instance's range
        for i in range(4):
            sl = slice(offsets[i], offsets[i + 1])
            assert set(comp.ids[sl]) == set(beam.ids[sl])


def test_non_finite_inputs_are_lost_like_the_reference(ref_b2e):
    """NaN and infinite starting coordinates: the same particles lost at the
    same turn as in the reference, the rest untouched."""
    lat = w.fodo_ring()
    beam = w.ring_beam(64, seed=3)
    c = beam.coords.copy()
    c[3, 0] = np.nan
    c[10, 1] = np.inf
    c[17, 2] = -np.inf
    c[25, 5] = np.nan
    c[40, 4] = np.nan
    b = Beam(c, beam.ids)
    res = gpu_track(lat, b, w.ring_p_central(), 5)
    rows, nl, eff, _ = ref_b2e.track(lat, b.coords, b.ids, w.ring_p_central(), 5)
    assert_parity(res, rows, nl)


def test_ragged_ensemble_with_an_empty_instance(ref_b2e):
    lat, beam, offsets, overrides = w.ensemble(n_instances=4, n_min=3, n_max=140, seed=8)
    sizes = np.diff(offsets)
    sizes[1] = 0
    keep = np.concatenate([np.arange(offsets[i], offsets[i] + sizes[i]) for i in range(4)]).astype(int)
    beam = Beam(beam.coords[keep], beam.ids[keep])
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    with Tracker(lat, w.ring_p_central(), 8) as t:
        t.load_ensemble(offsets, overrides)
        res = t.track(beam)
    for i in (0, 2, 3):
        sl = slice(offsets[i], offsets[i + 1])
        els = []
        for j, e in enumerate(lat.elements):
            params = dict(e.params)
            for (ie, name, vals) in overrides:
                if ie == j:
                    params[name] = float(vals[i])
            els.append(Element(e.name, e.type, params))
        rows, nl, _, _ = ref_b2e.track(Lattice(els), beam.coords[sl], beam.ids[sl], w.ring_p_central(), 8)
        sub = type(res)(res.coords[sl], res.ids[sl], res.lost_pass[sl], res.lost_element[sl],
                        int((res.lost_pass[sl] < 0).sum()), 0.0)
        assert_parity(sub, rows, nl)


def test_lattice_too_large_for_shared_memory(ref_b2e):
    """650 elements do not fit the shared-memory staging: the kernel reads the
    element records from global memory, with the same results."""
    cell = [e for e in w.fodo_ring().elements]
    lat = Lattice([Element(f"{e.name}_{k}", e.type, dict(e.params)) for k in range(10) for e in cell])
    assert len(lat) > 600
    beam = w.ring_beam(48, seed=5)
    res = gpu_track(lat, beam, w.ring_p_central(), 2)
    rows, nl, _, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 2)
    assert_parity(res, rows, nl)


def test_ring_with_exact_drifts(ref_b2e):
    """EDRIFT (exactDrift, csbend.c:3767-3790) in place of the second drift of
    every cell, with losses: bit-identical to the reference."""
    els = [Element(e.name, "EDRIFT", {"L": e.params["L"]}) if e.name == "D2" else e for e in w.fodo_ring().elements]
    lat = Lattice(els)
    assert sum(e.type == "EDRIFT" for e in lat.elements) == 8
    beam = Beam(np.concatenate([w.ring_beam(200, seed=6).coords, _lossy_beam(200, seed=8).coords]),
                np.arange(1, 401))
    res = gpu_track(lat, beam, w.ring_p_central(), 60)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 60)
    assert 200 <= nl < 400
    assert_parity(res, rows, nl)
    assert res.effort == eff


@pytest.mark.parametrize("rf", [{"L": 0.5, "N_KICKS": 0}, {"L": 0.5, "N_KICKS": 5}, {"VOLT": 0.0},
                                {"L": 0.4, "VOLT": 0.0}], ids=["matrix", "kicks", "no_volt", "no_volt_drift"])
def test_ring_rf_cavity_with_length(ref_b2e, rf):
    """RFCA with a length by the matrix method and by drift-kick-drift
    sections, and at zero voltage, bit-identical to the reference over 60
    turns with losses."""
    els = [Element(e.name, e.type, dict(e.params, **rf)) if e.type == "RFCA" else e for e in w.fodo_ring().elements]
    lat = Lattice(els)
    beam = Beam(np.concatenate([w.ring_beam(150, seed=31).coords, _lossy_beam(150, seed=32).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 60)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 60)
    assert 150 <= nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_with_rolled_dipoles(ref_b2e):
    """CSBEND ETILT (exit-face offsets, csbend.c:4723-4769 and :1359-1364)
    alone, with TILT and a misalignment, with edge angles, with DZ; 60 turns
    with losses, bit-identical to the reference."""
    errs = [{"ETILT": 2e-3}, {"ETILT": -1.5e-3, "TILT": 0.05, "DX": 1e-4},
            {"ETILT": 1e-3, "E1": 0.1, "E2": 0.08}, {"ETILT": 5e-4, "DZ": 2e-4}]
    els, k = [], 0
    for e in w.fodo_ring().elements:
        if e.type == "CSBEND":
            e = Element(e.name + str(k), e.type, dict(e.params, **errs[k % len(errs)]))
            k += 1
        els.append(e)
    lat = Lattice(els)
    beam = Beam(np.concatenate([w.ring_beam(150, seed=33).coords, _lossy_beam(150, seed=34).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 60)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 60)
    assert 100 <= nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_with_second_order_edges(ref_b2e):
    """EDGE_ORDER=2 on every dipole, with edge angles and a fringe integral:
    60 turns with losses, bit-identical to the reference."""
    els, k = [], 0
    for e in w.fodo_ring().elements:
        if e.type == "CSBEND":
            e = Element(e.name + str(k), e.type, dict(e.params, EDGE_ORDER=2, E1=0.12 - 0.05 * (k % 3),
                                                      E2=0.09 * (k % 2), HGAP=0.02, FINT=0.5))
            k += 1
        els.append(e)
    lat = Lattice(els)
    beam = Beam(np.concatenate([w.ring_beam(150, seed=35).coords, _lossy_beam(150, seed=36).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 60)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 60)
    assert 100 <= nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


@pytest.mark.parametrize("case", ["plain", "negative_angle", "synch_rad"])
def test_ring_with_gradient_dipoles(ref_b2e, case):
    """CSBEND with K1/K2 field terms (the expansion of csbend.c:186-663, the
    field sums :101-150 in the kick and, with SYNCH_RAD, in the radiation and
    edge corrections), NONLINEAR=0 on some, second-order edges on some,
    negative angles: 60 turns with losses, bit-identical to the reference."""
    import math
    errs = [{"K1": 0.15, "K2": 2.0}, {"K1": -0.2, "NONLINEAR": 0}, {"K2": -3.0, "EDGE_ORDER": 2, "E1": 0.1},
            {"K1": 0.1, "K2": 1.0, "FSE": 1e-3}]
    base = w.radiating_ring(edge_angle=0.05) if case == "synch_rad" else w.fodo_ring()
    els, k = [], 0
    for e in base.elements:
        if e.type == "CSBEND":
            params = dict(e.params, **errs[k % len(errs)])
            if case == "negative_angle" and k % 2:
                params.update(ANGLE=-params["ANGLE"], TILT=math.pi)
            e = Element(e.name + str(k), e.type, params)
            k += 1
        els.append(e)
    lat = Lattice(els)
    beam = Beam(np.concatenate([w.ring_beam(150, seed=51).coords, _lossy_beam(150, seed=52).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 60)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 60)
    assert 0 < nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


@pytest.mark.parametrize("kw", [{}, {"compact_every": 2}, {"passes_per_launch": 3}],
                         ids=["fused", "compacted", "split_launches"])
def test_watch_records_equal_the_reference(ref_b2e, kw):
    """WATCH elements (coordinate mode): on the passes each writes
    (START_PASS, INTERVAL, END_PASS), the particles alive at it and their
    coordinates equal what the reference hands dump_watch_particles, bit for
    bit; the tracking itself is unchanged by them.  With compaction the rows
    move between launches and the records follow the IDs."""
    from test_oracle_pin import _ring_with_watches
    lat = _ring_with_watches()
    beam = Beam(np.concatenate([w.ring_beam(300, seed=55).coords, _lossy_beam(300, seed=56).coords]),
                np.arange(1, 601))
    ref_b2e.set_watch(2_000_000)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 12)
    ref_rows = ref_b2e.watch_rows()
    ref_b2e.set_watch(0)
    with Tracker(lat, w.ring_p_central(), 12, **kw) as t:
        t.set_watch(1 << 30)
        res = t.track(beam)
        recs = t.watch()
    assert_parity(res, rows, nl)
    w1, w2 = lat.index("W1")[0], lat.index("W2")[0]
    assert [(r["element"], r["pass"]) for r in recs] == [(w1, q) for q in (1, 4, 7, 10)] + [(w2, q) for q in range(5)]
    for r in recs:
        sel = ref_rows[(ref_rows[:, 0] == r["element"]) & (ref_rows[:, 1] == r["pass"])]
        sel = sel[np.argsort(sel[:, 2], kind="stable")]
        assert np.array_equal(r["ids"], sel[:, 2].astype(np.int64)), (r["element"], r["pass"])
        assert np.array_equal(r["coords"], sel[:, 3:9]), (r["element"], r["pass"])


def test_watch_budget_is_enforced():
    from elegant_b200._native import EngineError
    from test_oracle_pin import _ring_with_watches
    beam = w.ring_beam(1000, seed=57)
    with Tracker(_ring_with_watches(), w.ring_p_central(), 12) as t:
        t.set_watch(1000)
        with pytest.raises(EngineError, match="WATCH"):
            t.track(beam)


@pytest.mark.parametrize("case", ["plain", "synch_rad"])
def test_ring_with_steering(ref_b2e, case):
    """KQUAD/KSEXT correctors (HKICK, VKICK, calibrations; multipole.c:785-786,
    :1190-1191, :1281-1284), a pole-tip strength from BORE and B (:771-773,
    :834-837), and with SYNCH_RAD the steering kicks in F2 (:1333): 60 turns
    with losses, bit-identical to the reference."""
    from test_oracle_pin import _ring_with_steering
    base = None
    if case == "synch_rad":
        base = Lattice([Element(e.name, e.type, dict(e.params, SYNCH_RAD=1)) if e.type in ("KQUAD", "KSEXT") else e
                        for e in w.fodo_ring().elements])
    lat = _ring_with_steering(base)
    beam = Beam(np.concatenate([w.ring_beam(150, seed=61).coords, _lossy_beam(150, seed=62).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 60)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 60)
    assert 0 < nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ensemble_of_corrector_settings(ref_b2e):
    """Per-instance HKICK/VKICK overrides (an ensemble of orbit-corrector
    settings): each instance equal to the reference run with its settings."""
    lat = w.fodo_ring()
    quads = [i for i, e in enumerate(lat.elements) if e.type == "KQUAD"]
    n_inst = 5
    rng = np.random.default_rng(17)
    overrides = []
    for i in quads[:6]:
        overrides.append((i, "HKICK", rng.normal(0, 1e-4, n_inst)))
        overrides.append((i, "VKICK", rng.normal(0, 1e-4, n_inst)))
    overrides[0][2][0] = 0.0  # an instance without that corrector
    counts = [40, 64, 90, 33, 128]
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    beam = Beam(_lossy_beam(int(offsets[-1]), seed=63).coords * 0.5, np.arange(1, int(offsets[-1]) + 1))
    with Tracker(lat, w.ring_p_central(), 15) as t:
        t.load_ensemble(offsets, overrides)
        res = t.track(beam)
    for k in range(n_inst):
        sl = slice(offsets[k], offsets[k + 1])
        els = []
        for j, e in enumerate(lat.elements):
            params = dict(e.params)
            for (ie, name, vals) in overrides:
                if ie == j:
                    params[name] = float(vals[k])
            els.append(Element(e.name, e.type, params))
        rows, nl, _, _ = ref_b2e.track(Lattice(els), beam.coords[sl], beam.ids[sl], w.ring_p_central(), 15)
        sub = type(res)(res.coords[sl], res.ids[sl], res.lost_pass[sl], res.lost_element[sl],
                        int((res.lost_pass[sl] < 0).sum()), 0.0)
        assert_parity(sub, rows, nl)


@pytest.mark.parametrize("mode", ["light", "pmaximum"])
def test_ring_fiducial_modes(ref_b2e, mode):
    """RFCA FIDUCIAL light and pmaximum (findFiducialTime, simple_rfca.c:97-147)
    on a zero-length cavity mid-ring and one with a length: 40 turns with
    losses, bit-identical to the reference; and as per-instance ensembles."""
    base = list(w.fodo_ring().elements)
    rf = next(e for e in base if e.type == "RFCA")
    els = [e for e in base if e.type != "RFCA"]
    els.insert(20, Element("RF1", "RFCA", dict(rf.params, FIDUCIAL=mode)))
    els.append(Element("RF2", "RFCA", dict(rf.params, L=0.4, N_KICKS=4, VOLT=5e5, FIDUCIAL=mode)))
    lat = Lattice(els)
    beam = Beam(np.concatenate([w.ring_beam(150, seed=71).coords, _lossy_beam(150, seed=72).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 40)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 40)
    assert 0 < nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_fiducial_pmaximum_without_a_particle_is_an_error():
    """A beam whose first particle has the highest delta leaves pmaximum no
    fiducial particle: the reference stops; the engine returns an error."""
    from elegant_b200._native import EngineError
    lat = Lattice([Element("D", "DRIF", {"L": 1.0}),
                   Element("RF", "RFCA", {"VOLT": 1e6, "FREQ": 5e8, "FIDUCIAL": "pmaximum"})])
    coords = np.zeros((3, 6))
    coords[:, 5] = [1e-3, 0.0, -1e-3]
    with pytest.raises(EngineError, match="No available particle"):
        gpu_track(lat, Beam(coords, np.arange(1, 4)), w.ring_p_central(), 2)


@pytest.mark.parametrize("negative", [False, True])
def test_ring_with_bend_steering(ref_b2e, negative):
    """CSBEND XKICK and YKICK (the expansion's b0 = XKICK/ANGLE and c0 =
    YKICK/ANGLE, csbend.c:867-868, in the field sums of the kick), alone and
    with K1/K2, with negative angles: 30 turns with losses, bit-identical to
    the reference."""
    from test_oracle_pin import _ring_with_bend_steering
    lat = _ring_with_bend_steering(negative)
    beam = Beam(np.concatenate([w.ring_beam(150, seed=81).coords, _lossy_beam(150, seed=82).coords]),
                np.arange(1, 301))
    # 30 turns: the uncorrected vertical kicks drive every particle out by turn 40
    res = gpu_track(lat, beam, w.ring_p_central(), 30)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 30)
    assert 0 < nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_with_quad_fringes(ref_b2e):
    """KQUAD fringe fields (quadFringe, fringe.c:24-175, at multipole.c:1031-1037
    and :1088-1094): linear and third-order, with and without the linear
    part, a nonlinear factor, misaligned, one face only: 60 turns with
    losses, bit-identical to the reference (elegant's fringe.c compiled in)."""
    from test_oracle_pin import _ring_with_quad_fringes
    lat = _ring_with_quad_fringes()
    beam = Beam(np.concatenate([w.ring_beam(150, seed=91).coords, _lossy_beam(150, seed=92).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 60)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 60)
    assert 0 < nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_with_linked_cavities(ref_b2e):
    """RFCA PHASE_REFERENCE groups (simple_rfca.c:410-470): later cavities of
    a group take the first one's fiducial phase; 40 turns with losses,
    bit-identical to the reference, and per-instance ensembles alike."""
    from test_oracle_pin import _ring_with_linked_cavities
    lat = _ring_with_linked_cavities()
    beam = Beam(np.concatenate([w.ring_beam(150, seed=101).coords, _lossy_beam(150, seed=102).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 40)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 40)
    assert 0 < nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff


def test_ring_with_simple_edges(ref_b2e):
    """CSBEND EDGE_EFFECTS 3 (applySimpleDipoleEdgeKick, csbend.c:5639-5665):
    40 turns with losses, bit-identical to the reference."""
    from test_oracle_pin import _ring_with_simple_edges
    lat = _ring_with_simple_edges()
    beam = Beam(np.concatenate([w.ring_beam(150, seed=111).coords, _lossy_beam(150, seed=112).coords]),
                np.arange(1, 301))
    res = gpu_track(lat, beam, w.ring_p_central(), 40)
    rows, nl, eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, w.ring_p_central(), 40)
    assert 0 < nl < 300
    assert_parity(res, rows, nl)
    assert res.effort == eff
