"""GPU parity of the CSR step (CSRCSBEND + CSRDRIFT) against elegant's own
track_through_csbendCSR / track_through_driftCSR (oracle/_ref, shared maths):
bit-identical final coordinates and bit-identical per-kick wake arrays."""
import numpy as np
import pytest

from elegant_b200 import Beam, Element, Lattice, Tracker, workloads as w
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


def test_chicane_beam_stored_in_ct_order(ref_b2e):
    """Rows sorted by c*t: neighbouring particles share histogram bins, which
    takes the binning's per-warp aggregation path."""
    lat = w.chicane(bins=80, n_kicks=4)
    beam = w.chicane_beam(20000, seed=21)
    order = np.argsort(beam.coords[:, 4], kind="stable")
    check(*run_both(ref_b2e, lat, Beam(beam.coords[order], beam.ids[order])))


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


def test_chicane_with_exact_drifts(ref_b2e):
    """EDRIFT before the first dipole, between a CSRDRIFT and the next dipole
    and after the last one (exactDrift, csbend.c:3767-3790)."""
    lat = w.chicane(bins=150, n_kicks=5)
    els = []
    for e in lat.elements:
        if e.name == "B1":
            els.append(Element("E0", "EDRIFT", {"L": 0.3}))
        if e.name == "B2":
            els.append(Element("E1", "EDRIFT", {"L": 0.2}))
        els.append(e)
    els.append(Element("E2", "EDRIFT", {"L": 1.0}))
    beam = w.chicane_beam(12000, seed=19)
    check(*run_both(ref_b2e, Lattice(els), beam))


def test_chicane_with_rolled_dipoles(ref_b2e):
    """ETILT on every CSRCSBEND (two with a TILT as well): the exit-face
    offsets (csbend.c:2942-2952), wakes and coordinates bit-identical."""
    lat = w.chicane(bins=150, n_kicks=5)
    lat = Lattice([Element(e.name, e.type, dict(e.params, ETILT=1e-3 * (1 + i % 3), TILT=0.02 * (i % 2)))
                   if e.type == "CSRCSBEND" else e for i, e in enumerate(lat.elements)])
    beam = w.chicane_beam(15000, seed=29)
    check(*run_both(ref_b2e, lat, beam))


def test_chicane_with_second_order_edges(ref_b2e):
    """EDGE_ORDER=2 (apply_edge_effects, csbend.c:4266-4307) at the CSR
    dipoles' entrance and exit, with edge angles and a fringe integral."""
    lat = w.chicane(bins=150, n_kicks=5)
    lat = Lattice([Element(e.name, e.type, dict(e.params, EDGE_ORDER=2, E1=0.02, E2=0.03, HGAP=0.01, FINT=0.4))
                   if e.type == "CSRCSBEND" else e for e in lat.elements])
    beam = w.chicane_beam(15000, seed=43)
    check(*run_both(ref_b2e, lat, beam))


def test_chicane_without_charge_is_plain_tracking(ref_b2e):
    lat = w.chicane(bins=100, n_kicks=3, charge=0.0)
    beam = w.chicane_beam(5000, seed=2)
    check(*run_both(ref_b2e, lat, beam))


def _bunch_train(sizes, chirps, seed):
    from elegant_b200.beam import Beam
    parts, next_id = [], 1
    for k, (n, h) in enumerate(zip(sizes, chirps)):
        b = w.chicane_beam(n, seed=seed + k, chirp=h)
        parts.append(Beam(b.coords, np.arange(next_id, next_id + n)))
        next_id += n
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    return Beam(np.concatenate([p.coords for p in parts]), np.concatenate([p.ids for p in parts])), offsets


@pytest.mark.parametrize("drift_kicks", [1, 3])
def test_bunch_train_matches_single_bunches(ref_b2e, drift_kicks):
    """Bunches tracked together, each with its own histogram, wake and macro
    charge, give every bunch the reference's single-bunch result bit for bit
    (one bunch holds a single particle: no CSR for it)."""
    lat = w.chicane(bins=120, n_kicks=4)
    lat = Lattice([Element(e.name, e.type, dict(e.params, N_KICKS=drift_kicks)) if e.type == "CSRDRIFT" else e
                   for e in lat.elements])
    sizes, chirps = [3000, 1, 7000, 4500], [-10.0, -8.0, -15.0, -5.0]
    beam, offsets = _bunch_train(sizes, chirps, seed=50)
    with Tracker(lat, P0, 1) as t:
        t.load_ensemble(offsets, [])
        res = t.track(beam)
        wakes = t.csr_wakes(10_000_000)
    nb = len(sizes)
    wakes = wakes.reshape(-1, nb, 120)
    for b in range(nb):
        sl = slice(offsets[b], offsets[b + 1])
        rows, nl, _, ref_wakes = ref_b2e.track(lat, beam.coords[sl], beam.ids[sl], P0, 1, capture_wakes=True)
        sub = type(res)(res.coords[sl], res.ids[sl], res.lost_pass[sl], res.lost_element[sl],
                        int((res.lost_pass[sl] < 0).sum()), 0.0)
        ref_c, ref_ids, ref_loss = by_id(rows)
        order = np.argsort(sub.ids)
        assert sub.n_left == nl
        assert np.array_equal(sub.ids[order], ref_ids)
        alive = ref_loss < 0
        assert np.array_equal(sub.coords[order][alive], ref_c[alive]), b
        if sizes[b] > 1:
            assert np.array_equal(wakes[:, b, :].ravel(), ref_wakes), b


def _surrogate():
    import os
    from elegant_b200.wake_surrogate import WakeSurrogate
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "elegant_b200", "data",
                        "wakenet_1024.npz")
    return WakeSurrogate.load(path, max_batch=16)


def test_surrogate_zero_tolerance_is_the_plain_wake():
    """With tolerance 0 every kick whose integral is not empty falls back, and
    the fallback is the plain wake bit for bit; kicks with an empty integral
    (slippage under one bin) are exact in both paths."""
    lat = w.chicane(bins=200, n_kicks=6)
    beam = w.chicane_beam(20000, seed=31)
    with Tracker(lat, P0, 1) as t:
        plain = t.track(beam)
        plain_w = t.csr_wakes(10_000_000)
    sur = _surrogate()
    with Tracker(lat, P0, 1) as t:
        t.set_csr_surrogate(sur, tolerance=0.0, gate_stride=8)
        res = t.track(beam)
        wk = t.csr_wakes(10_000_000)
        stats = t.csr_surrogate_stats()
    assert np.array_equal(wk, plain_w)
    assert np.array_equal(res.coords, plain.coords)
    assert stats["evaluations"] == 4 * 6 and stats["fallbacks"] <= stats["evaluations"]


def test_surrogate_wakes_follow_the_plain_wakes():
    """At the default 1% gate, every kick's wake agrees with the plain wake of
    the same histogram to the gate's tolerance (or is the plain wake)."""
    lat = w.chicane(bins=600, n_kicks=20)
    beam = w.chicane_beam(200000, seed=32)
    sur = _surrogate()
    with Tracker(lat, P0, 1) as t:
        t.set_csr_surrogate(sur, tolerance=0.01, gate_stride=16)
        t.track(beam)
        stats = t.csr_surrogate_stats()
    errs = stats["gate_errors"]
    assert stats["evaluations"] == 80 and errs.size == 80
    assert np.all(np.isfinite(errs))
    # the fallback count is what the gate decided
    assert stats["fallbacks"] == int((errs > 0.01).sum())


class _HostExchange:
    """Two tracking contexts in two host threads on one GPU, each holding half
    of every bunch, exchanging through host memory at the engine's CSR
    reduction points (a stand-in for NCCL between GPUs: no kernel waits on
    another; the host threads meet at a barrier with a timeout)."""

    def __init__(self, n):
        import threading
        self.n = n
        self.barrier = threading.Barrier(n, timeout=120)
        self.slots = [None] * n

    def reducer(self, rank):
        import torch
        from elegant_b200.parallel import DeviceBuffer, REDUCE_MAX_U64, REDUCE_MIN_U64, REDUCE_SUM_U32

        def fn(op, ptr, count, stream):
            s = torch.cuda.ExternalStream(stream)
            t = torch.as_tensor(DeviceBuffer(ptr, count, "<i4" if op == REDUCE_SUM_U32 else "<i8"), device="cuda")
            with torch.cuda.stream(s):
                host = t.cpu().numpy().copy()
            self.slots[rank] = host
            self.barrier.wait()
            vals = np.stack(self.slots)
            if op == REDUCE_MIN_U64:
                out = vals.view(np.uint64).min(axis=0).view(np.int64)
            elif op == REDUCE_MAX_U64:
                out = vals.view(np.uint64).max(axis=0).view(np.int64)
            else:
                out = vals.sum(axis=0).astype(vals.dtype)
            self.barrier.wait()
            with torch.cuda.stream(s):
                t.copy_(torch.from_numpy(out))
            s.synchronize()
            return 0
        return fn


@pytest.mark.parametrize("train", [False, True])
def test_bunches_split_over_two_ranks_match_one(train):
    """Every bunch's particles split between two ranks, each rank's engine
    reducing min/max, histograms and counts with the other: the union of the
    two runs equals the one-rank run bit for bit, and both ranks log the same
    per-kick wakes."""
    import threading
    lat = w.chicane(bins=120, n_kicks=4)
    lat = Lattice([Element(e.name, e.type, dict(e.params, N_KICKS=2)) if e.type == "CSRDRIFT" else e
                   for e in lat.elements])
    sizes = [6000, 9000] if train else [12000]
    beam, offsets = _bunch_train(sizes, [-10.0, -14.0][:len(sizes)], seed=70)
    with Tracker(lat, P0, 1) as t:
        if train:
            t.load_ensemble(offsets, [])
        full = t.track(beam)
        full_w = t.csr_wakes(10_000_000)
    parts = []
    for r in range(2):
        idx = np.concatenate([np.arange(offsets[b] + r, offsets[b + 1], 2) for b in range(len(sizes))])
        loc = np.concatenate([[0], np.cumsum([len(range(offsets[b] + r, offsets[b + 1], 2))
                                              for b in range(len(sizes))])]).astype(np.int64)
        parts.append((idx, loc))
    ex = _HostExchange(2)
    results, errors = [None, None], []

    def run(r):
        try:
            from elegant_b200.beam import Beam
            idx, loc = parts[r]
            with Tracker(lat, P0, 1) as t:
                if train:
                    t.load_ensemble(loc, [])
                t.set_csr_reducer(ex.reducer(r))
                res = t.track(Beam(beam.coords[idx], beam.ids[idx]))
                results[r] = (res, t.csr_wakes(10_000_000))
        except Exception as e:  # reported below
            errors.append(e)
            ex.barrier.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for x in th:
        x.start()
    for x in th:
        x.join(timeout=300)
    assert not errors, errors
    for r in range(2):
        assert np.array_equal(results[r][1], full_w)
    order = np.argsort(full.ids)
    ids = np.concatenate([results[r][0].ids for r in range(2)])
    coords = np.concatenate([results[r][0].coords for r in range(2)])
    lost = np.concatenate([results[r][0].lost_pass for r in range(2)])
    o2 = np.argsort(ids)
    assert np.array_equal(ids[o2], full.ids[order])
    assert np.array_equal(lost[o2], full.lost_pass[order])
    alive = full.lost_pass[order] < 0
    assert np.array_equal(coords[o2][alive], full.coords[order][alive])


@pytest.mark.parametrize("bins", [2, 4096])
def test_chicane_extreme_bin_counts(ref_b2e, bins):
    lat = w.chicane(bins=bins, n_kicks=3)
    beam = w.chicane_beam(30000, seed=bins)
    check(*run_both(ref_b2e, lat, beam))


@pytest.mark.parametrize("bins,kicks", [(150, 4), (600, 6)])
def test_chicane_igf_bit_exact(ref_b2e, bins, kicks):
    """Steady-state CSR by the integrated Green's function (IGF=1): the
    device's chi/Green's-function tables, convolution and kicks equal the
    reference's bit for bit, per-kick wakes included."""
    lat = w.chicane(bins=bins, n_kicks=kicks)
    lat = Lattice([Element(e.name, e.type, dict(e.params, STEADY_STATE=1, IGF=1)) if e.type == "CSRCSBEND" else e
                   for e in lat.elements])
    beam = w.chicane_beam(25000, seed=bins + 1)
    check(*run_both(ref_b2e, lat, beam))


def test_torch_nccl_reducer_single_rank_is_identity():
    """The NCCL reducer (torch.distributed on the engine's stream) in a one-rank
    job: every exchange is an identity, so results equal the plain run bit
    for bit -- the plumbing (device-buffer views, stream ordering, the uint64
    key mapping) is exercised on the GPU."""
    import os
    import socket

    import torch.distributed as dist
    from elegant_b200.parallel import torch_csr_reducer

    lat = w.chicane(bins=150, n_kicks=4)
    beam, offsets = _bunch_train([8000, 5000], [-10.0, -12.0], seed=80)
    with Tracker(lat, P0, 1) as t:
        t.load_ensemble(offsets, [])
        ref = t.track(beam)
        ref_w = t.csr_wakes(10_000_000)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        with Tracker(lat, P0, 1) as t:
            t.load_ensemble(offsets, [])
            t.set_csr_reducer(torch_csr_reducer(dist))
            res = t.track(beam)
            wk = t.csr_wakes(10_000_000)
    finally:
        dist.destroy_process_group()
    assert np.array_equal(wk, ref_w)
    assert np.array_equal(res.coords, ref.coords)
    assert np.array_equal(res.lost_pass, ref.lost_pass)


@pytest.mark.parametrize("case", ["default", "fine_bins_3kicks", "dz", "no_sg", "steady_plain", "gap", "gap_mode0",
                                  "ring_2p", "ring_mode0_2p"])
def test_csrdrift_modes_bit_exact(case):
    """CSRDRIFT in Stupakov mode, a CSRDRIFT starting behind the dipole's
    wake and one ahead of the first dipole on the second pass: final
    coordinates and every dipole wake equal elegant's code (a fresh copy of
    the library per run, as a new elegant process) bit for bit."""
    from csr_cases import stupakov_cases
    from reforacle import RefOracle
    lat = stupakov_cases()[case]
    passes = 2 if case.endswith("2p") else 1
    beam = w.chicane_beam(20000, seed=31)
    with Tracker(lat, P0, passes) as t:
        res = t.track(beam)
        wakes = t.csr_wakes(10_000_000)
    rows, nl, _, ref_wakes = RefOracle("b2e", private=True).track(lat, beam.coords, beam.ids, P0, passes,
                                                                  capture_wakes=True)
    check(res, wakes, rows, nl, ref_wakes)


def test_stupakov_bunch_train_matches_single_bunches():
    """Bunches in Stupakov CSRDRIFTs: each bunch's own histogram, wake and
    phi solutions (its own carried start value) reproduce a separate
    reference run of that bunch bit for bit; the one-particle bunch drifts."""
    from reforacle import RefOracle
    lat = w.chicane(bins=300, n_kicks=4, stupakov=True, drift={"N_KICKS": 2})
    sizes, chirps = [3000, 1, 7000, 4500], [-10.0, -8.0, -15.0, -5.0]
    beam, offsets = _bunch_train(sizes, chirps, seed=51)
    with Tracker(lat, P0, 1) as t:
        t.load_ensemble(offsets, [])
        res = t.track(beam)
    for b in range(len(sizes)):
        sl = slice(offsets[b], offsets[b + 1])
        rows, nl, _, _ = RefOracle("b2e", private=True).track(lat, beam.coords[sl], beam.ids[sl], P0, 1)
        ref_c, ref_ids, ref_loss = by_id(rows)
        order = np.argsort(res.ids[sl])
        assert int((res.lost_pass[sl] < 0).sum()) == nl
        assert np.array_equal(res.ids[sl][order], ref_ids)
        alive = ref_loss < 0
        assert np.array_equal(res.coords[sl][order][alive], ref_c[alive]), b


@pytest.mark.parametrize("case", ["low_pass", "high_pass", "both_odd_bins", "round_trip_only", "no_clip_stupakov"])
def test_csr_histogram_filters_bit_exact(case):
    """LOW/HIGH_FREQUENCY_CUTOFF filters of the histogram (one CTA per
    bunch: twiddles, forward pairs, ramps, inverse, clipping) equal elegant's
    applyLHPassFilters on the shared transform, bit for bit."""
    from csr_cases import filter_cases
    from reforacle import RefOracle
    lat = filter_cases()[case]
    beam = w.chicane_beam(20000, seed=32)
    with Tracker(lat, P0, 1) as t:
        res = t.track(beam)
        wakes = t.csr_wakes(10_000_000)
    rows, nl, _, ref_wakes = RefOracle("b2e", private=True).track(lat, beam.coords, beam.ids, P0, 1,
                                                                  capture_wakes=True)
    check(res, wakes, rows, nl, ref_wakes)


@pytest.mark.parametrize("variant", ["default", "steady_plain", "igf"])
def test_csr_wake_output_file_matches_reference(ref_b2e, tmp_path, variant):
    """CSRCSBEND's OUTPUT_FILE: the engine's page records written as SDDS by
    elegant_b200.sdds.write_csr_wake (one file per dipole, one page per
    kick), read back with the protocol reader of tests/sdds_protocol.py, equal
    bit for bit to what the reference's own writer was handed on the same run
    (every column and parameter of every page; the IGF wake has no T1/T2)."""
    from elegant_b200.sdds import write_csr_wake
    from reforacle import CAPTURE_PARAMS, captured_pages
    from sdds_protocol import SddsFile
    lat = w.chicane(bins=150, n_kicks=5)
    extra = {"steady_plain": {"STEADY_STATE": 1, "TRAPAZOID_INTEGRATION": 0}, "igf": {"STEADY_STATE": 1, "IGF": 1},
             "default": {}}[variant]
    lat = Lattice([Element(e.name, e.type, dict(e.params, **extra)) if e.type == "CSRCSBEND" else e
                   for e in lat.elements])
    beam = w.chicane_beam(12000, seed=23)
    with Tracker(lat, P0, 1) as t:
        t.set_csr_pages(True)
        t.track(beam)
        pages = t.csr_pages()
    ref_b2e.track(lat, beam.coords, beam.ids, P0, 1, capture_wakes=True)
    cap = captured_pages(ref_b2e)
    assert len(pages) == cap["parameters"].shape[0] == 4 * 5
    read = []
    for el in sorted({p["element"] for p in pages}):
        path = tmp_path / f"wake_{el}.sdds"
        write_csr_wake(path, [p for p in pages if p["element"] == el])
        f = SddsFile(path)
        assert [c["name"] for c in f.columns] == ["s", "LinearDensity", "LinearDensityDeriv", "DeltaGamma",
                                                  "GammaDeriv", "DeltaGammaT1", "DeltaGammaT2"]
        read += f.pages
    columns = ["s", "LinearDensity", "LinearDensityDeriv", "DeltaGamma", "GammaDeriv"]
    if variant != "igf":
        columns += ["DeltaGammaT1", "DeltaGammaT2"]
    for name in columns:
        ours = np.concatenate([pg["columns"][name] for pg in read])
        assert ours.shape == cap[name].shape, name
        bad = np.flatnonzero(ours != cap[name])
        assert bad.size == 0, f"{name}: {bad.size} values differ, first {bad[:5]}"
    for k, name in enumerate(CAPTURE_PARAMS):
        ours = np.array([pg["parameters"][name] for pg in read], dtype=np.float64)
        assert np.array_equal(ours, cap["parameters"][:, k]), name


def test_watch_points_in_a_chicane(ref_b2e):
    """WATCH elements between and after the CSR dipoles: the particles the
    reference hands dump_watch_particles there, bit for bit, and the tracking
    unchanged."""
    lat = w.chicane(bins=150, n_kicks=5)
    els = []
    for e in lat.elements:
        els.append(e)
        if e.name in ("B2", "B4"):
            els.append(Element("W" + e.name, "WATCH", {"FILENAME": "%s.w"}))
    lat = Lattice(els)
    beam = w.chicane_beam(12000, seed=61)
    ref_b2e.set_watch(100000)
    rows, nl, _, ref_wakes = ref_b2e.track(lat, beam.coords, beam.ids, P0, 1, capture_wakes=True)
    ref_rows = ref_b2e.watch_rows()
    ref_b2e.set_watch(0)
    with Tracker(lat, P0, 1) as t:
        t.set_watch(1 << 28)
        res = t.track(beam)
        wakes = t.csr_wakes(10_000_000)
        recs = t.watch()
    check(res, wakes, rows, nl, ref_wakes)
    assert [r["element"] for r in recs] == lat.index("WB2") + lat.index("WB4")
    for r in recs:
        sel = ref_rows[ref_rows[:, 0] == r["element"]]
        sel = sel[np.argsort(sel[:, 2], kind="stable")]
        assert np.array_equal(r["ids"], sel[:, 2].astype(np.int64))
        assert np.array_equal(r["coords"], sel[:, 3:9])
