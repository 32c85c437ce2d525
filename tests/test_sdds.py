"""SDDS output in elegant's phase-space, loss and caller layouts (CPU).

Every file is read back with tests/sdds_protocol.py, a reader written from
the SDDS protocol apart from the writer (elegant_b200.sdds), which itself
reads every SDDS file the reference ships (binary in both byte orders and
ASCII, with and without row counts)."""
import glob
import os

import numpy as np
import pytest

from elegant_b200 import workloads as w
from elegant_b200.sdds import write_losses, write_phase_space
from elegant_b200.track import TrackResult
from sdds_protocol import SddsFile

REFERENCE = os.environ.get("ELEGANT_REFERENCE_TREE", "/root/reference")


def read_sdds(path):
    """(parameters, columns) of a one-page file, by the independent reader."""
    f = SddsFile(path)
    assert len(f.pages) == 1
    return f.pages[0]["parameters"], f.pages[0]["columns"]


def column_type(path, name):
    return next(c["type"] for c in SddsFile(path).columns if c["name"] == name)


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="needs the reference tree")
def test_reader_reads_the_reference_sdds_files():
    """The protocol reader against files the SDDS toolkit wrote: every page
    read to the last byte (binary) or line (ASCII), with columns of equal
    length, in all three encodings."""
    files = sorted(glob.glob(os.path.join(REFERENCE, "**", "*.sdds"), recursive=True))
    assert len(files) > 50
    modes = set()
    for path in files:
        f = SddsFile(path)
        modes.add((f.mode, f.endian if f.mode == "binary" else ""))
        assert f.pages, path
        for page in f.pages:
            lengths = {len(v) for v in page["columns"].values()}
            assert len(lengths) <= 1, path
    assert {("binary", ">"), ("binary", "<"), ("ascii", "")} <= modes


def _result():
    rng = np.random.default_rng(2)
    n = 50
    c = rng.normal(0, 1e-3, (n, 6))
    lost = np.full(n, -1, dtype=np.int32)
    lost[[3, 7, 20]] = [0, 5, 9]
    elem = np.full(n, -1, dtype=np.int32)
    elem[[3, 7, 20]] = [2, 10, 64]
    return TrackResult(c, np.arange(1, n + 1, dtype=np.int64), lost, elem, int((lost < 0).sum()), 0.0)


@pytest.mark.parametrize("mode", ["binary", "ascii"])
def test_phase_space_round_trip(tmp_path, mode):
    r = _result()
    p0 = 5870.8
    path = tmp_path / f"final.{mode}.sdds"
    write_phase_space(path, r, p0, step=3, charge=1e-9, mode=mode)
    head = open(path, "rb").read(200)
    assert head.startswith(b"SDDS1\n")
    params, cols = read_sdds(path)
    alive = r.lost_pass < 0
    assert params["Step"] == 3 and params["Particles"] == alive.sum()
    assert params["pCentral"] == p0 and params["Charge"] == 1e-9
    assert np.array_equal(cols["particleID"], r.ids[alive])
    assert np.array_equal(cols["x"], r.coords[alive, 0])
    p = p0 * (1 + r.coords[alive, 5])
    assert np.array_equal(cols["p"], p)
    np.testing.assert_allclose(cols["t"], r.coords[alive, 4] / (2.99792458e8 * p / np.sqrt(p * p + 1)), rtol=1e-15)


def test_losses_layout(tmp_path):
    r = _result()
    lat = w.fodo_ring()
    path = tmp_path / "losses.sdds"
    write_losses(path, r, lat, 5870.8)
    params, cols = read_sdds(path)
    assert list(cols) == ["x", "xp", "y", "yp", "s", "p", "particleID", "Pass"]
    assert cols["particleID"].tolist() == [4, 8, 21] and cols["Pass"].tolist() == [0, 5, 9]
    z = np.cumsum([e.length for e in lat.elements])
    assert cols["s"].tolist() == [z[2], z[10], z[64]]


@pytest.mark.parametrize("mode", ["binary", "ascii"])
def test_caller_outputs_round_trip(tmp_path, mode):
    from elegant_b200.sdds import write_aperture, write_frequency_map, write_momentum_aperture
    side = {"delta": 0.0123, "found": True, "lost_on_pass": 7, "x_lost": 0.02, "y_lost": 1e-6, "s_lost": 3.5,
            "delta_when_lost": 0.0131, "delta_lost": 0.0125}
    rows = [{"name": "QF", "type": "KQUAD", "s": 0.8, "positive": side, "negative": dict(side, delta=-0.01)},
            {"name": "QF", "type": "KQUAD", "s": 4.6, "positive": side, "negative": dict(side, found=False)}]
    p = tmp_path / f"ma.{mode}"
    write_momentum_aperture(p, rows, step=2, mode=mode)
    pv, c = read_sdds(p)
    assert pv["Step"] == 2 and c["ElementName"] == ["QF", "QF"] and list(c["ElementOccurence"]) == [1, 2]
    assert list(c["deltaNegative"]) == [-0.01, 0.0123] and list(c["deltaNegativeFound"]) == [1, 0]
    assert list(c["lostOnPassPositive"]) == [7, 7] and column_type(p, "deltaPositiveFound") == "short"
    fm = [{"x": 1e-3, "y": 2e-3, "delta": 0.0, "nux": 0.21, "nuy": 0.33, "s": 30.4, "dnux": 1e-7, "dnuy": 2e-7,
           "dnu": 2.2e-7, "dx": 0.0, "dy": 0.0, "diffusion": -13.3, "diffusionRate": -15.0}]
    p = tmp_path / f"fma.{mode}"
    write_frequency_map(p, fm, include_changes=True, mode=mode)
    _, c = read_sdds(p)
    assert c["nux"][0] == 0.21 and c["diffusion"][0] == -13.3
    ap = {"lines": [{"x": -0.01, "y": 0.0, "x_lost": -0.011, "y_lost": 0.0},
                    {"x": 0.0, "y": 0.008, "x_lost": None, "y_lost": None}],
          "x_limit": [-0.01, 0.0], "y_limit": [0.0, 0.008], "area": 4e-5}
    p = tmp_path / f"ap.{mode}"
    write_aperture(p, ap, mode=mode)
    pv, c = read_sdds(p)
    assert pv["Area"] == 4e-5 and list(c["xClipped"]) == [-0.01, 0.0] and c["xLost"][1] > 1e300


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="needs the reference tree")
def test_product_reader_agrees_with_the_protocol_reader_on_reference_files():
    """elegant_b200.sdds.read_sdds_pages (the engine's input reader) against
    the independent protocol reader on every SDDS file in the reference tree
    (ASCII and binary, both byte orders, fixed-value parameters, float,
    short and string columns): every page, column and parameter equal, float
    columns compared at their declared 32-bit width."""
    from elegant_b200.sdds import read_sdds_pages
    files = sorted(glob.glob(os.path.join(REFERENCE, "**", "*.sdds"), recursive=True))
    assert len(files) > 50
    checked = 0
    for f in files:
        mine = read_sdds_pages(f)
        ref = SddsFile(f)
        assert len(mine) == len(ref.pages), f
        for (pv, cv), page in zip(mine, ref.pages):
            for k, v in page["columns"].items():
                got = cv[k]
                if isinstance(got, list):
                    assert list(v) == got, (f, k)
                else:
                    assert np.array_equal(np.asarray(v, dtype=got.dtype), got, equal_nan=True), (f, k)
            for k, v in page["parameters"].items():
                assert v == pv[k] or (v != v and pv[k] != pv[k]), (f, k)
        checked += 1
    assert checked == len(files)


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="needs the reference tree")
def test_beam_from_an_elegant_phase_space_file():
    """&sdds_beam's point-particle conversion (sdds_beam.c:408-440) of the
    reference's own big-endian beam file: s = t c p / gamma, delta =
    (p - p0)/p0, IDs by row, every sample_interval-th row, the p window."""
    from elegant_b200.sdds import beam_from_sdds
    f = os.path.join(REFERENCE, "doc/examples/full457MeV/beamFile.sdds")
    page = SddsFile(f).pages[0]["columns"]
    p = np.asarray(page["p"])
    p0 = float(np.median(p))
    b = beam_from_sdds(f, p0)
    assert b.n == len(p) and np.array_equal(b.ids, np.arange(1, b.n + 1))
    assert np.array_equal(b.coords[:, 0], np.asarray(page["x"]))
    assert np.array_equal(b.coords[:, 4], np.asarray(page["t"]) * 2.99792458e8 * p / np.sqrt(p * p + 1))
    assert np.array_equal(b.coords[:, 5], (p - p0) / p0)
    half = beam_from_sdds(f, p0, sample_interval=2, p_lower=p0 * 0.999, p_upper=p0 * 1.001)
    sel = np.arange(0, len(p), 2)
    sel = sel[(p[sel] >= p0 * 0.999) & (p[sel] <= p0 * 1.001)]
    assert np.array_equal(half.coords[:, 1], np.asarray(page["xp"])[sel])
    assert np.array_equal(half.ids, sel + 1)


@pytest.mark.parametrize("mode", ["binary", "ascii"])
def test_pages_appended_per_step(tmp_path, mode):
    """One page per step, as elegant writes its final/losses files: the second
    step appended to the first, read back by the protocol reader and by the
    engine's own input reader."""
    from elegant_b200.sdds import read_sdds_pages
    path = str(tmp_path / f"steps.{mode}")
    for step, seed in ((1, 5), (2, 6)):
        b = w.ring_beam(50 + step, seed=seed)
        res = TrackResult(b.coords, b.ids, np.full(b.n, -1, np.int32), np.full(b.n, -1, np.int32), b.n, 0.0)
        write_phase_space(path, res, 1000.0, step=step, mode=mode, append=step > 1)
    f = SddsFile(path)
    assert [p["parameters"]["Step"] for p in f.pages] == [1, 2]
    assert [len(p["columns"]["x"]) for p in f.pages] == [51, 52]
    mine = read_sdds_pages(path)
    assert [pv["Step"] for pv, _ in mine] == [1, 2]
    assert np.array_equal(mine[1][1]["x"], f.pages[1]["columns"]["x"])


def test_watch_file_layout(tmp_path):
    """write_watch: dump_watch_particles' columns and parameters
    (sdds_support.c:403-520, :703-860), EXCLUDE_SLOPES and the PID window,
    PassCentralTime as the Kahan-summed revolution times."""
    from elegant_b200.sdds import watch_pass_central_times, write_watch
    rng = np.random.default_rng(9)
    recs = []
    for q in (0, 3, 6):
        n = 20 - q
        c = rng.normal(0, 1e-3, (n, 6))
        recs.append({"pass": q, "ids": np.arange(1, n + 1), "coords": c})
    p0, z, length = 2000.0, 7.5, 30.4
    write_watch(str(tmp_path / "w.sdds"), recs, p0, z, length, step=2, charge=1e-12,
                watch={"EXCLUDE_SLOPES": 1, "START_PID": 3, "END_PID": 15})
    f = SddsFile(str(tmp_path / "w.sdds"))
    names = [c["name"] for c in f.columns]
    assert names == ["x", "y", "t", "p", "dt", "particleID"]
    t0 = watch_pass_central_times([0, 3, 6], z, length, p0)
    root = np.sqrt(p0 * p0 + 1)
    # the Kahan sum of three equal steps against plain arithmetic: within an ulp
    assert abs(t0[2] - (z + 6 * length) * root / (2.99792458e8 * p0)) < 1e-20
    for page, r, t in zip(f.pages, recs, t0):
        keep = (r["ids"] >= 3) & (r["ids"] <= 15)
        prm = page["parameters"]
        assert prm["Pass"] == r["pass"] and prm["Step"] == 2 and prm["Particles"] == keep.sum()
        assert prm["PassCentralTime"] == t and prm["s"] == z and prm["PassLength"] == length
        assert abs(prm["Charge"] - 1e-12 * keep.sum()) < 1e-24
        assert np.array_equal(page["columns"]["particleID"], r["ids"][keep])
        pp = p0 * (1 + r["coords"][keep, 5])
        tt = r["coords"][keep, 4] / (2.99792458e8 * pp / np.sqrt(pp * pp + 1))
        assert np.array_equal(page["columns"]["t"], tt) and np.array_equal(page["columns"]["dt"], tt - t)


@pytest.mark.skipif(not os.path.isdir(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref")),
                    reason="needs oracle/_ref")
@pytest.mark.parametrize("window", [(-1, -1), (20, 700)])
def test_watch_statistics_against_accumulate_beam_sums(window):
    """The parameter/centroid-mode reduction against elegant's own
    accumulate_beam_sums (compute_centroids.c, compiled into the reference
    build) on the same rows: centroids of x..delta and t, and the sparse
    second moments, to rounding (elegant sums with Kahan's compensation in
    its array order, numpy pairwise)."""
    import ctypes
    from elegant_b200.sdds import watch_statistics
    from reforacle import RefOracle
    lib = RefOracle("libm").lib
    f = lib.b2e_ref_beam_sums
    f.restype = ctypes.c_long
    rng = np.random.default_rng(17)
    n, p0 = 1000, 2000.0
    c = np.column_stack([rng.normal(0, 1e-3, n), rng.normal(0, 1e-4, n), rng.normal(0, 5e-4, n),
                         rng.normal(0, 5e-5, n), rng.normal(3.0, 1e-3, n), rng.normal(0, 1e-3, n)])
    c[:, 0] += 2.0 * c[:, 5]  # dispersion, so that ecx differs from ex
    ids = rng.permutation(n) + 1
    rows = np.column_stack([c, ids]).astype(np.float64).copy()
    cen = np.zeros(7)
    sig = np.zeros(49)
    npc = f(rows.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(n), ctypes.c_double(p0), ctypes.c_long(window[0]),
            ctypes.c_long(window[1]), cen.ctypes.data_as(ctypes.c_void_p), sig.ctypes.data_as(ctypes.c_void_p))
    st = watch_statistics(c, ids, p0, *window)
    assert st["n"] == npc and npc > 0
    assert np.allclose(st["centroid"], cen, rtol=1e-12, atol=1e-18)
    sig = sig.reshape(7, 7)
    assert np.allclose(st["sigma"], sig, rtol=1e-11, atol=1e-30)
    assert (st["sigma"] == 0).sum() == (sig == 0).sum()  # the same sparse pattern
    assert st["ecx"] < st["ex"]


@pytest.mark.parametrize("wmode", [1, 2], ids=["parameter", "centroid"])
def test_watch_parameter_and_centroid_layouts(tmp_path, wmode):
    """Parameter mode: 31 columns, centroid mode: the first 19
    (sdds_support.c:359-393); one page per step, one row per recorded pass,
    the values from watch_statistics."""
    from elegant_b200.sdds import watch_pass_central_times, watch_statistics, write_watch
    rng = np.random.default_rng(3)
    recs = [{"pass": q, "ids": np.arange(1, 101 - q), "coords": rng.normal(0, 1e-3, (100 - q, 6))}
            for q in (0, 2, 4)]
    path = str(tmp_path / "wp.sdds")
    for step in (1, 2):
        write_watch(path, recs, 2000.0, 4.0, 30.4, step=step, charge=1e-12, watch={"MODE": wmode},
                    original_particles=100, previous_element="QF", append=step > 1)
    f = SddsFile(path)
    assert len(f.pages) == 2
    names = [c["name"] for c in f.columns]
    assert len(names) == (31 if wmode == 1 else 19) and names[:6] == ["Step", "Pass", "ElapsedTime",
                                                                       "ElapsedCoreTime", "MemoryUsage", "Cx"]
    page = f.pages[1]
    assert page["parameters"]["Step"] == 2 and page["parameters"]["PreviousElementName"] == "QF"
    col = page["columns"]
    assert list(col["Pass"]) == [0, 2, 4] and list(col["Particles"]) == [100, 98, 96]
    t0 = watch_pass_central_times([0, 2, 4], 4.0, 30.4, 2000.0)
    for k, r in enumerate(recs):
        st = watch_statistics(r["coords"], r["ids"], 2000.0)
        assert col["Cx"][k] == st["centroid"][0] and col["dCt"][k] == st["Ct"] - t0[k]
        assert col["Transmission"][k] == len(r["ids"]) / 100
        if wmode == 1:
            assert col["Sx"][k] == np.sqrt(st["sigma"][0, 0]) and col["ex"][k] == st["ex"]
