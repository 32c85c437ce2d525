"""The .ele runner (elegant_b200/ele.py): namelist parsing, &bunched_beam
statistics, what it declines (CPU), and a tracking job end to end (GPU)."""
import glob
import os

import numpy as np
import pytest

from elegant_b200.ele import BUNCHED_BEAM, EleError, bunched_beam, parse_namelists, run_ele

REFERENCE = os.environ.get("ELEGANT_REFERENCE_TREE", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="needs the reference tree")
def test_every_reference_run_file_parses():
    """All of the reference's example .ele files: comments, quoted strings
    with escapes, repeat counts (3*"gaussian") and indexed arrays."""
    files = sorted(glob.glob(os.path.join(REFERENCE, "**", "*.ele"), recursive=True))
    assert len(files) > 200
    for f in files:
        with open(f, errors="replace") as fh:
            cmds = parse_namelists(fh.read())
        assert cmds, f
    with open(os.path.join(REFERENCE, "doc/examples/bunchCompression/bunchComp/fourDipoleCSR.ele")) as fh:
        cmds = dict(parse_namelists(fh.read()))
    bb = cmds["bunched_beam"]
    assert bb["distribution_type"] == ["gaussian"] * 3 and bb["distribution_cutoff"] == ["3"] * 3
    assert bb["enforce_rms_values"] == ["1", "1", "1"] and cmds["run_setup"]["final"] == "%s.fin"


def test_namelist_syntax():
    text = '''! a comment
&run_setup lattice = "a b.lte", p_central_mev = 1e3, ! trailing comment
   final = %s.fin &end
&bunched_beam distribution_cutoff[1] = 2*4.5, centroid[4] = 1e-3, n_particles_per_bunch=8 &end
&track &end'''
    cmds = parse_namelists(text)
    assert [c for c, _ in cmds] == ["run_setup", "bunched_beam", "track"]
    assert cmds[0][1] == {"lattice": "a b.lte", "p_central_mev": "1e3", "final": "%s.fin"}
    assert cmds[1][1]["distribution_cutoff"] == [None, "4.5", "4.5"]
    assert cmds[1][1]["centroid"] == [None] * 4 + ["1e-3"]


def _bb(**kw):
    bb = dict(BUNCHED_BEAM)
    bb.update(kw)
    return bb


def test_bunched_beam_statistics():
    p0 = 1000 / 0.51099895
    bb = _bb(n_particles_per_bunch=40000, emit_nx=1e-6, beta_x=8.0, alpha_x=1.5, emit_y=2e-9, beta_y=3.0,
             alpha_y=-0.5, sigma_s=1e-3, sigma_dp=1e-4, momentum_chirp=-10.0, enforce_rms_values=[1, 1, 1],
             distribution_cutoff=[3.0, 3.0, 3.0], centroid=[1e-4, 0, 0, 0, 0, 0])
    b = bunched_beam(bb, p0, seed=3).coords
    x = b[:, 0] - b[:, 0].mean()
    xp = b[:, 1] - b[:, 1].mean()
    ex = np.sqrt((x * x).mean() * (xp * xp).mean() - (x * xp).mean() ** 2)
    assert abs(ex / (1e-6 / p0) - 1) < 1e-12  # enforced rms: the emittance exactly
    assert abs((x * x).mean() / (1e-6 / p0 * 8.0) - 1) < 1e-12
    assert abs(b[:, 0].mean() - 1e-4) < 1e-15
    assert abs(b[:, 4].std() / 1e-3 - 1) < 1e-12
    # chirp: delta = sigma_dp g + h s
    slope = np.polyfit(b[:, 4], b[:, 5], 1)[0]
    assert abs(slope + 10.0) < 0.1
    # cutoff at 2 sigma: the truncated Gaussian's values end near 2 sigma
    # (after centring and the exact-Twiss map, a little beyond it), where
    # 20,000 untruncated draws would reach about 4
    raw = bunched_beam(_bb(n_particles_per_bunch=20000, distribution_cutoff=[2.0, 2.0, 2.0], sigma_s=1.0,
                           sigma_dp=1.0), p0, seed=4).coords
    assert np.abs(raw[:, 4]).max() < 2.1
    sym = bunched_beam(_bb(n_particles_per_bunch=4000, emit_x=1e-9, emit_y=1e-9, sigma_s=1e-3, sigma_dp=1e-3,
                           symmetrize=1), p0, seed=5).coords
    assert np.abs(sym.mean(axis=0)).max() < 1e-18


def test_runner_declines_what_it_does_not_run(tmp_path):
    lte = tmp_path / "a.lte"
    lte.write_text("D: DRIF, L=1\nL1: LINE=(D)\n")
    cases = [("&run_setup lattice = a.lte, p_central = 100, sigma = %s.sig &end\n&track &end", "sigma"),
             ("&run_setup lattice = a.lte, p_central = 100 &end\n&sasefel beta = 1 &end", "sasefel"),
             ("&run_setup lattice = a.lte, p_central = 100 &end\n&bunched_beam distribution_type[0] = "
              '3*"uniform-ellipse", n_particles_per_bunch = 4 &end\n&track &end', "uniform-ellipse")]
    for text, word in cases:
        ele = tmp_path / "job.ele"
        ele.write_text(text)
        with pytest.raises(EleError, match=word):
            run_ele(str(ele))


@pytest.mark.gpu
def test_runner_tracks_a_chicane_job(tmp_path):
    """A CSR chicane job written as elegant would: the final file and the
    dipole's OUTPUT_FILE come out, and the final coordinates equal a direct
    engine run of the same generated beam."""
    from elegant_b200 import Tracker
    from elegant_b200.lattice import parse_lte
    from sdds_protocol import SddsFile
    (tmp_path / "chic.lte").write_text(
        'Q: CHARGE, TOTAL=1e-9\n'
        'B1: CSRCSBEND, L=0.5, ANGLE=0.05, N_KICKS=5, BINS=150, SG_HALFWIDTH=2, OUTPUT_FILE="%s.B1.wake"\n'
        'B2: CSRCSBEND, L=0.5, ANGLE=-0.05, N_KICKS=5, BINS=150, SG_HALFWIDTH=2\n'
        'D1: CSRDRIFT, L=2\n'
        'BL: LINE=(Q, B1, D1, B2)\n')
    (tmp_path / "job.ele").write_text(
        '&run_setup lattice = chic.lte, use_beamline = BL, p_central_mev = 1000, final = %s.fin,\n'
        '   random_number_seed = 77 &end\n'
        '&run_control n_passes = 1 &end\n'
        '&bunched_beam n_particles_per_bunch = 20000, emit_nx = 1e-6, emit_ny = 1e-6, beta_x = 10,\n'
        '   beta_y = 10, sigma_s = 1e-3, sigma_dp = 1e-4, momentum_chirp = -10, distribution_cutoff[0] = 3*3 &end\n'
        '&track &end\n')
    out = run_ele(str(tmp_path / "job.ele"))
    fin = SddsFile(str(tmp_path / "job.fin"))
    wake = SddsFile(str(tmp_path / "job.B1.wake"))
    assert len(wake.pages) == 5 and fin.pages[0]["parameters"]["Particles"] == out["steps"][0]["survivors"]
    bb = dict(BUNCHED_BEAM, n_particles_per_bunch=20000, emit_nx=1e-6, emit_ny=1e-6, beta_x=10.0, beta_y=10.0,
              sigma_s=1e-3, sigma_dp=1e-4, momentum_chirp=-10.0, distribution_cutoff=[3.0, 3.0, 3.0])
    p0 = 1000 / 0.51099895
    beam = bunched_beam(bb, p0, seed=77)
    lat = parse_lte((tmp_path / "chic.lte").read_text(), "BL", outputs={})
    with Tracker(lat, p0, 1) as t:
        ref = t.track(beam)
    alive = ref.lost_pass < 0
    assert np.array_equal(fin.pages[0]["columns"]["x"], ref.coords[alive, 0])
    assert np.array_equal(fin.pages[0]["columns"]["particleID"], ref.ids[alive])


def test_find_aperture_checks():
    """setup_aperture_search's input checks (aperture_search.c:118-170)."""
    from elegant_b200.ele import FIND_APERTURE, _check_find_aperture
    ok = dict(FIND_APERTURE, output="%s.aper", mode="n-line", n_lines=7)
    assert _check_find_aperture(ok) == ("n-line", False, 7)
    assert _check_find_aperture(dict(ok, xmin=0.0, xmax=0.0, xpmax=1e-3, ypmax=1e-3, ymin=0.0, ymax=0.0)) == \
        ("n-line", True, 7)
    assert _check_find_aperture(dict(ok, mode="five-line")) == ("five-line", False, 5)
    bad = [(dict(ok, output=None), "no output"), (dict(ok, xmin=0.2), "xmin >= xmax"),
           (dict(ok, xmin=0.0, xmax=0.0, xpmax=1e-3), "must not have xpmin==xpmax"),
           (dict(ok, mode="three-line", xmin=0.0, xmax=0.0, xpmax=1e-3, ypmax=1e-3, ymax=0.0), "slope-based"),
           (dict(ok, nx=2), "nx < 3"), (dict(ok, n_splits=1, split_fraction=1.5), "split_fraction"),
           (dict(ok, optimization_mode=1, n_lines=2), "optimization"),
           (dict(ok, mode="single-particle"), "single-particle")]
    for fa, words in bad:
        with pytest.raises(EleError, match=words):
            _check_find_aperture(fa)


@pytest.mark.gpu
def test_runner_aperture_commands(tmp_path):
    """&find_aperture (n-line, and slope mode with optimization_mode) and
    &momentum_aperture (fiducialize, output_mode 1; output_mode 2) from a
    run file: the files written equal the direct calls."""
    from elegant_b200 import workloads as w
    from elegant_b200.aperture import find_aperture_lines
    from elegant_b200.momentum_aperture import local_momentum_acceptance, momentum_aperture
    from sdds_protocol import SddsFile
    lat = w.fodo_ring(rf=False)
    lines = []
    for e in lat.elements:
        kv = ", ".join(f"{k}={v!r}" for k, v in e.params.items())
        lines.append(f"{e.name}: {e.type}" + (f", {kv}" if kv else ""))
    names = " ".join(e.name for e in lat.elements)
    (tmp_path / "ring.lte").write_text("\n".join(lines) + f"\nRING: LINE=({names.replace(' ', ', ')})\n")
    p0 = w.ring_p_central()
    (tmp_path / "da.ele").write_text(
        f'&run_setup lattice = ring.lte, use_beamline = RING, p_central = {p0!r} &end\n'
        '&run_control n_passes = 40 &end\n'
        '&find_aperture output = %s.aper, mode = "n-line", n_lines = 7, xmax = 0.03, ymax = 0.02, nx = 13,\n'
        '   n_splits = 1 &end\n'
        '&momentum_aperture output = %s.mmap, include_type_pattern = "KQUAD", process_elements = 2,\n'
        '   delta_step_size = 0.0015, fiducialize = 1, output_mode = 1 &end\n'
        '&find_aperture mode = "n-line", n_lines = 5, xmin = 0, xmax = 0, ymin = 0, ymax = 0, xpmax = 4e-3,\n'
        '   ypmax = 3e-3, nx = 11, optimization_mode = 1 &end\n'
        '&momentum_aperture output = %s.lma, s_start = 2, process_elements = 3, delta_step_size = 0.001,\n'
        '   delta_negative_limit = -0.02, delta_positive_limit = 0.02, output_mode = 2 &end\n')
    out = run_ele(str(tmp_path / "da.ele"))
    aper = SddsFile(str(tmp_path / "da.aper")).pages[0]
    want = find_aperture_lines(lat, p0, 40, lines=7, xmax=0.03, ymax=0.02, nx=13, n_splits=1)
    assert list(aper["columns"]["x"]) == [l["x"] for l in want["lines"]]
    assert aper["parameters"]["Area"] == want["area"]
    mmap = SddsFile(str(tmp_path / "da.mmap")).pages[0]
    rows, _ = momentum_aperture(lat, p0, 40, include_type_pattern="KQUAD", process_elements=2,
                                delta_step_size=0.0015, fiducialize=True)
    assert list(mmap["columns"]["delta"]) == [r[s]["delta"] for r in rows for s in ("negative", "positive")]
    slope = find_aperture_lines(lat, p0, 40, lines=5, nx=11, slope=True, xpmax=4e-3, ypmax=3e-3)
    assert out["steps"][-2]["area"] == slope["area"]
    lma = SddsFile(str(tmp_path / "da.lma")).pages[0]["columns"]
    rows, _ = local_momentum_acceptance(lat, p0, 40, s_start=2.0, process_elements=3, delta_step_size=0.001,
                                        delta_negative_limit=-0.02, delta_positive_limit=0.02)
    assert list(lma["deltaPositive"]) == [r["positive"]["delta"] for r in rows]
    assert list(lma["deltaNegative"]) == [r["negative"]["delta"] for r in rows]
    assert list(lma["ElementName"]) == [r["name"] for r in rows]


def test_runner_sdds_beam_checks(tmp_path):
    (tmp_path / "a.lte").write_text("D: DRIF, L=1\nL1: LINE=(D)\n")
    cases = [('&sdds_beam input = b.sdds, input_type = "spiffe" &end', "spiffe"),
             ("&sdds_beam input = b.sdds, center_arrival_time = 1 &end", "center_arrival_time"),
             ("&sdds_beam &end", "no input")]
    for text, word in cases:
        (tmp_path / "job.ele").write_text("&run_setup lattice = a.lte, p_central = 100 &end\n" + text + "\n&track &end")
        with pytest.raises(EleError, match=word):
            run_ele(str(tmp_path / "job.ele"))


@pytest.mark.gpu
def test_runner_tracks_an_sdds_beam(tmp_path):
    """&sdds_beam + &track: a phase-space file written by the engine (t, p
    columns), read back page by page (two steps, two pages), tracked; the
    final file equals tracking beam_from_sdds directly."""
    from elegant_b200 import Tracker, workloads as w
    from elegant_b200.sdds import beam_from_sdds, write_phase_space
    from elegant_b200.track import TrackResult
    from sdds_protocol import SddsFile
    lat = w.fodo_ring(rf=False)
    p0 = w.ring_p_central()
    lines = [f"{e.name}: {e.type}, " + ", ".join(f"{k}={v!r}" for k, v in e.params.items()) for e in lat.elements]
    (tmp_path / "ring.lte").write_text("\n".join(lines) + "\nRING: LINE=(" + ", ".join(e.name for e in lat.elements)
                                       + ")\n")
    path = str(tmp_path / "in.sdds")
    for step in (1, 2):
        b = w.ring_beam(3000, seed=60 + step)
        res = TrackResult(b.coords, b.ids, np.full(b.n, -1, np.int32), np.full(b.n, -1, np.int32), b.n, 0.0)
        write_phase_space(path, res, p0, step=step, append=step > 1)
    (tmp_path / "job.ele").write_text(
        f"&run_setup lattice = ring.lte, use_beamline = RING, p_central = {p0!r}, final = %s.fin &end\n"
        "&run_control n_passes = 20, n_steps = 2 &end\n"
        "&sdds_beam input = in.sdds &end\n&track &end\n")
    run_ele(str(tmp_path / "job.ele"))
    fin = SddsFile(str(tmp_path / "job.fin"))
    assert len(fin.pages) == 2
    for k in range(2):
        beam = beam_from_sdds(path, p0, page=k)
        with Tracker(lat, p0, 20) as t:
            ref = t.track(beam)
        alive = ref.lost_pass < 0
        assert np.array_equal(fin.pages[k]["columns"]["x"], ref.coords[alive, 0])


@pytest.mark.gpu
def test_runner_writes_watch_files(tmp_path):
    """A WATCH with FILENAME in the .lte: the runner writes one page per
    recorded pass; the rows equal the engine's WATCH records."""
    from elegant_b200 import Tracker, workloads as w
    from elegant_b200.lattice import parse_lte
    from sdds_protocol import SddsFile
    lat = w.fodo_ring(rf=False)
    lines = [f"{e.name}: {e.type}, " + ", ".join(f"{k}={v!r}" for k, v in e.params.items()) for e in lat.elements]
    lines.append('W1: WATCH, FILENAME="%s.w1", INTERVAL=2, START_PASS=1, END_PASS=7')
    lines.append('W2: WATCH, FILENAME="%s.w2", MODE="parameter"')
    names = [e.name for e in lat.elements]
    names.insert(10, "W1")
    names.append("W2")
    (tmp_path / "ring.lte").write_text("\n".join(lines) + "\nRING: LINE=(" + ", ".join(names) + ")\n")
    p0 = w.ring_p_central()
    (tmp_path / "job.ele").write_text(
        f"&run_setup lattice = ring.lte, use_beamline = RING, p_central = {p0!r}, random_number_seed = 5 &end\n"
        "&run_control n_passes = 10 &end\n"
        "&bunched_beam n_particles_per_bunch = 2000, emit_x = 1e-8, emit_y = 1e-8, beta_x = 10, beta_y = 10,\n"
        "   sigma_dp = 1e-3, sigma_s = 1e-3 &end\n&track &end\n")
    run_ele(str(tmp_path / "job.ele"))
    f = SddsFile(str(tmp_path / "job.w1"))
    assert [pg["parameters"]["Pass"] for pg in f.pages] == [1, 3, 5, 7]
    lat2 = parse_lte((tmp_path / "ring.lte").read_text(), "RING")
    from elegant_b200.ele import BUNCHED_BEAM
    bb = dict(BUNCHED_BEAM, n_particles_per_bunch=2000, emit_x=1e-8, emit_y=1e-8, beta_x=10.0, beta_y=10.0,
              sigma_dp=1e-3, sigma_s=1e-3)
    beam = bunched_beam(bb, p0, seed=5)
    with Tracker(lat2, p0, 10) as t:
        t.set_watch(1 << 30)
        t.track(beam)
        recs = t.watch()
    w1 = [r for r in recs if r["element"] == lat2.index("W1")[0]]
    for pg, r in zip(f.pages, w1):
        assert np.array_equal(pg["columns"]["x"], r["coords"][:, 0])
        assert np.array_equal(pg["columns"]["particleID"], r["ids"])
    # parameter mode: one page, a row per pass, the statistics of the records
    from elegant_b200.sdds import watch_statistics
    w2 = [r for r in recs if r["element"] == lat2.index("W2")[0]]
    f2 = SddsFile(str(tmp_path / "job.w2"))
    assert len(f2.pages) == 1 and list(f2.pages[0]["columns"]["Pass"]) == list(range(10)) == [r["pass"] for r in w2]
    for k, r in enumerate(w2):
        st = watch_statistics(r["coords"], r["ids"], p0)
        assert f2.pages[0]["columns"]["Cx"][k] == st["centroid"][0]
        assert f2.pages[0]["columns"]["ex"][k] == st["ex"]


@pytest.mark.gpu
def test_runner_watch_files_under_a_small_budget(tmp_path, monkeypatch):
    """A device-memory budget smaller than the run's WATCH records: the runner
    tracks in calls of fewer passes (continuing the same run) and the files
    are the same as with the whole run in one call."""
    import elegant_b200.ele as ele
    from elegant_b200 import workloads as w
    from sdds_protocol import SddsFile
    lat = w.fodo_ring(rf=False)
    lines = [f"{e.name}: {e.type}, " + ", ".join(f"{k}={v!r}" for k, v in e.params.items()) for e in lat.elements]
    lines += ['W1: WATCH, FILENAME="%s.w1"', 'W2: WATCH, FILENAME="%s.w2", MODE="centroid"']
    names = [e.name for e in lat.elements]
    names.insert(7, "W1")
    names.append("W2")
    (tmp_path / "ring.lte").write_text("\n".join(lines) + "\nRING: LINE=(" + ", ".join(names) + ")\n")
    p0 = w.ring_p_central()
    job = (f"&run_setup lattice = ring.lte, use_beamline = RING, p_central = {p0!r}, final = %s.fin,\n"
           "   random_number_seed = 9 &end\n&run_control n_passes = 12 &end\n"
           "&bunched_beam n_particles_per_bunch = 1000, emit_x = 5e-8, emit_y = 5e-8, beta_x = 10, beta_y = 10,\n"
           "   sigma_dp = 3e-3, sigma_s = 1e-3 &end\n&track &end\n")
    (tmp_path / "a.ele").write_text(job)
    (tmp_path / "b.ele").write_text(job)
    run_ele(str(tmp_path / "a.ele"))
    monkeypatch.setattr(ele, "WATCH_BUDGET_BYTES", 2 * 7 * 8 * 1000 * 3)  # three passes per call
    run_ele(str(tmp_path / "b.ele"))
    for ext in ("w1", "w2", "fin"):
        fa, fb = SddsFile(str(tmp_path / f"a.{ext}")), SddsFile(str(tmp_path / f"b.{ext}"))
        assert len(fa.pages) == len(fb.pages)
        for pa, pb in zip(fa.pages, fb.pages):
            for k, v in pa["columns"].items():
                if k in ("ElapsedTime", "ElapsedCoreTime", "MemoryUsage"):
                    continue
                assert np.array_equal(np.asarray(v), np.asarray(pb["columns"][k])), (ext, k)
