"""The momentum-aperture search's batching against elegant's serial scan
(CPU, on the reference build): all trials of a refinement level tracked at
once, one particle per run, give each element's last survivor, first loss
and its pass exactly; plus the element selection and the wedge placement."""
import numpy as np

from elegant_b200 import workloads as w
from elegant_b200.momentum_aperture import momentum_aperture, scan_deltas, select_elements, wedge_lattice
from ma_reference import oracle_trials, serial_momentum_aperture
from reforacle import RefOracle

P0 = w.ring_p_central()


def test_selection_and_wedges():
    lat = w.fodo_ring()
    z = np.cumsum([e.length for e in lat.elements])
    sel = select_elements(lat, s_start=3.0, s_end=8.0, include_type_pattern="K*")
    assert sel and all(lat.elements[i].type in ("KQUAD", "KSEXT") and 3.0 <= z[i] < 8.0 for i in sel)
    assert select_elements(lat, include_type_pattern="KQUAD", skip_elements=2, process_elements=3) == \
        [i for i, e in enumerate(lat.elements) if e.type == "KQUAD"][2:5]
    last = len(lat.elements) - 1
    wl, wedges = wedge_lattice(lat, [sel[0], last], 1)
    assert wl.elements[wedges[0]].type == "MALIGN" and wl.elements[wedges[0] - 1] is lat.elements[sel[0]]
    # the last element's wedge fires ahead of the first selected element
    assert wl.elements[wedges[1] + 1] is lat.elements[sel[0]] or wl.elements[wedges[1] + 2] is lat.elements[sel[0]]
    assert scan_deltas(0.0, 0.0025, 0.01)[-1] <= 0.01 and len(scan_deltas(0.0, -0.0025, -0.01)) == 5


def test_batched_search_matches_the_serial_scan():
    lat = w.fodo_ring()
    kw = dict(include_type_pattern="KQUAD", process_elements=3, delta_step_size=0.0015, splits=2)
    ref = RefOracle("b2e")
    serial = serial_momentum_aperture(ref, lat, P0, 40, **kw)
    rows, _ = momentum_aperture(lat, P0, 40, track_trials=oracle_trials(ref), **kw)
    assert len(rows) == len(serial) == 3
    for row, s in zip(rows, serial):
        for side, label in ((0, "negative"), (1, "positive")):
            got = row[label]
            assert (got["delta"], got["delta_lost"], got["lost_on_pass"]) == s[side], (row["name"], label)
        assert row["negative"]["delta"] < 0 < row["positive"]["delta"]


def mid_rf_ring():
    """The ring with its cavity moved into the third cell and made short
    (50 GHz, 20 MV): on a single pass a trial reaches it with its momentum
    offset, so the RF phase reference decides the energy it gets."""
    from elegant_b200 import Element, Lattice
    base = w.fodo_ring()
    rf = next(e for e in base.elements if e.type == "RFCA")
    els = [e for e in base.elements if e.type != "RFCA"]
    return Lattice(els[:24] + [Element("RF", "RFCA", dict(rf.params, FREQ=5e10, VOLT=2e7))] + els[24:])


def test_fiducialized_search_matches_the_serial_scan():
    """fiducialize = 1: one fiducial particle's RF phase for every trial
    (momentumAperture.c:385-410, :560-566).  The batched form (a fiducial row
    in every instance, the wedge on the trial's ID only) against the serial
    scan on the reference build, on one pass of mid_rf_ring, where the phase
    reference changes the answer; on 40 passes of the plain ring the wedge
    fires on pass 1, after each trial has set its own phase on pass 0 on the
    design orbit, and both settings agree."""
    kw = dict(include_type_pattern="KQUAD", process_elements=2, delta_step_size=0.0015, splits=2)
    ref = RefOracle("b2e")
    for lat, passes in ((mid_rf_ring(), 1), (w.fodo_ring(), 40)):
        serial = serial_momentum_aperture(ref, lat, P0, passes, fiducialize=True, **kw)
        rows, _ = momentum_aperture(lat, P0, passes, track_trials=oracle_trials(ref), fiducialize=True, **kw)
        for row, s in zip(rows, serial):
            for side, label in ((0, "negative"), (1, "positive")):
                got = row[label]
                assert (got["delta"], got["delta_lost"], got["lost_on_pass"]) == s[side], (row["name"], label)
        plain = serial_momentum_aperture(ref, lat, P0, passes, **kw)
        assert (plain != serial) == (passes == 1)


def test_output_mode_1_layout(tmp_path):
    """One row per element and side, negative first (momentumAperture.c:141-160,
    :715-731), read back with the independent SDDS reader."""
    from elegant_b200.sdds import write_momentum_aperture
    from sdds_protocol import SddsFile
    side = {"delta": -0.01, "found": True, "lost_on_pass": 3, "x_lost": 1e-3, "y_lost": 0.0, "s_lost": 2.5,
            "delta_when_lost": -0.011, "delta_lost": -0.0115}
    rows = [{"name": "QF", "type": "KQUAD", "s": 1.3, "occurrence": 2, "negative": side,
             "positive": dict(side, delta=0.02, found=False, lost_on_pass=-1)}]
    write_momentum_aperture(str(tmp_path / "ma1.sdds"), rows, output_mode=1)
    page = SddsFile(str(tmp_path / "ma1.sdds")).pages[0]
    c = page["columns"]
    assert list(c["direction"]) == [-1, 1] and list(c["deltaFound"]) == [1, 0]
    assert list(c["delta"]) == [-0.01, 0.02] and list(c["ElementOccurence"]) == [2, 2]
    assert list(c["lostOnPass"]) == [3, -1] and list(c["ElementName"]) == ["QF", "QF"]


def test_local_acceptance_grid():
    """output_mode 2's grid (momentumAperture.c:864-866, :823-827) with the
    reference's operations: 81 points over +-0.1 at 0.0025, the positive
    side from index 40; and starts away from zero."""
    from elegant_b200.momentum_aperture import acceptance_grid
    n, step, cut, deltas = acceptance_grid(-0.1, 0.1, 0.0, 0.0, 0.0025)
    assert (n, cut) == (81, 40) and step == 0.2 / 80
    assert deltas[0] == -0.1 and deltas[39] == -0.1 + 39 * step and deltas[40] == 0.0 and deltas[80] == 40 * step
    n, step, cut, deltas = acceptance_grid(-0.05, 0.04, -0.01, 0.02, 0.003)
    assert n == int(((0.04 - 0.02) + (-0.01 + 0.05)) / 0.003 + 1) and deltas[cut] == 0.02
    assert all(d < 0 for d in deltas[:cut]) and all(d >= 0.02 for d in deltas[cut:])


def test_local_acceptance_matches_the_serial_restatement():
    """output_mode 2 (multiparticleLocalMomentumAcceptance): the batched form
    (one instance per grid delta, a fiducial row first, the wedge at each
    selected element's entrance on its ID block) against one oracle run per
    particle, on one pass of mid_rf_ring (the fiducial's RF phase matters)
    and 40 passes of the ring."""
    from elegant_b200.momentum_aperture import local_momentum_acceptance
    from ma_reference import oracle_instances, serial_local_acceptance
    ref = RefOracle("b2e")
    kw = dict(process_elements=3, delta_step_size=0.0007, delta_negative_limit=-0.02, delta_positive_limit=0.02,
              s_start=2.0)
    for lat, passes in ((mid_rf_ring(), 1), (w.fodo_ring(), 40)):
        serial = serial_local_acceptance(ref, lat, P0, passes, **kw)
        rows, _ = local_momentum_acceptance(lat, P0, passes, track_trials=oracle_instances(ref), **kw)
        assert len(rows) == len(serial) == 3
        for row, s in zip(rows, serial):
            for side, label in ((0, "negative"), (1, "positive")):
                assert (row[label]["delta"], row[label]["delta_lost"]) == s[side], (row["name"], label)
        assert any(r["positive"]["found"] or r["negative"]["found"] for r in rows)


def test_local_acceptance_checks():
    import pytest
    from elegant_b200.momentum_aperture import local_momentum_acceptance
    lat = w.fodo_ring()
    with pytest.raises(ValueError, match="wildcards"):
        local_momentum_acceptance(lat, P0, 1, include_name_pattern="Q*")
    with pytest.raises(ValueError, match="include_type_pattern"):
        local_momentum_acceptance(lat, P0, 1, include_type_pattern="KQUAD")
    with pytest.raises(ValueError, match="invalid"):
        local_momentum_acceptance(lat, P0, 1, delta_negative_start=-0.0999)


def test_output_mode_2_layout(tmp_path):
    """The two limits per element (momentumAperture.c:163-180), read back
    with the independent SDDS reader."""
    from elegant_b200.sdds import write_momentum_aperture
    from sdds_protocol import SddsFile
    rows = [{"name": "QF", "type": "KQUAD", "s": 1.3, "occurrence": 2,
             "negative": {"delta": -0.01, "found": True, "delta_lost": -0.011},
             "positive": {"delta": 1.7976931348623157e308, "found": False, "delta_lost": None}}]
    write_momentum_aperture(str(tmp_path / "ma2.sdds"), rows, step=3, output_mode=2)
    page = SddsFile(str(tmp_path / "ma2.sdds")).pages[0]
    c = page["columns"]
    assert list(c) == ["ElementName", "s", "ElementType", "ElementOccurence", "deltaPositive", "deltaNegative"]
    assert list(c["deltaNegative"]) == [-0.01] and list(c["deltaPositive"]) == [1.7976931348623157e308]
    assert page["parameters"]["Step"] == 3 and list(c["ElementOccurence"]) == [2]


def test_forbid_resonance_crossing_bookkeeping():
    """forbid_resonance_crossing (momentumAperture.c:515-603) on the CPU with
    stand-in tunes (tune x crosses the half integer at delta = +0.0015 and
    -0.0152): the batched search against the reference's scan, losses,
    crossings and the last survivor's tunes; without forbid the tunes are
    only reported."""
    from ma_reference import oracle_run_trial, oracle_trials_with_tunes, serial_scan_with_tunes
    lat = w.fodo_ring()
    kw = dict(include_type_pattern="KQUAD", process_elements=2, delta_step_size=0.002, splits=2)
    ref = RefOracle("b2e")
    for forbid in (True, False):
        serial = serial_scan_with_tunes(oracle_run_trial(ref, P0), lat, 40, forbid, **kw)
        rows, _ = momentum_aperture(lat, P0, 40, track_trials=oracle_trials_with_tunes(ref),
                                    forbid_resonance_crossing=forbid, **kw)
        for row, s in zip(rows, serial):
            for side, label in ((0, "negative"), (1, "positive")):
                got = row[label]
                assert (got["delta"], got["delta_lost"], got["lost_on_pass"], got["nux"], got["nuy"]) == s[side]
        if forbid:
            assert all(r["positive"]["delta"] < 0.0015 and r["positive"]["lost_on_pass"] == -1 for r in rows)
        else:
            assert all(r["positive"]["nux"] > 0.5 for r in rows)
