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
