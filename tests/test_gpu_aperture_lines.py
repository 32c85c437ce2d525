"""Line-mode dynamic aperture on the device: every refinement level of every
line is one engine run; the last survivor and the loss pass of each line
equal elegant's serial walk on its own code (oracle/_ref), one particle per
run (a lattice without RF, see tests/da_line_reference.py)."""
import pytest

from elegant_b200 import workloads as w
from elegant_b200.aperture import find_aperture_lines
from da_line_reference import serial_line_search

pytestmark = pytest.mark.gpu
P0 = w.ring_p_central()


@pytest.mark.parametrize("lines,splits,full", [(11, 2, False), (9, 1, True), (1, 3, False)])
def test_lines_equal_serial_walk(ref_b2e, lines, splits, full):
    lat = w.fodo_ring(rf=False)
    kw = dict(lines=lines, xmax=0.03, ymax=0.02, nx=15, n_splits=splits, full_plane=full)
    serial, origin = serial_line_search(ref_b2e, lat, P0, 50, **kw)
    got = find_aperture_lines(lat, P0, 50, **kw)
    assert got["origin_stable"] == origin
    for g, s in zip(got["lines"], serial):
        assert (g["x"], g["y"], g["lost_pass"]) == s


def test_lines_with_rf_share_the_origin_phase_reference():
    got = find_aperture_lines(w.fodo_ring(), P0, 100, lines=7, xmax=0.03, ymax=0.02, nx=13, n_splits=1)
    assert got["origin_stable"] and got["area"] > 0
    assert all(l["lost_pass"] >= 0 for l in got["lines"])


@pytest.mark.parametrize("lines,splits", [(11, 2), (5, 1)])
def test_slope_mode_equals_serial_walk(ref_b2e, lines, splits):
    """Slope mode (xmin == xmax, aperture_search.c:1029-1035): the lines in
    (x', y') on the device against the serial walk."""
    lat = w.fodo_ring(rf=False)
    kw = dict(lines=lines, nx=15, n_splits=splits, slope=True, xpmax=4e-3, ypmax=3e-3)
    serial, origin = serial_line_search(ref_b2e, lat, P0, 50, **kw)
    got = find_aperture_lines(lat, P0, 50, **kw)
    assert got["origin_stable"] == origin
    for g, s in zip(got["lines"], serial):
        assert (g["x"], g["y"], g["lost_pass"]) == s
