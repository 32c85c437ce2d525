"""Line-mode dynamic aperture (CPU, on the reference build): the batched
search (all lines of a refinement level in one run) equals elegant's serial
walk point by point, and the island trimming and area equal elegant's own
trimApertureSearchResult compiled from its sources."""
import ctypes

import numpy as np
import pytest

from elegant_b200 import workloads as w
from elegant_b200.aperture import find_aperture_lines, line_factors, trim_aperture
from da_line_reference import serial_line_search
from reforacle import RefOracle

P0 = w.ring_p_central()


def _oracle_points(oracle):
    def run(lattice, p_central, n_passes, coords):
        lost = np.full(len(coords), -1, dtype=np.int32)
        end = np.zeros_like(coords)
        for k in range(len(coords)):
            rows, n_left, _ = oracle.track(lattice, coords[k:k + 1], np.array([1]), p_central, n_passes)[:3]
            end[k] = rows[0, :6]
            if n_left == 0:
                lost[k] = int(rows[0, 7])
        return lost, end
    return run


@pytest.mark.parametrize("lines,splits,full", [(11, 0, False), (5, 2, False), (3, 1, False), (9, 1, True)])
def test_batched_lines_equal_serial_walk(lines, splits, full):
    lat = w.fodo_ring(rf=False)
    ref = RefOracle("b2e")
    kw = dict(lines=lines, xmax=0.03, ymax=0.02, nx=11, n_splits=splits, full_plane=full)
    serial, origin = serial_line_search(ref, lat, P0, 30, **kw)
    got = find_aperture_lines(lat, P0, 30, track_points=_oracle_points(ref), **kw)
    assert got["origin_stable"] == origin
    for g, s in zip(got["lines"], serial):
        assert (g["x"], g["y"], g["lost_pass"]) == s
    assert got["area"] > 0


@pytest.mark.parametrize("lines,splits", [(7, 1), (3, 0)])
def test_slope_mode_lines_equal_serial_walk(lines, splits, tmp_path):
    """Slope mode (xmin == xmax): the lines in (x', y'), points offsetting the
    slopes (aperture_search.c:1029-1035, :1070-1076); and its output file's
    column set (:32-39), read with the independent SDDS reader."""
    from elegant_b200.sdds import write_aperture
    from sdds_protocol import SddsFile
    lat = w.fodo_ring(rf=False)
    ref = RefOracle("b2e")
    kw = dict(lines=lines, nx=11, n_splits=splits, slope=True, xpmax=4e-3, ypmax=3e-3)
    serial, origin = serial_line_search(ref, lat, P0, 30, **kw)
    got = find_aperture_lines(lat, P0, 30, track_points=_oracle_points(ref), **kw)
    assert got["origin_stable"] == origin and got["slope"]
    for g, s in zip(got["lines"], serial):
        assert (g["x"], g["y"], g["lost_pass"]) == s
    assert any(g["lost_pass"] >= 0 for g in got["lines"])
    write_aperture(str(tmp_path / "da.sdds"), got)
    page = SddsFile(str(tmp_path / "da.sdds")).pages[0]
    assert [k for k in page["columns"]][:4] == ["xp", "yp", "xpClipped", "ypClipped"]
    assert list(page["columns"]["xp"]) == [g["x"] for g in got["lines"]]
    with pytest.raises(ValueError):
        find_aperture_lines(lat, P0, 30, lines=3, slope=True, xpmax=1e-3, ypmax=0.0)


@pytest.mark.parametrize("full", [False, True])
def test_trim_and_area_equal_elegant(full):
    lib = RefOracle("libm").lib
    f = lib.trimApertureSearchResult
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_long] + [ctypes.c_void_p] * 4 + [ctypes.c_long]
    rng = np.random.default_rng(3)
    for lines in (3, 5, 11, 21):
        fx, fy = line_factors(lines, full)
        for _ in range(20):
            r = rng.uniform(0.2, 1.0, lines)
            x = [float(v) for v in r * np.array(fx)]
            y = [float(v) for v in r * np.array(fy)]
            cx, cy = (ctypes.c_double * lines)(*x), (ctypes.c_double * lines)(*y)
            cfx, cfy = (ctypes.c_double * lines)(*fx), (ctypes.c_double * lines)(*fy)
            want = f(lines, cx, cy, cfx, cfy, int(full))
            got = trim_aperture(lines, x, y, fx, fy, full)
            assert got == want and x == list(cx) and y == list(cy)
