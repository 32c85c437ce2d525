"""SDDS output in elegant's phase-space and loss layouts (CPU)."""
import numpy as np
import pytest

from elegant_b200 import workloads as w
from elegant_b200.sdds import read_sdds, write_losses, write_phase_space
from elegant_b200.track import TrackResult


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
