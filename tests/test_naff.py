"""The NAFF method (numpy statement, tests/naff_reference.py) on signals of
known frequency, and the frequency-map grid (no GPU)."""
import math

import numpy as np
import pytest

from elegant_b200.frequency_map import grid
from naff_reference import adjust_tune_half_plane, naff


@pytest.mark.parametrize("n", [256, 1000, 1024])
def test_naff_recovers_known_frequencies(n):
    rng = np.random.default_rng(n)
    tol = {256: 2e-6, 1000: 3e-8, 1024: 3e-8}[n]
    for _ in range(20):
        nu = rng.uniform(0.05, 0.45)
        nu2 = 0.05 + (nu + 0.15) % 0.4  # a weaker line at least 0.1 away
        amp, ph = rng.uniform(0.5, 2), rng.uniform(-3, 3)
        t = np.arange(n)
        x = amp * np.cos(2 * np.pi * nu * t + ph) + 0.05 * amp * np.cos(2 * np.pi * nu2 * t) + 0.3
        f, a, p = naff(x)
        assert abs(f - nu) < tol, (f, nu)
        assert abs(a / amp - 1) < 1e3 * tol
        assert abs(math.remainder(p - ph, 2 * math.pi)) < 1e4 * tol
    # a clean line is found to near machine precision
    t = np.arange(n)
    f, _, _ = naff(np.cos(2 * np.pi * 0.2137 * t))
    assert abs(f - 0.2137) < 1e-10


def test_half_plane_from_the_slope_phase():
    """x = cos(2 pi nu t), x' = -sin: the tune is nu; with the roles
    reversed (a tune above one half) it is 1 - nu."""
    t = np.arange(512)
    nu = 0.23
    fx, _, px = naff(np.cos(2 * np.pi * nu * t))
    fxp, _, pxp = naff(-np.sin(2 * np.pi * nu * t))
    assert abs(adjust_tune_half_plane(fx, px, pxp) - nu) < 1e-9
    fxp, _, pxp = naff(np.sin(2 * np.pi * nu * t))
    assert abs(adjust_tune_half_plane(fx, px, pxp) - (1 - nu)) < 1e-9


def test_grid_order_and_spacing():
    pts = grid(-0.01, 0.01, 1e-6, 0.005, 3, 2, delta_min=-0.01, delta_max=0.01, ndelta=2)
    assert len(pts) == 12
    assert pts[0] == (-0.01, 1e-6, -0.01) and pts[1][1] == 1e-6 + (0.005 - 1e-6)
    assert pts[2][0] == -0.01 + 1 * ((0.01 - -0.01) / 2)
    q = grid(0.0, 0.01, 0.0, 0.01, 4, 4, quadratic_spacing=True)
    assert q[0][0] == 0.0 + 0.01 * math.sqrt(1 / 4) and q[-1][0] == 0.01
