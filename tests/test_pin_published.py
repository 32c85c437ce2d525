"""The numerics the reference takes from its un-vendored SDDS toolkit, checked
against independent published implementations (scipy), on the CPU.

- Savitzky-Golay smoothing and first derivative (the toolkit's
  SavitzkyGolaySmooth, called by CSRCSBEND at csbend.c:2570, :2580 and by the
  Stupakov CSRDRIFT at :3958, :3973): the project's filter (b2e_sg.h, linked
  into the reference build, the restatement and the kernels) against
  scipy.signal.savgol_filter with mode='interp' -- a degree-`order` least-
  squares fit over 2*half+1 points, and at either end the fit over the first
  or last window evaluated at the point's own offset, which is the edge rule
  b2e_sg.h defines.
- SolveForPhiStupakov's roots (csbend.c:4169-4202, zeroNewton/zeroInterp of
  the toolkit): the project's root finders (b2e_roots.h) against
  scipy.optimize.brentq on the same equation, within the reference's own
  acceptance test |24 ds - f(phi)| < 24 ds / 1e4.
"""
import ctypes
import os

import numpy as np
import pytest

scipy_signal = pytest.importorskip("scipy.signal")
scipy_optimize = pytest.importorskip("scipy.optimize")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    path = os.path.join(ROOT, "oracle", "_build", "libb2e_oracle.so")
    lib = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.b2e_oracle_sg_apply.restype = ctypes.c_long
    lib.b2e_oracle_sg_apply.argtypes = [dp, ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_long]
    lib.b2e_oracle_stupakov_phi.restype = ctypes.c_double
    lib.b2e_oracle_stupakov_phi.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
    return lib


def project_sg(lib, data, order, half, deriv):
    out = np.ascontiguousarray(data, dtype=np.float64).copy()
    rc = lib.b2e_oracle_sg_apply(out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size, order, half, half,
                                 deriv)
    assert rc == 1
    return out


def profiles(rng, n):
    """A binned line density with shot noise (the CSR histogram) and a rough
    signal with sharp edges."""
    z = np.linspace(-4, 4, n)
    dens = rng.poisson(2000 * np.exp(-z * z / 2) + 5).astype(float)
    rough = np.where(np.abs(z) < 1.5, 1.0, 0.0) + 0.1 * rng.standard_normal(n)
    return [dens, rough]


@pytest.mark.parametrize("order", [1, 2, 3, 4])
@pytest.mark.parametrize("half", [1, 2, 3, 5, 8, 16])
@pytest.mark.parametrize("deriv", [0, 1])
def test_savitzky_golay_against_scipy(lib, order, half, deriv):
    width = 2 * half + 1
    if order >= width:
        pytest.skip("degree needs a wider window")
    rng = np.random.default_rng(order * 100 + half * 10 + deriv)
    for n in (600, 97, width + 1):
        for data in profiles(rng, n):
            ours = project_sg(lib, data, order, half, deriv)
            ref = scipy_signal.savgol_filter(data, width, order, deriv=deriv, mode="interp")
            scale = np.abs(data).max()
            err = np.abs(ours - ref).max() / scale
            assert err < 1e-11, (n, err)


def test_savitzky_golay_edges_are_the_window_fit(lib):
    """The first and last `half` points take the fit over the end windows: a
    polynomial of the filter's degree passes through unchanged everywhere,
    edges included, and so does its derivative."""
    n, half, order = 40, 4, 3
    i = np.arange(n, dtype=float)
    poly = 0.5 - 0.25 * i + 0.01 * i ** 2 - 3e-4 * i ** 3
    dpoly = -0.25 + 0.02 * i - 9e-4 * i ** 2
    np.testing.assert_allclose(project_sg(lib, poly, order, half, 0), poly, rtol=0, atol=1e-11)
    np.testing.assert_allclose(project_sg(lib, poly, order, half, 1), dpoly, rtol=0, atol=1e-11)


def _f(phi, x):
    return phi ** 3 * (phi + 4 * x) / (phi + x)


def test_stupakov_phi_against_brentq(lib):
    """Over the (x, ds, phim) range a CSRDRIFT meets: where the equation has a
    root in [0, phim] both find it and ours passes the reference's acceptance
    test and lies within the root's tolerance band; where it has none, ours
    reports -1."""
    rng = np.random.default_rng(7)
    solved = none = 0
    phi_last = ctypes.c_double(-1.0)
    for _ in range(3000):
        phim = 10 ** rng.uniform(-3, -0.5)
        x = 10 ** rng.uniform(-4, 1) * phim
        ds = _f(phim, x) / 24 * 10 ** rng.uniform(-6, 0.2)
        ours = lib.b2e_oracle_stupakov_phi(x, ds, phim, ctypes.byref(phi_last))
        target = 24 * ds
        if _f(phim, x) < target * (1 - 1e-4):  # no root in [0, phim]
            assert ours == -1 or abs(target - _f(ours, x)) < target / 1e4
            none += 1
            continue
        if ours == phim and abs(target - _f(phim, x)) < target / 1e4:
            solved += 1
            continue
        root = scipy_optimize.brentq(lambda p: _f(p, x) - target, 0.0, phim, xtol=1e-300, rtol=1e-15)
        assert 0 <= ours <= phim
        assert abs(target - _f(ours, x)) < target / 1e4
        slope = (_f(root * (1 + 1e-7), x) - _f(root, x)) / (root * 1e-7)
        assert abs(ours - root) <= 1.01 * (target / 1e4) / slope + 1e-15 * root
        solved += 1
    assert solved > 1000 and none > 100
