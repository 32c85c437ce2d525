"""Pins the CPU oracles (no GPU needed).

- the C restatement (oracle/b2e_oracle.c) reproduces elegant's own tracking
  code (oracle/_ref, compiled from the reference sources) row for row, bit for
  bit, in both maths modes, including lost-particle bookkeeping;
- the shared elementary functions agree with glibc's to within the ring's
  intrinsic sensitivity: after 10 turns within 1e-10 relative, and after
  many turns no further apart than a one-ulp perturbation of the initial
  coordinates grows by itself under the reference with glibc.
"""
import math

import numpy as np
import pytest

from elegant_b200 import workloads as w
from elegant_b200.beam import Beam
from reforacle import PortOracle, RefOracle, by_id

P0 = w.ring_p_central()


def lossy_beam(n=200, seed=3):
    rng = np.random.default_rng(seed)
    c = np.zeros((n, 6))
    c[:, 0] = rng.uniform(-0.022, 0.022, n)
    c[:, 1] = rng.uniform(-3e-3, 3e-3, n)
    c[:, 2] = rng.uniform(-0.015, 0.015, n)
    c[:, 3] = rng.uniform(-2e-3, 2e-3, n)
    c[:, 4] = rng.normal(0, 5e-3, n)
    c[:, 5] = rng.uniform(-0.03, 0.03, n)
    return Beam(c, np.arange(1, n + 1))


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("case", ["matched", "lossy"])
def test_port_reproduces_reference(math, case):
    lat = w.fodo_ring()
    beam = w.ring_beam(120, seed=7) if case == "matched" else lossy_beam()
    turns = 25
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, turns)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, turns)
    assert n1 == n2 and e1 == e2
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])  # survivors, same array order
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])    # every (id, lossPass)
    if case == "lossy":
        assert n1 < beam.n


def test_port_reproduces_reference_misaligned():
    from elegant_b200 import Element, Lattice
    lat = w.fodo_ring()
    els = []
    for i, e in enumerate(lat.elements):
        if e.type == "KQUAD":
            e = Element(e.name, e.type, dict(e.params, DX=2e-4, DY=-1e-4 * (i % 2), FSE=1e-3))
        if e.type == "KSEXT":
            e = Element(e.name, e.type, dict(e.params, TILT=0.02, DZ=1e-3))
        els.append(e)
    lat2 = Lattice(els)
    beam = w.ring_beam(80, seed=2)
    r1, n1, _, _ = RefOracle("b2e").track(lat2, beam.coords, beam.ids, P0, 15)
    r2, n2, _ = PortOracle("b2e").track(lat2, beam.coords, beam.ids, P0, 15)
    assert n1 == n2 and np.array_equal(r1[:n1, :7], r2[:n2, :7])


def _rel(a, b):
    scale = np.maximum(np.abs(a), a.std(axis=0) + 1e-300)
    return (np.abs(a - b) / scale).max(axis=0)


def test_shared_math_within_1e10_after_10_turns():
    lat = w.fodo_ring()
    beam = w.ring_beam(100, seed=5)
    a = by_id(RefOracle("libm").track(lat, beam.coords, beam.ids, P0, 10)[0])
    b = by_id(RefOracle("b2e").track(lat, beam.coords, beam.ids, P0, 10)[0])
    assert np.array_equal(a[2], b[2])
    assert _rel(a[0], b[0]).max() <= 1e-10


def test_shared_math_within_one_ulp_envelope_after_200_turns():
    """The ring amplifies a one-ulp change of x by many orders of magnitude
    over hundreds of turns; the libm/shared-maths difference must stay inside
    (a small multiple of) that intrinsic envelope."""
    lat = w.fodo_ring()
    beam = w.ring_beam(60, seed=5)
    turns = 200
    ref = RefOracle("libm")
    a = by_id(ref.track(lat, beam.coords, beam.ids, P0, turns)[0])
    b = by_id(RefOracle("b2e").track(lat, beam.coords, beam.ids, P0, turns)[0])
    pert = beam.copy()
    pert.coords[:, 0] = np.nextafter(pert.coords[:, 0], np.inf)
    c = by_id(ref.track(lat, pert.coords, pert.ids, P0, turns)[0])
    assert np.array_equal(a[2], b[2])
    envelope = _rel(a[0], c[0])
    diff = _rel(a[0], b[0])
    assert (diff <= 20 * envelope + 1e-15).all(), (diff, envelope)


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("variant", ["default", "steady_plain", "no_sg", "igf"])
def test_port_reproduces_reference_csr(math, variant):
    """CSRCSBEND + CSRDRIFT: the restatement reproduces the reference's final
    rows and every per-kick wake (captured through the reference's own
    OUTPUT_FILE writer) bit for bit."""
    from elegant_b200 import Element, Lattice
    lat = w.chicane(bins=120, n_kicks=4, sg_halfwidth=0 if variant == "no_sg" else 2)
    if variant == "steady_plain":
        els = []
        for i, e in enumerate(lat.elements):
            if e.type == "CSRCSBEND":
                e = Element(e.name, e.type, dict(e.params, **({"STEADY_STATE": 1} if i % 2 else
                                                              {"TRAPAZOID_INTEGRATION": 0})))
            if e.type == "CSRDRIFT":
                e = Element(e.name, e.type, dict(e.params, N_KICKS=3))
            els.append(e)
        lat = Lattice(els)
    if variant == "igf":
        lat = Lattice([Element(e.name, e.type, dict(e.params, STEADY_STATE=1, IGF=1)) if e.type == "CSRCSBEND" else e
                       for e in lat.elements])
    beam = w.chicane_beam(6000, seed=11)
    p0 = 1000 / 0.51099895
    r1, n1, e1, w1 = RefOracle(math).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    r2, n2, e2, w2 = PortOracle(math).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    assert n1 == n2 and w1.size == w2.size > 0
    assert np.array_equal(w1, w2)
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])


def test_igf_shared_math_close_to_libm():
    """The IGF wake through the shared pow/log against glibc's: final
    coordinates of the chicane within 1e-10 relative."""
    from elegant_b200 import Element, Lattice
    lat = w.chicane(bins=120, n_kicks=4)
    lat = Lattice([Element(e.name, e.type, dict(e.params, STEADY_STATE=1, IGF=1)) if e.type == "CSRCSBEND" else e
                   for e in lat.elements])
    beam = w.chicane_beam(6000, seed=12)
    p0 = 1000 / 0.51099895
    a = by_id(RefOracle("libm").track(lat, beam.coords, beam.ids, p0, 1)[0])
    b = by_id(RefOracle("b2e").track(lat, beam.coords, beam.ids, p0, 1)[0])
    assert np.array_equal(a[2], b[2])
    assert _rel(a[0], b[0]).max() <= 1e-10


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("case", ["default", "fine_bins_3kicks", "dz", "no_sg", "steady_plain", "gap", "gap_mode0",
                                  "ring_2p", "ring_mode0_2p"])
def test_port_reproduces_reference_csrdrift_modes(math, case):
    """CSRDRIFT in Stupakov mode (phi solutions, cases C and D), a CSRDRIFT
    that starts behind the dipole's wake, and one ahead of the first dipole
    on a second pass: the restatement reproduces elegant's own code bit for
    bit.  Each reference run loads a fresh copy of the library, so
    SolveForPhiStupakov's carried start value begins as in a new process."""
    from csr_cases import stupakov_cases
    lat = stupakov_cases()[case]
    passes = 2 if case.endswith("2p") else 1
    beam = w.chicane_beam(5000, seed=21)
    p0 = 1000 / 0.51099895
    r1, n1, _, w1 = RefOracle(math, private=True).track(lat, beam.coords, beam.ids, p0, passes, capture_wakes=True)
    r2, n2, _, w2 = PortOracle(math).track(lat, beam.coords, beam.ids, p0, passes, capture_wakes=True)
    assert n1 == n2 and w1.size == w2.size > 0
    assert np.array_equal(w1, w2)
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])


def test_stupakov_drift_differs_from_mode_0():
    """The Stupakov wake is a different model from the mode-0 propagated
    dipole wake: the final momenta differ (by far more than rounding)."""
    p0 = 1000 / 0.51099895
    beam = w.chicane_beam(5000, seed=22)
    a = by_id(RefOracle("b2e").track(w.chicane(bins=200, n_kicks=4), beam.coords, beam.ids, p0, 1)[0])[0]
    b = by_id(RefOracle("b2e", private=True).track(w.chicane(bins=200, n_kicks=4, stupakov=True), beam.coords,
                                                   beam.ids, p0, 1)[0])[0]
    assert np.abs(a[:, 5] - b[:, 5]).max() > 1e-3 * np.abs(a[:, 5]).max()


def test_stupakov_phi_solver():
    """The root finders behind SolveForPhiStupakov: every solution satisfies
    24 ds = phi^3 (phi + 4x)/(phi + x) to the reference's 1e-4 relative
    tolerance, x = 0 gives the cube root, a start far from the root still
    converges (the scanning fallback), and ds beyond phim has no solution."""
    import ctypes
    from reforacle import PortOracle as _P
    lib = _P("b2e").lib
    f = lib.b2e_oracle_stupakov_phi
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double] * 3 + [ctypes.POINTER(ctypes.c_double)]

    def fn(p, x):
        return p * p * p * (p + 4 * x) / (p + x)
    for x in (0.0, 1e-3, 0.1, 0.5, 3.0):
        last = ctypes.c_double(-1)
        for ds in np.geomspace(1e-9, 4e-6, 25):
            phi = f(x, ds, 0.05, ctypes.byref(last))
            assert 0 < phi <= 0.05
            assert abs(24 * ds - fn(phi, x)) <= 24 * ds / 1e4
            if x == 0.0:
                assert abs(phi - (24 * ds) ** (1 / 3)) < 1e-4 * phi
    last = ctypes.c_double(1e-12)
    phi = f(0.3, 1e-7, 0.05, ctypes.byref(last))
    assert abs(24e-7 - fn(phi, 0.3)) <= 24e-7 / 1e4
    last = ctypes.c_double(-1)
    assert f(0.01, 1.0, 0.05, ctypes.byref(last)) == -1
    assert f(0.01, 0.0, 0.05, ctypes.byref(last)) == 0
    assert f(0.01, -1e-9, 0.05, ctypes.byref(last)) == -1


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("case", ["low_pass", "high_pass", "both_odd_bins", "round_trip_only", "no_clip_stupakov"])
def test_port_reproduces_reference_csr_filters(math, case):
    """The histogram filters (applyLHPassFilters through the shared real
    transform): restatement and elegant's own code agree bit for bit."""
    from csr_cases import filter_cases
    lat = filter_cases()[case]
    beam = w.chicane_beam(5000, seed=23)
    p0 = 1000 / 0.51099895
    r1, n1, _, w1 = RefOracle(math, private=True).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    r2, n2, _, w2 = PortOracle(math).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    assert n1 == n2 and w1.size == w2.size > 0
    assert np.array_equal(w1, w2)
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])


def _numpy_lh(h, start_hp, end_hp, start_lp, end_lp, clip):
    """applyLHPassFilters with numpy's FFT (an independent transform)."""
    n = h.size
    freq = n // 2 + 1
    X = np.fft.rfft(h)
    scale = np.ones(freq)
    end_lp, end_hp = max(end_lp, start_lp), max(end_hp, start_hp)
    if start_lp > 0:
        i1 = min(max(int(start_lp * freq), 0), freq - 1)
        i2 = min(max(int(end_lp * freq), 0), freq - 1)
        d = 0 if i1 == i2 else 1.0 / (i2 - i1)
        f = 1.0
        for i in range(i1, i2 + 1):
            scale[i] *= f
            f = max(f - d, 0)
        scale[i2 + 1:] = 0
    if start_hp > 0:
        i1 = min(max(int(start_hp * freq), 0), freq - 1)
        i2 = min(max(int(end_hp * freq), 0), freq - 1)
        d = 0 if i1 == i2 else 1.0 / (i2 - i1)
        scale[:i1] = 0
        f = 0.0
        for i in range(i1, i2 + 1):
            scale[i] *= f
            f = min(f + d, 1)
    y = np.fft.irfft(X * scale, n)
    if clip:
        y = np.where(y < 0, 0, y)
        y *= h.sum() / y.sum()
    return y


@pytest.mark.parametrize("n", [8, 9, 120, 151, 600, 1024])
@pytest.mark.parametrize("cut", [(-1, -1, 0.2, 0.4), (0.05, 0.1, -1, -1), (0.02, 0.02, 0.3, 0.6), (0.0, -1, -1, -1)])
def test_histogram_filter_transform_against_numpy(n, cut):
    """The project's real transform (b2e_fft.h, any n) and the filter ramps
    agree with numpy's FFT to rounding, with and without clipping."""
    import ctypes
    lib = PortOracle("b2e").lib
    f = lib.b2e_oracle_lh_pass_filters
    f.restype = ctypes.c_long
    f.argtypes = [ctypes.c_void_p, ctypes.c_long] + [ctypes.c_double] * 4 + [ctypes.c_int]
    rng = np.random.default_rng(n)
    x = np.arange(n)
    h = np.round(50 * np.exp(-0.5 * ((x - n / 2) / (n / 8)) ** 2) + rng.poisson(5, n)).astype(float)
    for clip in (0, 1):
        ours = h.copy()
        f(ours.ctypes.data, n, *cut, clip)
        ref = _numpy_lh(h, *cut, clip)
        assert np.allclose(ours, ref, rtol=1e-11, atol=1e-11 * h.max()), (clip, np.abs(ours - ref).max())


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_with_exact_drifts(math):
    """EDRIFT (exactDrift, csbend.c:3767-3790) in the ring, with losses."""
    from elegant_b200 import Element, Lattice
    lat = Lattice([Element(e.name, "EDRIFT", {"L": e.params["L"]}) if e.name == "D2" else e
                   for e in w.fodo_ring().elements])
    beam = lossy_beam(150, seed=13)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])


def _ring_with_cavity(**rf):
    from elegant_b200 import Element, Lattice
    return Lattice([Element(e.name, e.type, dict(e.params, **rf)) if e.type == "RFCA" else e
                    for e in w.fodo_ring().elements])


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("rf", [{"L": 0.5, "N_KICKS": 0}, {"L": 0.5, "N_KICKS": 5}, {"VOLT": 0.0},
                                {"L": 0.4, "VOLT": 0.0}], ids=["matrix", "kicks", "no_volt", "no_volt_drift"])
def test_port_reproduces_reference_rf_cavity_with_length(math, rf):
    """RFCA with a length: the matrix method (N_KICKS = 0, simple_rfca.c:823-945),
    drift-kick-drift sections (N_KICKS > 0, :569-700), and zero voltage
    (:380-392), with losses."""
    lat = _ring_with_cavity(**rf)
    beam = lossy_beam(160, seed=17)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])


def _ring_with_bend_errors():
    """The ring with its dipoles rolled by ETILT: one alone, one with a TILT
    as well, one folded into a negative angle (tilt + PI), one with a quarter
    turn of TILT (the exact-rotation branch)."""
    from elegant_b200 import Element, Lattice
    errs = [{"ETILT": 2e-3}, {"ETILT": -1.5e-3, "TILT": 0.05, "DX": 1e-4},
            {"ETILT": 1e-3, "E1": 0.1, "E2": 0.08}, {"ETILT": 5e-4, "DZ": 2e-4}]
    els, k = [], 0
    for e in w.fodo_ring().elements:
        if e.type == "CSBEND":
            e = Element(e.name + str(k), e.type, dict(e.params, **errs[k % len(errs)]))
            k += 1
        els.append(e)
    return Lattice(els)


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_rolled_bends(math):
    """CSBEND ETILT: the exit-face offsets of computeEtiltCentroidOffset
    (csbend.c:4723-4769) added after the exit rotation (:1359-1364), with
    losses."""
    lat = _ring_with_bend_errors()
    beam = lossy_beam(150, seed=19)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    # the roll moves the orbit: the same beam ends elsewhere without it
    r0, n0, _, _ = RefOracle(math).track(w.fodo_ring(), beam.coords, beam.ids, P0, 20)
    assert not np.array_equal(r0[:min(n0, n1), :4], r1[:min(n0, n1), :4])


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_csr_rolled_bends(math):
    """CSRCSBEND ETILT: the offsets at the CSR exit (csbend.c:2942-2952),
    negative-angle dipoles included."""
    from elegant_b200 import Element, Lattice
    lat = w.chicane(bins=120, n_kicks=4, sg_halfwidth=2)
    lat = Lattice([Element(e.name, e.type, dict(e.params, ETILT=1e-3 * (1 + i % 3), TILT=0.02 * (i % 2)))
                   if e.type == "CSRCSBEND" else e for i, e in enumerate(lat.elements)])
    beam = w.chicane_beam(5000, seed=23)
    p0 = 1000 / 0.51099895
    r1, n1, e1, w1 = RefOracle(math).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    r2, n2, e2, w2 = PortOracle(math).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    assert n1 == n2 and w1.size == w2.size > 0
    assert np.array_equal(w1, w2)
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_second_order_edges(math):
    """EDGE_ORDER=2 (apply_edge_effects, csbend.c:4266-4307) on ring dipoles
    with edge angles and a fringe integral, with losses; and on CSRCSBENDs."""
    from elegant_b200 import Element, Lattice
    els, k = [], 0
    for e in w.fodo_ring().elements:
        if e.type == "CSBEND":
            e = Element(e.name + str(k), e.type, dict(e.params, EDGE_ORDER=2, E1=0.12 - 0.05 * (k % 3),
                                                      E2=0.09 * (k % 2), HGAP=0.02, FINT=0.5))
            k += 1
        els.append(e)
    beam = lossy_beam(150, seed=37)
    r1, n1, e1, _ = RefOracle(math).track(Lattice(els), beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(Lattice(els), beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    lat = w.chicane(bins=120, n_kicks=4, sg_halfwidth=2)
    lat = Lattice([Element(e.name, e.type, dict(e.params, EDGE_ORDER=2, E1=0.02, E2=0.03, HGAP=0.01, FINT=0.4))
                   if e.type == "CSRCSBEND" else e for e in lat.elements])
    beam = w.chicane_beam(5000, seed=41)
    p0 = 1000 / 0.51099895
    r1, n1, _, w1 = RefOracle(math).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    r2, n2, _, w2 = PortOracle(math).track(lat, beam.coords, beam.ids, p0, 1, capture_wakes=True)
    assert n1 == n2 and np.array_equal(w1, w2)
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])


def _ring_with_gradient_dipoles(base=None, negative=False):
    """The ring with combined-function dipoles: K1 and K2 in the bends
    (computeCSBENDFields' expansion), one of them NONLINEAR=0, one with
    second-order edges (the edge map's n = -b1/h), one with an FSE;
    negative=True folds every other dipole into a negative angle (a TILT of
    PI)."""
    from elegant_b200 import Element, Lattice
    errs = [{"K1": 0.15, "K2": 2.0}, {"K1": -0.2, "NONLINEAR": 0}, {"K2": -3.0, "EDGE_ORDER": 2, "E1": 0.1},
            {"K1": 0.1, "K2": 1.0, "FSE": 1e-3}]
    els, k = [], 0
    for e in (base or w.fodo_ring()).elements:
        if e.type == "CSBEND":
            params = dict(e.params, **errs[k % len(errs)])
            if negative and k % 2:
                params.update(ANGLE=-params["ANGLE"], TILT=math.pi)
            e = Element(e.name + str(k), e.type, params)
            k += 1
        els.append(e)
    return Lattice(els)


def _mixed_beam(seed):
    return Beam(np.concatenate([w.ring_beam(100, seed=seed).coords, lossy_beam(100, seed=seed + 1).coords]),
                np.arange(1, 201))


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("case", ["plain", "negative_angle", "synch_rad"])
def test_port_reproduces_reference_gradient_dipoles(math, case):
    """CSBEND with K1/K2 field terms (csbend.c:101-150, :186-663, the kick
    :1591-1601 and the radiation :1603-1622, :1211-1276), with losses."""
    base = w.radiating_ring(edge_angle=0.05) if case == "synch_rad" else None
    lat = _ring_with_gradient_dipoles(base, negative=case == "negative_angle")
    beam = _mixed_beam(47)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and 0 < n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    r0, n0, _, _ = RefOracle(math).track(base or w.fodo_ring(), beam.coords, beam.ids, P0, 20)
    assert not np.array_equal(r0[:min(n0, n1), :4], r1[:min(n0, n1), :4])


def _ring_with_watches():
    from elegant_b200 import Element, Lattice
    els = list(w.fodo_ring().elements)
    els.insert(3, Element("W1", "WATCH", {"FILENAME": "%s.w1", "INTERVAL": 3, "START_PASS": 1}))
    els.insert(30, Element("W2", "WATCH", {"FILENAME": "%s.w2", "END_PASS": 4}))
    els.append(Element("W3", "WATCH", {"FILENAME": "%s.w3", "DISABLE": 1}))
    return Lattice(els)


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_with_watches(math):
    """WATCH elements change no coordinate and no loss (do_tracking.c:1585-1635,
    NO_APERTURE); the reference's WATCH rows (what dump_watch_particles is
    handed) are the particles alive there on the passes it writes
    (sdds_support.c:738-741)."""
    lat = _ring_with_watches()
    beam = lossy_beam(150, seed=53)
    ref = RefOracle(math)
    ref.set_watch(100000)
    r1, n1, e1, _ = ref.track(lat, beam.coords, beam.ids, P0, 12)
    rows = ref.watch_rows()
    ref.set_watch(0)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 12)
    r0, n0, e0, _ = RefOracle(math).track(w.fodo_ring(), beam.coords, beam.ids, P0, 12)
    assert n1 == n2 == n0 and e1 == e2 == e0 and n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7]) and np.array_equal(r1[:, 6:8], r0[:, 6:8])
    w1, w2 = lat.index("W1")[0], lat.index("W2")[0]
    assert sorted(set(rows[rows[:, 0] == w1, 1])) == [1, 4, 7, 10]
    assert sorted(set(rows[rows[:, 0] == w2, 1])) == [0, 1, 2, 3, 4]
    assert not (rows[:, 0] == lat.index("W3")[0]).any()
    # the particles at W2 on pass 0 are the beam less those lost before it
    first = rows[(rows[:, 0] == w2) & (rows[:, 1] == 0)]
    lost_early = {int(i) for i, lp in zip(r1[:, 6], r1[:, 7]) if lp == 0}
    assert set(first[:, 2].astype(int)) <= set(beam.ids) - (lost_early - set(first[:, 2].astype(int)))


def _ring_with_steering(base=None):
    """The ring with correctors in its multipoles (multipole.c:785-786,
    :848-849, :1190-1191, :1281-1284): HKICK/VKICK with calibrations on the
    quadrupoles and sextupoles, one quadrupole tilted, one strength from a
    pole-tip field and bore (:771-773, :834-837), and parameters the tracking
    ignores (HSTEERING, PITCH under MALIGN_METHOD 0)."""
    from elegant_b200 import Element, Lattice
    els, k = [], 0
    for e in (base or w.fodo_ring()).elements:
        if e.type in ("KQUAD", "KSEXT"):
            extra = [{"HKICK": 2e-4, "HSTEERING": 1}, {"VKICK": -1.5e-4, "VCALIBRATION": 1.1},
                     {"HKICK": -1e-4, "VKICK": 5e-5, "HCALIBRATION": 0.9, "TILT": 0.01, "PITCH": 1e-3},
                     {}][k % 4]
            if e.type == "KQUAD" and k == 5:
                extra = {"BORE": 0.02, "B": 0.2 * e.params["K1"] / 1.2, "FSE": 1e-3}
            if e.type == "KSEXT" and k == 7:
                extra = {"BORE": 0.03, "B": 0.01, "HKICK": 1e-4}
            e = Element(e.name + str(k), e.type, dict(e.params, **extra))
            k += 1
        els.append(e)
    return Lattice(els)


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("case", ["plain", "synch_rad"])
def test_port_reproduces_reference_steering(math, case):
    """KQUAD/KSEXT HKICK, VKICK, calibrations and pole-tip strengths, with
    the steering kicks inside the radiation's F2 when SYNCH_RAD is on."""
    base = None
    if case == "synch_rad":
        from elegant_b200 import Element, Lattice
        base = Lattice([Element(e.name, e.type, dict(e.params, SYNCH_RAD=1)) if e.type in ("KQUAD", "KSEXT") else e
                        for e in w.fodo_ring().elements])
    lat = _ring_with_steering(base)
    beam = _mixed_beam(61)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and 0 < n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    r0, n0, _, _ = RefOracle(math).track(base or w.fodo_ring(), beam.coords, beam.ids, P0, 20)
    assert not np.array_equal(r0[:min(n0, n1), :4], r1[:min(n0, n1), :4])


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("mode", ["light", "pmax", "tm"])
def test_port_reproduces_reference_fiducial_modes(math, mode):
    """RFCA FIDUCIAL (findFiducialTime, simple_rfca.c:62-257): light (zEnd - L
    + sOffset over c), pmaximum (the highest-delta particle after the first),
    tmean by an abbreviation; a zero-length cavity mid-ring and one with a
    length, with losses."""
    from elegant_b200 import Element, Lattice
    base = list(w.fodo_ring().elements)
    rf = next(e for e in base if e.type == "RFCA")
    els = [e for e in base if e.type != "RFCA"]
    els.insert(20, Element("RF1", "RFCA", dict(rf.params, FIDUCIAL=mode)))
    els.append(Element("RF2", "RFCA", dict(rf.params, L=0.4, N_KICKS=4, VOLT=5e5, FIDUCIAL=mode)))
    lat = Lattice(els)
    beam = _mixed_beam(71)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 15)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 15)
    assert n1 == n2 and e1 == e2 and 0 < n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    if mode != "tm":
        r0, n0, _, _ = RefOracle(math).track(Lattice([Element(e.name, e.type, dict(e.params, FIDUCIAL="tmean"))
                                                      if e.type == "RFCA" else e for e in lat.elements]),
                                             beam.coords, beam.ids, P0, 15)
        assert not np.array_equal(r0[:min(n0, n1), :6], r1[:min(n0, n1), :6])


def test_fiducial_pmaximum_without_a_particle_fails_like_the_reference():
    """pmaximum takes only a particle after the first with a higher delta
    (simple_rfca.c:126-147): a beam whose first particle is highest stops the
    reference, and the oracle too."""
    from elegant_b200 import Element, Lattice
    lat = Lattice([Element("D", "DRIF", {"L": 1.0}),
                   Element("RF", "RFCA", {"VOLT": 1e6, "FREQ": 5e8, "FIDUCIAL": "pmaximum"})])
    coords = np.zeros((3, 6))
    coords[:, 5] = [1e-3, 0.0, -1e-3]
    with pytest.raises(RuntimeError, match="fiducial"):
        RefOracle("b2e").track(lat, coords, np.arange(1, 4), P0, 2)
    with pytest.raises(RuntimeError, match="fiducial"):
        PortOracle("b2e").track(lat, coords, np.arange(1, 4), P0, 2)
    coords[:, 5] = [0.0, 1e-3, 1e-3]
    RefOracle("b2e").track(lat, coords, np.arange(1, 4), P0, 2)


def test_fiducial_mode_first_is_rejected():
    from elegant_b200 import Element
    from elegant_b200.lattice import LatticeError
    with pytest.raises(LatticeError, match="first"):
        Element("RF", "RFCA", {"VOLT": 1e6, "FIDUCIAL": "first"})
    with pytest.raises(LatticeError, match="invalid fiducial"):
        Element("RF", "RFCA", {"VOLT": 1e6, "FIDUCIAL": "median"})
    assert Element("RF", "RFCA", {"FIDUCIAL": "p"}).params["FIDUCIAL"] == 2


def _ring_with_bend_steering(negative=False):
    """Bends with XKICK (the field term b0 = XKICK/ANGLE, csbend.c:867) and
    YKICK (the skew term c0 = YKICK/ANGLE, :868, which makes the reference
    sum every term of the expansion), alone or with K1/K2; every other bend
    folded to a negative angle when asked."""
    from elegant_b200 import Element, Lattice
    errs = [{"XKICK": 2e-4}, {"XKICK": -1e-4, "K1": 0.1}, {"YKICK": 1.5e-4}, {"XKICK": 5e-5, "NONLINEAR": 0},
            {"YKICK": -1e-4, "K2": 0.5}, {}]
    els, k = [], 0
    for e in w.fodo_ring().elements:
        if e.type == "CSBEND":
            params = dict(e.params, **errs[k % len(errs)])
            if negative and k % 2:
                params.update(ANGLE=-params["ANGLE"], TILT=math.pi)
            e = Element(e.name + str(k), e.type, params)
            k += 1
        els.append(e)
    return Lattice(els)


@pytest.mark.parametrize("math", ["libm", "b2e"])
@pytest.mark.parametrize("negative", [False, True])
def test_port_reproduces_reference_bend_steering(math, negative):
    lat = _ring_with_bend_steering(negative)
    beam = _mixed_beam(81)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and 0 < n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    r0, n0, _, _ = RefOracle(math).track(w.fodo_ring(), beam.coords, beam.ids, P0, 20)
    assert not np.array_equal(r0[:min(n0, n1), :4], r1[:min(n0, n1), :4])


def _ring_with_quad_fringes():
    """Quadrupoles with fringe fields (quadFringe, fringe.c:24-175): linear
    (EDGE_EFFECTS 1) and linear + third order (2) with fringe integrals, one
    without the linear part, one with a nonlinear factor, one with the
    entrance only, one with a negative (off) value; and effective lengths
    (LEFFECTIVE: exact end drifts, multipole.c:766-770, :1028-1030), one
    radiating."""
    from elegant_b200 import Element, Lattice
    fi = {"I0P": 0.02, "I1P": 1e-3, "I2P": 2e-5, "I3P": 1e-6, "LAMBDA2P": 3e-6,
          "I0M": 0.025, "I1M": -1e-3, "I2M": 1e-5, "I3M": -2e-6, "LAMBDA2M": 1e-6}
    variants = [dict(fi, EDGE1_EFFECTS=1, EDGE2_EFFECTS=1), dict(fi, EDGE1_EFFECTS=2, EDGE2_EFFECTS=2),
                dict(fi, EDGE1_EFFECTS=2, EDGE2_EFFECTS=2, EDGE1_LINEAR=0, EDGE2_LINEAR=0),
                dict(fi, EDGE1_EFFECTS=2, EDGE2_EFFECTS=2, EDGE2_NONLINEAR_FACTOR=0.5, DX=1e-4, TILT=0.01),
                {"EDGE1_EFFECTS": 2, "LEFFECTIVE": 0.26}, {"EDGE1_EFFECTS": -1, "EDGE2_EFFECTS": 2},
                {"LEFFECTIVE": 0.27, "SYNCH_RAD": 1}]
    els, k = [], 0
    for e in w.fodo_ring().elements:
        if e.type == "KQUAD":
            e = Element(e.name + str(k), e.type, dict(e.params, **variants[k % len(variants)]))
            k += 1
        els.append(e)
    return Lattice(els)


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_quad_fringes(math):
    lat = _ring_with_quad_fringes()
    beam = _mixed_beam(91)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and 0 < n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    r0, n0, _, _ = RefOracle(math).track(w.fodo_ring(), beam.coords, beam.ids, P0, 20)
    assert not np.array_equal(r0[:min(n0, n1), :4], r1[:min(n0, n1), :4])


def _ring_with_linked_cavities():
    """Three extra cavities: two sharing PHASE_REFERENCE 7 with the ring's own
    cavity (each with its own PHASE and one at another frequency), one
    alone; the group's later cavities take the first one's fiducial phase
    (simple_rfca.c:410-470)."""
    from elegant_b200 import Element, Lattice
    base = list(w.fodo_ring().elements)
    rf = next(e for e in base if e.type == "RFCA")
    els = [e for e in base if e.type != "RFCA"]
    els.insert(10, Element("RFA", "RFCA", dict(rf.params, VOLT=3e5, PHASE_REFERENCE=7)))
    els.insert(30, Element("RFB", "RFCA", dict(rf.params, VOLT=2e5, PHASE=170.0, FREQ=rf.params["FREQ"] * 2,
                                               PHASE_REFERENCE=7)))
    els.insert(45, Element("RFC", "RFCA", dict(rf.params, VOLT=2e5, PHASE=175.0, PHASE_REFERENCE=9)))
    els.append(Element("RF", "RFCA", dict(rf.params, PHASE=178.0, PHASE_REFERENCE=7)))
    return Lattice(els)


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_linked_cavities(math):
    lat = _ring_with_linked_cavities()
    beam = _mixed_beam(101)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and 0 < n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
    from elegant_b200 import Element, Lattice
    unlinked = Lattice([Element(e.name, e.type, {k: v for k, v in e.params.items() if k != "PHASE_REFERENCE"})
                        for e in lat.elements])
    r0, n0, _, _ = RefOracle(math).track(unlinked, beam.coords, beam.ids, P0, 20)
    assert not np.array_equal(r0[:min(n0, n1), :6], r1[:min(n0, n1), :6])


def _ring_with_simple_edges():
    """Bends with EDGE_EFFECTS 3 (applySimpleDipoleEdgeKick, csbend.c:5639-5665)
    on one or both faces, with edge angles and a fringe gap, one radiating."""
    from elegant_b200 import Element, Lattice
    variants = [{"EDGE1_EFFECTS": 3, "EDGE2_EFFECTS": 3, "E1": 0.05, "E2": 0.03, "HGAP": 0.01},
                {"EDGE1_EFFECTS": 3, "E1": -0.04}, {"EDGE2_EFFECTS": 3, "E2": 0.06, "HGAP": 0.02, "FINT": 0.4},
                {"EDGE1_EFFECTS": 3, "EDGE2_EFFECTS": 3, "E1": 0.02, "E2": 0.02, "SYNCH_RAD": 1}]
    els, k = [], 0
    for e in w.fodo_ring().elements:
        if e.type == "CSBEND":
            e = Element(e.name + str(k), e.type, dict(e.params, **variants[k % len(variants)]))
            k += 1
        els.append(e)
    return Lattice(els)


@pytest.mark.parametrize("math", ["libm", "b2e"])
def test_port_reproduces_reference_simple_edges(math):
    lat = _ring_with_simple_edges()
    beam = _mixed_beam(111)
    r1, n1, e1, _ = RefOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    r2, n2, e2 = PortOracle(math).track(lat, beam.coords, beam.ids, P0, 20)
    assert n1 == n2 and e1 == e2 and 0 < n1 < beam.n
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])
    assert np.array_equal(r1[:, 6:8], r2[:, 6:8])
