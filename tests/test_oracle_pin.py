"""Pins the CPU oracles (no GPU needed).

- the C restatement (oracle/b2e_oracle.c) reproduces elegant's own tracking
  code (oracle/_ref, compiled from the reference sources) row for row, bit for
  bit, in both maths modes, including lost-particle bookkeeping;
- the shared elementary functions agree with glibc's to within the ring's
  intrinsic sensitivity: after 10 turns within 1e-10 relative, and after
  many turns no further apart than a one-ulp perturbation of the initial
  coordinates grows by itself under the reference with glibc.
"""
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
