"""Synchrotron radiation in KQUAD/KSEXT/CSBEND on the CPU oracles.

- SYNCH_RAD is deterministic: the restatement reproduces elegant's own
  multipole_tracking2 / track_through_csbend with radiation (oracle/_ref) bit
  for bit, edges included.
- The energy radiated by an on-axis particle in one turn is the textbook
  U0 = C_gamma E^4 / rho to within the (1+delta)^2 weighting over the turn.
- ISR: the restatement draws with the engine's counter-based generator, the
  reference build with its own serial one; both give the same quantum
  excitation in distribution.
"""
import math

import numpy as np
import pytest

from elegant_b200 import workloads as w
from elegant_b200.beam import Beam
from reforacle import PortOracle, RefOracle, by_id

P0 = w.ring_p_central()


@pytest.mark.parametrize("math_mode", ["libm", "b2e"])
@pytest.mark.parametrize("edge", [0.0, 0.04])
def test_port_reproduces_reference_with_synch_rad(math_mode, edge):
    lat = w.radiating_ring(edge_angle=edge)
    beam = w.ring_beam(300, seed=5)
    r1, n1, _, _ = RefOracle(math_mode).track(lat, beam.coords, beam.ids, P0, 60)
    r2, n2, _ = PortOracle(math_mode).track(lat, beam.coords, beam.ids, P0, 60)[:3]
    assert n1 == n2 > 250
    assert np.array_equal(r1[:n1, :7], r2[:n2, :7])


def test_energy_radiated_per_turn_matches_u0():
    lat = w.radiating_ring()
    lat = type(lat)([e for e in lat.elements if e.type != "RFCA"])
    b = Beam(np.zeros((1, 6)), np.array([1]))
    rows, n, _, _ = RefOracle("b2e").track(lat, b.coords, b.ids, P0, 1)
    bend = next(e for e in lat.elements if e.type == "CSBEND")
    rho = bend.params["L"] / bend.params["ANGLE"]
    e_gev = P0 * 0.51099895e-3
    a = 8.8463e-5 * e_gev ** 4 / rho / e_gev          # U0 / E
    expected = -a / (1 + a)                               # d(delta)/ds ~ -(1+delta)^2
    assert n == 1
    assert abs(rows[0, 5] / expected - 1) < 2e-3, (rows[0, 5], expected)


def test_isr_excitation_matches_reference_in_distribution():
    """All particles start on the design orbit; after 40 turns the energy
    spread and bunch length come from quantum excitation alone.  The reference
    build (its own generator) and the restatement (the engine's) agree within
    the statistical error (1.8 % on each rms for 1,500 particles)."""
    lat = w.radiating_ring(isr=True)
    n, turns = 1500, 40
    coords = np.zeros((n, 6))
    ids = np.arange(1, n + 1)
    r1, n1, _, _ = RefOracle("b2e", private=True).track(lat, coords, ids, P0, turns)
    port = PortOracle("b2e")
    port.set_isr(1234)
    r2, n2, _ = port.track(lat, coords, ids, P0, turns)[:3]
    port.set_isr(0)
    assert n1 == n2 == n
    s1, s2 = r1[:n1, 5].std(), r2[:n2, 5].std()
    assert s1 > 2e-4 and abs(s1 / s2 - 1) < 0.1, (s1, s2)
    z1, z2 = r1[:n1, 4].std(), r2[:n2, 4].std()
    assert abs(z1 / z2 - 1) < 0.1, (z1, z2)
    assert abs(r1[:n1, 5].mean() - r2[:n2, 5].mean()) < 4 * s1 / math.sqrt(n)
    # without ISR the on-axis particles stay together
    r0, n0, _ = port.track(w.radiating_ring(), coords, ids, P0, 5)[:3]
    assert np.ptp(r0[:n0, 5]) == 0


def test_isr_deviates_are_addressed_not_sequenced():
    """Same seed, same result whatever the particle order; another seed, a
    different result."""
    lat = w.radiating_ring(isr=True)
    beam = w.ring_beam(200, seed=8)
    port = PortOracle("b2e")
    port.set_isr(7)
    a = by_id(port.track(lat, beam.coords, beam.ids, P0, 10)[0])[0]
    perm = np.random.default_rng(0).permutation(beam.n)
    b = by_id(port.track(lat, beam.coords[perm], beam.ids[perm], P0, 10)[0])[0]
    port.set_isr(8)
    c = by_id(port.track(lat, beam.coords, beam.ids, P0, 10)[0])[0]
    port.set_isr(0)
    assert np.array_equal(a, b)
    assert not np.array_equal(a[:, 5], c[:, 5])


def test_philox_known_answers():
    """Philox4x32-10 against the published known-answer vectors of its
    authors (counter and key all zeros, all ones, and the digits of pi)."""
    import ctypes
    lib = PortOracle("b2e").lib
    f = lib.b2e_oracle_philox
    f.argtypes = [ctypes.POINTER(ctypes.c_uint32)] * 3
    cases = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
             ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
             ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
              (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in cases:
        c = (ctypes.c_uint32 * 4)(*ctr)
        k = (ctypes.c_uint32 * 2)(*key)
        out = (ctypes.c_uint32 * 4)()
        f(c, k, out)
        assert tuple(out) == want, [hex(v) for v in out]
