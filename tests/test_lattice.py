"""Host-side lattice handling: .lte subset reader, elegant defaults, errors."""
import pytest

from elegant_b200 import Element, Lattice, LatticeError, parse_lte
from elegant_b200 import _native as nat
from elegant_b200 import workloads as w
from elegant_b200.optics import periodic_twiss

LTE = """
! a two-cell test line
D1: DRIF, L=0.5
QF: KQUAD, L=0.3, K1=1.2, &
    N_KICKS=8
QD: QF, K1=-1.2
B: CSBEND, L=1.0, ANGLE="2*pi/16", N_KICKS=8
S: KSEXT, L=0.2, K2=5
MA: MAXAMP, X_MAX=0.02, Y_MAX=0.02, ELLIPTICAL=1
CELL: LINE=(MA, D1, QF, D1, B, B, QD, S)
RING: LINE=(2*CELL, -(D1, QF))
USE, RING
"""


def test_parse_lte_expands_lines():
    lat = parse_lte(LTE)
    assert len(lat) == 2 * 8 + 2
    assert [e.name for e in lat.elements[-2:]] == ["QF", "D1"]
    qd = lat.elements[6]
    assert qd.type == "KQUAD" and qd.get("K1") == -1.2 and qd.get("N_KICKS") == 8
    b = lat.elements[4]
    assert abs(b.get("ANGLE") - 2 * 3.141592653589793 / 16) < 1e-15
    assert b.get("N_SLICES") == 8  # N_KICKS is an alias of N_SLICES for CSBEND
    assert lat.total_length == pytest.approx(2 * 3.8 + 0.8)


def test_defaults_follow_reference_tables():
    q = Element("Q", "KQUAD", {"L": 0.3, "K1": 1})
    assert q.get("N_SLICES") == 1 and q.get("INTEGRATION_ORDER") == 4
    b = Element("B", "CSBEND", {"L": 1, "ANGLE": 0.1})
    assert b.get("N_SLICES") == 4 and b.get("FINT") == 0.5 and b.get("EDGE1_EFFECTS") == 1
    r = Element("R", "RFCA", {})
    assert r.get("FREQ") == 500e6 and r.get("T_REFERENCE") == -1
    slots = b.slots()
    assert slots[12] == 4 and slots[11] == 0.5


def test_unsupported_inputs_fail_loudly():
    with pytest.raises(LatticeError):
        Element("W", "WIGGLER", {})
    with pytest.raises(LatticeError):
        Element("Q", "KQUAD", {"L": 0.3, "RADIAL": 1})
    with pytest.raises(LatticeError):
        parse_lte("A: DRIF, L=1\nL1: LINE=(A, B)\nUSE, L1\n")


def test_lte_round_trip():
    lat = w.fodo_ring()
    again = parse_lte(lat.to_lte())
    assert [(e.type, e.params) for e in again.elements] == [(e.type, e.params) for e in lat.elements]


def test_ctypes_layout():
    import ctypes
    assert ctypes.sizeof(nat.Element) == 4 + 4 + 32 + 8 * nat.MAX_PARAMS
    arr = w.fodo_ring().to_ctypes()
    assert arr[2].type == nat.KQUAD and arr[2].p[1] == 1.2


def test_ring_optics_stable():
    tw = periodic_twiss(w.fodo_ring(rf=False))
    assert 0 < tw.tune_x < 0.5 and 0 < tw.tune_y < 0.5 and tw.beta_x > 0 and tw.beta_y > 0


def test_maxamp_exponents_take_elegants_names():
    """MAXAMP's EXPONENT and YEXPONENT (track_data.c:994-995) land in their
    slots from an .lte line; YEXPONENT 0 leaves the y exponent to EXPONENT."""
    lat = parse_lte("MA: MAXAMP, X_MAX=0.02, Y_MAX=0.01, ELLIPTICAL=1, EXPONENT=4, YEXPONENT=6\nL: LINE=(MA)\n")
    s = lat.elements[0].slots()
    assert s[3] == 4 and s[4] == 6
    assert Element("MA", "MAXAMP", {}).slots()[3] == 2 and Element("MA", "MAXAMP", {}).slots()[4] == 0
    with pytest.raises(LatticeError):
        Element("MA", "MAXAMP", {"Y_EXPONENT": 6}).slots()


def test_lte_parameters_of_the_wider_element_set():
    """.lte text with the RFCA fiducial string and phase group, KQUAD
    correctors, fringe integrals and effective length, CSBEND steering:
    parsed into engine slots and written back unchanged."""
    text = ('D: DRIF, L=1\nRF: RFCA, VOLT=1e6, FREQ=5e8, FIDUCIAL="light", PHASE_REFERENCE=3\n'
            'Q: KQUAD, L=0.3, K1=1, HKICK=1e-4, EDGE1_EFFECTS=2, I0P=0.01, LEFFECTIVE=0.28, HSTEERING=1\n'
            'B: CSBEND, L=1, ANGLE=0.1, XKICK=1e-4, YKICK=2e-5\nL1: LINE=(D,RF,Q,B)\nUSE, L1\n')
    lat = parse_lte(text)
    rf, q, b = lat.elements[1], lat.elements[2], lat.elements[3]
    assert rf.params["FIDUCIAL"] == 1 and rf.slots()[9] == 3  # B2E_RFCA_FIDUCIAL, B2E_RFCA_PHASE_REFERENCE
    # B2E_KMULT_HKICK, _EDGE1_EFFECTS, _LEFFECTIVE, _EDGE1_LINEAR (default 1); B2E_BEND_XKICK, _YKICK
    assert q.slots()[15] == 1e-4 and q.slots()[21] == 2 and q.slots()[37] == 0.28 and q.slots()[23] == 1
    assert b.slots()[38] == 1e-4 and b.slots()[39] == 2e-5
    again = parse_lte(lat.to_lte())
    assert [e.params for e in again.elements] == [e.params for e in lat.elements]
