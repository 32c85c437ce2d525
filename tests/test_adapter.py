"""The drop-in adapter (elegant_b200/adapter/b2e_adapter.c), compiled against
the reference's own track.h and linked with the reference's objects and the
engine (oracle/_ref/libb2e_ref_adapter.so, built by oracle/Makefile.ref).

elegant's ELEMENT_LIST and element structures are built by oracle/ref_driver.c
from the reference's parameter tables (track_data.c), handed to
b2e_adapter_track as do_tracking would hand them, and the rows it returns are
compared with the reference's own tracking of the same line (shared
elementary functions): bit-identical survivors, identical (ID, loss pass)
pairs, survivors first in the row order.  Lines the engine cannot take are
declined before anything changes (CPU-only tests).
"""
import ctypes
import os

import numpy as np
import pytest

from elegant_b200 import Element, Lattice, workloads as w
from reforacle import by_id, lattice_spec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libb2e_ref_adapter.so")


@pytest.fixture(scope="module")
def adapter():
    if not os.path.exists(LIB):
        pytest.skip("adapter library not built (needs the reference tree)")
    lib = ctypes.CDLL(LIB)
    lib.b2e_ref_adapter_track.restype = ctypes.c_long
    return lib


def adapter_track(lib, lattice, beam, p0, passes):
    n = beam.n
    rows = np.zeros((n, 7))
    rows[:, :6] = beam.coords
    rows[:, 6] = beam.ids
    out = np.zeros((max(n, 1), 8))
    eff = ctypes.c_double()
    err = ctypes.create_string_buffer(512)
    st = lib.b2e_ref_adapter_track(lattice_spec(lattice).encode(), ctypes.c_double(p0),
                                   rows.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(n), ctypes.c_long(passes),
                                   out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(eff), err, ctypes.c_long(512))
    return st, out[:n], eff.value, err.value.decode()


def _lossy(n, seed):
    from elegant_b200.beam import Beam
    rng = np.random.default_rng(seed)
    c = np.zeros((n, 6))
    c[:, 0] = rng.uniform(-0.022, 0.022, n)
    c[:, 1] = rng.uniform(-3e-3, 3e-3, n)
    c[:, 2] = rng.uniform(-0.015, 0.015, n)
    c[:, 3] = rng.uniform(-2e-3, 2e-3, n)
    c[:, 4] = rng.normal(0, 5e-3, n)
    c[:, 5] = rng.uniform(-0.03, 0.03, n)
    return Beam(c, np.arange(1, n + 1))


def _ring_variant():
    els = []
    for i, e in enumerate(w.fodo_ring().elements):
        if e.type == "KQUAD":
            e = Element(e.name, e.type, dict(e.params, DX=2e-4 * ((i % 3) - 1), FSE=1e-3))
        if e.name == "D2":
            e = Element(e.name, "EDRIFT", {"L": e.params["L"]})
        els.append(e)
    return Lattice(els)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ring", "ring_variant", "steering", "quad_fringes", "chicane"])
def test_adapter_equals_reference_tracking(adapter, ref_b2e, case):
    from elegant_b200.beam import Beam
    if case == "chicane":
        lat, beam, p0, passes = w.chicane(bins=150, n_kicks=5), w.chicane_beam(10000, seed=3), 1000 / 0.51099895, 1
    else:
        if case == "steering":
            from test_oracle_pin import _ring_with_steering
            lat = _ring_with_steering()  # HKICK/VKICK, calibrations, BORE/B, HSTEERING and PITCH through the tables
        elif case == "quad_fringes":
            from test_oracle_pin import _ring_with_quad_fringes
            lat = _ring_with_quad_fringes()
        else:
            lat = w.fodo_ring() if case == "ring" else _ring_variant()
        good, bad = w.ring_beam(150, seed=4), _lossy(150, seed=5)
        beam = Beam(np.concatenate([good.coords, bad.coords]), np.arange(1, 301))
        p0, passes = w.ring_p_central(), 40
    st, rows, eff, err = adapter_track(adapter, lat, beam, p0, passes)
    assert st >= 0, err
    ref_rows, nl, ref_eff, _ = ref_b2e.track(lat, beam.coords, beam.ids, p0, passes)
    assert st == nl and eff == ref_eff
    assert (rows[:st, 7] == -1).all() and (rows[st:, 7] >= 0).all()  # survivors first, as do_tracking leaves them
    a, b = by_id(rows), by_id(ref_rows)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    alive = b[2] < 0
    assert np.array_equal(a[0][alive], b[0][alive])
    if case != "chicane":
        assert nl < beam.n


def test_adapter_declines_what_the_engine_cannot_take(adapter):
    """An element type outside the engine's set, or a parameter away from its
    table default where the engine has no slot, is declined before any
    device work (so no GPU is needed here) and the rows are left as given."""
    beam = w.ring_beam(20, seed=1)
    cases = [
        ("D:DRIF L=0.5;S:SEXT L=0.2 K2=3", "SEXT"),
        ("D:DRIF L=0.5;Q:KQUAD L=0.3 K1=1.0 PITCH=0.001 MALIGN_METHOD=1", "MALIGN_METHOD"),
        ("D:DRIF L=0.5;Q:KQUAD L=0.3 K1=1.0 RADIAL=1", "RADIAL"),
        ("B:CSBEND L=1 ANGLE=0.1 FINT1=0.3", "FINT1"),
        ("B:CSRCSBEND L=0.5 ANGLE=0.05 BINS=100 OUTPUT_FILE=wake.sdds", "OUTPUT_FILE"),
        ("R:RFCA VOLT=1e6 FREQ=5e8 FIDUCIAL=first", "FIDUCIAL"),
    ]
    for spec, word in cases:
        n = beam.n
        rows = np.zeros((n, 7))
        rows[:, :6] = beam.coords
        rows[:, 6] = beam.ids
        out = np.zeros((n, 8))
        err = ctypes.create_string_buffer(512)
        st = adapter.b2e_ref_adapter_track(spec.encode(), ctypes.c_double(w.ring_p_central()),
                                           rows.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(n), ctypes.c_long(3),
                                           out.ctypes.data_as(ctypes.c_void_p), None, err, ctypes.c_long(512))
        assert st == -1 and word in err.value.decode(), (spec, st, err.value)
        assert np.array_equal(out[:, :6], beam.coords) and (out[:, 7] == -1).all()
