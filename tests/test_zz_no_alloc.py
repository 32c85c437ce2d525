"""The allocation-free CSR dipole entry point (b2e_csr_bend_static).

It exists for callers that cannot allocate device memory while they track; it
keeps its working memory in a static device array.  Here it is called through
the C ABI on caller-owned device buffers, twice in a row, and each result must
equal -- bit for bit, the bar of every parity test in this suite -- what the
regular context path (b2e_track_host + b2e_csr_wakes) gives for the same
bend.  This file is collected last so that a stop-at-first-failure run has
already exercised everything else.
"""
import ctypes

import numpy as np
import pytest

from elegant_b200 import Element, Lattice, Tracker, workloads as w
from elegant_b200 import _native as nat

pytestmark = pytest.mark.gpu

P0 = 1000 / 0.51099895
CHARGE = 1e-9


def bend_element(**extra):
    return Element("B1", "CSRCSBEND", dict({"L": 0.5, "ANGLE": 0.05, "N_KICKS": 6, "BINS": 240, "SG_HALFWIDTH": 2},
                                           **extra))


class StaticCall:
    """Caller-owned device buffers for one call, made before the call."""

    def __init__(self, beam, wakes_needed):
        import torch
        dev = torch.device("cuda:0")
        self.n = beam.n
        self.cols = [torch.tensor(np.ascontiguousarray(beam.coords[:, i]), dtype=torch.float64, device=dev)
                     for i in range(6)]
        self.lost_pass = torch.full((beam.n,), -1, dtype=torch.int32, device=dev)
        self.lost_elem = torch.full((beam.n,), -1, dtype=torch.int32, device=dev)
        self.wakes = torch.zeros(wakes_needed, dtype=torch.float64, device=dev)
        self.ptrs = nat.pointer_array([c.data_ptr() for c in self.cols])
        self.err = ctypes.create_string_buffer(512)

    def __call__(self, lib, bend_arr):
        return lib.b2e_csr_bend_static(self.ptrs, ctypes.c_void_p(self.lost_pass.data_ptr()),
                                       ctypes.c_void_p(self.lost_elem.data_ptr()), ctypes.c_int64(self.n),
                                       ctypes.byref(bend_arr), ctypes.c_double(P0),
                                       ctypes.c_double(CHARGE / max(self.n, 1)),
                                       ctypes.c_void_p(self.wakes.data_ptr()), ctypes.c_int64(self.wakes.numel()),
                                       None, self.err, ctypes.c_int64(512))

    def results(self):
        coords = np.stack([c.cpu().numpy() for c in self.cols], axis=1)
        return coords, self.lost_pass.cpu().numpy(), self.wakes.cpu().numpy()


def static_call(lib, beam, bend_arr, wakes_needed):
    import torch
    call = StaticCall(beam, wakes_needed)
    rc = call(lib, bend_arr)
    torch.cuda.synchronize()
    assert rc == 0, call.err.value.decode()
    return call.results()


@pytest.mark.parametrize("extra", [{}, {"HIGH_FREQUENCY_CUTOFF0": 0.2, "LOW_FREQUENCY_CUTOFF0": 0.02}])
def test_static_bend_matches_context_path_twice(extra):
    lib = nat.load_library()
    lib.b2e_csr_bend_static.restype = ctypes.c_int
    bend = bend_element(**extra)
    lat = Lattice([Element("Q", "CHARGE", {"TOTAL": CHARGE}), bend])
    beam = w.chicane_beam(30000, seed=12)
    with Tracker(lat, P0, 1) as t:
        ref = t.track(beam)
        ref_wakes = t.csr_wakes(10_000_000)
    n_wakes = 6 * 240
    assert ref_wakes.shape == (n_wakes,)
    bend_arr = Lattice([bend]).to_ctypes()[0]
    for call in range(2):
        coords, lost, wakes = static_call(lib, beam, bend_arr, n_wakes)
        assert np.array_equal(lost, ref.lost_pass), f"call {call}: loss flags differ"
        assert np.array_equal(wakes, ref_wakes), f"call {call}: wakes differ"
        assert np.array_equal(coords, ref.coords), f"call {call}: coordinates differ"


def test_static_bend_rejects_oversize_requests():
    lib = nat.load_library()
    lib.b2e_csr_bend_static.restype = ctypes.c_int
    bend_arr = Lattice([bend_element()]).to_ctypes()[0]
    dummy = nat.pointer_array([1, 1, 1, 1, 1, 1])
    err = ctypes.create_string_buffer(256)
    rc = lib.b2e_csr_bend_static(dummy, ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_int64(1048577),
                                 ctypes.byref(bend_arr), ctypes.c_double(P0), ctypes.c_double(1e-15), None,
                                 ctypes.c_int64(0), None, err, ctypes.c_int64(256))
    assert rc == -1 and b"exceed the static limit" in err.value
    big = Lattice([Element("B", "CSRCSBEND", {"L": 0.5, "ANGLE": 0.05, "BINS": 4096})]).to_ctypes()[0]
    rc = lib.b2e_csr_bend_static(dummy, ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_int64(10),
                                 ctypes.byref(big), ctypes.c_double(P0), ctypes.c_double(1e-15), None,
                                 ctypes.c_int64(0), None, err, ctypes.c_int64(256))
    assert rc == -1 and b"BINS=4096" in err.value


def test_static_bend_allocates_no_device_memory():
    """After the per-device set-up call (n = 0), a call leaves the device's
    free memory unchanged: the buffers it uses are the caller's and the
    library's static array."""
    import torch
    lib = nat.load_library()
    lib.b2e_csr_bend_static.restype = ctypes.c_int
    bend_arr = Lattice([bend_element()]).to_ctypes()[0]
    err = ctypes.create_string_buffer(256)
    rc = lib.b2e_csr_bend_static(None, None, None, ctypes.c_int64(0), ctypes.byref(bend_arr), ctypes.c_double(P0),
                                 ctypes.c_double(0.0), None, ctypes.c_int64(0), None, err, ctypes.c_int64(256))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    call = StaticCall(w.chicane_beam(50000, seed=3), 6 * 240)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert call(lib, bend_arr) == 0, call.err.value.decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    assert (call.lost_pass.cpu().numpy() < 0).all()


@pytest.mark.parametrize("n,bins", [(1_048_576, 600), (40_000, 2048)])
def test_static_bend_at_its_limits(n, bins):
    """The largest particle count and the largest bin count the static array
    holds (the 2,048-bin wake kernel needs 65.6 KB of shared memory), equal to
    the context path bit for bit."""
    lib = nat.load_library()
    lib.b2e_csr_bend_static.restype = ctypes.c_int
    bend = bend_element(N_KICKS=4, BINS=bins)
    lat = Lattice([Element("Q", "CHARGE", {"TOTAL": CHARGE}), bend])
    beam = w.chicane_beam(n, seed=17)
    with Tracker(lat, P0, 1) as t:
        ref = t.track(beam)
        ref_wakes = t.csr_wakes(4 * bins + 1)
    coords, lost, wakes = static_call(lib, beam, Lattice([bend]).to_ctypes()[0], 4 * bins)
    assert np.array_equal(wakes, ref_wakes)
    assert np.array_equal(lost, ref.lost_pass)
    assert np.array_equal(coords, ref.coords)
