"""Turn-by-turn recording, the NAFF kernel and the frequency map on the
device.

- b2e_naff equals the numpy statement of the same method (tests/
  naff_reference.py) to 1e-11 in frequency on signals of known content.
- The turn-by-turn record after j passes equals elegant's own code tracked
  for j passes, bit for bit.
- fiducial_particles = 1: the RF phase reference comes from row 0 alone, so
  a particle's motion does not depend on which other particles share its
  run (as with elegant's separate fiducial particle).
- The frequency map's small-amplitude tunes are the one-turn matrix's.
"""
import ctypes
import math

import numpy as np
import pytest

from elegant_b200 import Tracker, workloads as w
from elegant_b200 import _native as nat
from elegant_b200.beam import Beam
from elegant_b200.frequency_map import frequency_map
from elegant_b200.optics import line_matrix
from naff_reference import naff
from reforacle import by_id

pytestmark = pytest.mark.gpu
P0 = w.ring_p_central()


@pytest.mark.parametrize("n", [256, 1000])
def test_naff_kernel_matches_numpy(n):
    import torch
    rng = np.random.default_rng(7)
    sig = []
    for _ in range(64):
        nu, nu2 = rng.uniform(0.03, 0.47), rng.uniform(0.03, 0.47)
        t = np.arange(n)
        sig.append(rng.uniform(0.5, 2) * np.cos(2 * np.pi * nu * t + rng.uniform(-3, 3)) +
                   0.1 * np.cos(2 * np.pi * nu2 * t) + rng.uniform(-1, 1))
    sig = np.array(sig)
    d = torch.tensor(sig, dtype=torch.float64, device="cuda")
    f, a, p = (torch.empty(len(sig), dtype=torch.float64, device="cuda") for _ in range(3))
    lib = nat.load_library()
    assert lib.b2e_naff(d.data_ptr(), len(sig), n, f.data_ptr(), a.data_ptr(), p.data_ptr(), None) == 0
    torch.cuda.synchronize()
    f, a, p = f.cpu().numpy(), a.cpu().numpy(), p.cpu().numpy()
    for k in range(len(sig)):
        rf, ra, rp = naff(sig[k])
        assert abs(f[k] - rf) < 1e-11, (k, f[k], rf)
        assert abs(a[k] - ra) < 1e-9 * ra
        assert abs(math.remainder(p[k] - rp, 2 * math.pi)) < 1e-8


def test_tbt_records_equal_reference_tracking(ref_b2e):
    lat = w.fodo_ring()
    beam = w.ring_beam(300, seed=61)
    with Tracker(lat, P0, 12, record_tbt=True) as t:
        t.track(beam)
        tbt = t.tbt()
    assert tbt.shape == (13, 4, beam.n)
    assert np.array_equal(tbt[0], beam.coords[:, :4].T)
    for j in (1, 5, 12):
        rows, nl, _, _ = ref_b2e.track(lat, beam.coords, beam.ids, P0, j)
        ref_c, ref_ids, ref_loss = by_id(rows)
        alive = ref_loss < 0
        order = np.argsort(beam.ids)
        rec = tbt[j][:, order].T
        assert np.array_equal(rec[alive], ref_c[alive][:, :4]), j
        assert np.isnan(rec[~alive]).all()


def test_fiducial_from_the_first_row_only():
    lat = w.fodo_ring()
    ref = np.zeros((1, 6))
    a = w.ring_beam(50, seed=62).coords
    b = w.ring_beam(70, seed=63).coords * 1.5
    out = []
    for extra in (a, np.concatenate([a, b])):
        coords = np.concatenate([ref, extra])
        with Tracker(lat, P0, 30, fiducial_particles=1) as t:
            r = t.track(Beam(coords, np.arange(1, len(coords) + 1)))
        out.append(r.coords[1:1 + len(a)])
    assert np.array_equal(out[0], out[1])
    with Tracker(lat, P0, 30) as t:  # the reference particle alone: the same phase reference
        r0 = t.track(Beam(ref, np.array([1])))
    with Tracker(lat, P0, 30, fiducial_particles=1) as t:
        r1 = t.track(Beam(np.concatenate([ref, a]), np.arange(1, 52)))
    assert np.array_equal(r0.coords[0], r1.coords[0])


def _linear_tunes(lat):
    m = line_matrix(type(lat)([e for e in lat.elements if e.type != "RFCA"]))
    out = []
    for p in (0, 2):
        a = m[p:p + 2, p:p + 2]
        cmu = 0.5 * (a[0, 0] + a[1, 1])
        smu = math.copysign(math.sqrt(1 - cmu * cmu), a[0, 1])
        out.append((math.atan2(smu, cmu) / (2 * math.pi)) % 1.0)
    return out


def test_frequency_map_small_amplitudes_give_the_linear_tunes():
    lat = w.fodo_ring()
    rows = frequency_map(lat, P0, 512, xmin=1e-6, xmax=4e-6, ymin=1e-6, ymax=4e-6, nx=3, ny=3, include_changes=True)
    nux0, nuy0 = _linear_tunes(lat)
    assert len(rows) == 9
    for r in rows:
        assert abs(r["nux"] - nux0) < 2e-3 and abs(r["nuy"] - nuy0) < 2e-3, (r, nux0, nuy0)
        assert r["diffusion"] < -6
    # larger amplitudes: detuning grows and some points are lost, and are left out
    big = frequency_map(lat, P0, 256, xmin=-0.015, xmax=0.015, ymin=1e-6, ymax=0.008, nx=7, ny=5)
    assert 0 < len(big) <= 35
    assert all(0 <= r["nux"] <= 1 and 0 <= r["nuy"] <= 1 for r in big)
