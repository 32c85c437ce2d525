"""The C ABI's error behaviour on the device: calls out of order, sizes that
do not match and parameters the engine does not support return the
documented status codes (include/elegant_b200.h) with a message, and the
context stays usable afterwards."""
import numpy as np
import pytest

from elegant_b200 import workloads as w
from elegant_b200._native import EngineError
from elegant_b200.beam import Beam
from elegant_b200.lattice import Element, Lattice
from elegant_b200.track import Tracker

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_LATTICE, ERR_STATE = -1, -2, -5
P0 = 1000 / 0.51099895


def test_track_before_upload_is_a_state_error_and_the_context_recovers():
    with Tracker(w.fodo_ring(), w.ring_p_central(), 3) as t:
        with pytest.raises(EngineError) as e:
            t.continue_tracking()
        assert e.value.code == ERR_STATE and "first" in str(e.value)
        res = t.track(w.ring_beam(50, seed=1))
        assert res.n_left == 50


def test_history_needs_record_history():
    with Tracker(w.fodo_ring(), w.ring_p_central(), 3) as t:
        t.track(w.ring_beam(40, seed=2))
        with pytest.raises(EngineError) as e:
            t.history()
        assert e.value.code == ERR_STATE


def test_history_is_refused_with_csr_elements():
    with Tracker(w.chicane(bins=100, n_kicks=2), P0, 1, record_history=True) as t:
        with pytest.raises(EngineError) as e:
            t.track(w.chicane_beam(1000, seed=3))
        assert e.value.code == ERR_LATTICE and "CSR" in str(e.value)


def test_ensemble_offsets_must_cover_the_beam():
    lat, beam, offsets, overrides = w.ensemble(n_instances=3, n_min=10, n_max=20, seed=4)
    with Tracker(lat, w.ring_p_central(), 2) as t:
        t.load_ensemble(offsets, overrides)
        with pytest.raises(EngineError) as e:
            t.track(Beam(beam.coords[:-1], beam.ids[:-1]))
        assert e.value.code == ERR_ARG and "offsets" in str(e.value)
        res = t.track(beam)  # the full beam still tracks
        assert res.coords.shape == beam.coords.shape


def test_ensemble_offsets_must_be_nondecreasing():
    with Tracker(w.fodo_ring(), w.ring_p_central(), 2) as t:
        with pytest.raises(EngineError) as e:
            t.load_ensemble(np.array([0, 10, 5]), [])
        assert e.value.code == ERR_ARG


def test_csr_elements_take_no_per_instance_overrides():
    lat = w.chicane(bins=100, n_kicks=2)
    with Tracker(lat, P0, 1) as t:
        with pytest.raises(EngineError) as e:
            t.load_ensemble(np.array([0, 10, 20]), [(1, "ANGLE", np.array([0.05, 0.06]))])
        assert e.value.code == ERR_LATTICE


@pytest.mark.parametrize("typ, params, words", [
    ("CSRCSBEND", {"L": 0.5, "ANGLE": 0.05, "BINS": 100, "K1": 0.5}, "K1"),
    ("CSBEND", {"L": 1.0, "ANGLE": 0.1, "EDGE1_EFFECTS": 2}, "EDGE"),
    ("RFCA", {"L": -0.2, "VOLT": 1e6, "FREQ": 5e8}, "negative length"),
    ("KQUAD", {"L": 0.2, "K1": 1.0, "INTEGRATION_ORDER": 3}, "INTEGRATION_ORDER"),
    ("CSRCSBEND", {"L": 0.5, "ANGLE": 0.05, "BINS": 100, "IGF": 1}, "STEADY_STATE"),
    ("CSRCSBEND", {"L": 0.5, "ANGLE": 0.05, "BINS": 1}, "bins"),
    ("KQUAD", {"L": 0.2, "K1": 1.0, "EDGE1_EFFECTS": 3}, "EDGE"),
    ("CSRCSBEND", {"L": 0.5, "ANGLE": 0.05, "BINS": 100, "XKICK": 1e-4}, "XKICK"),
])
def test_unsupported_parameters_are_rejected_at_load(typ, params, words):
    lat = Lattice([Element("D", "DRIF", {"L": 1.0}), Element("X", typ, params)])
    with pytest.raises(EngineError) as e:
        Tracker(lat, P0, 1)
    assert e.value.code == ERR_LATTICE and words in str(e.value)


def test_wakenet_rejects_bad_sizes():
    import torch
    from elegant_b200.wakenet import IN_CH, WakeNet
    with pytest.raises(EngineError) as e:
        WakeNet(bins=1000, max_batch=4)  # bins must be a multiple of 128
    assert e.value.code == ERR_ARG
    with WakeNet(bins=256, max_batch=2) as net:
        x = torch.zeros((3, IN_CH, 256), dtype=torch.float32, device="cuda")
        y = torch.zeros((3, 256), dtype=torch.float32, device="cuda")
        rc = net.lib.b2e_wakenet_forward(net._h, x.data_ptr(), 3, y.data_ptr(), None)
        assert rc == ERR_ARG  # above the network's maximum batch
        assert net.forward(x).shape == (3, 256)  # the binding splits the batch


def test_csrdrift_mode_change_behind_one_dipole_is_rejected():
    lat = w.chicane(bins=100, n_kicks=2)
    els = [Element(e.name, e.type, dict(e.params, USE_STUPAKOV=1)) if e.name == "D3" else e for e in lat.elements]
    els.insert(7, Element("D3B", "CSRDRIFT", {"L": 0.5}))
    with pytest.raises(EngineError) as e:
        Tracker(Lattice(els), P0, 1)
    assert e.value.code == ERR_LATTICE and "mode" in str(e.value)
