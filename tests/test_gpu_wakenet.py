"""Tensor-core (tcgen05/UMMA) kernels of the wake network on the GPU."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from elegant_b200 import _native as nat
    lib = nat.load_library()
    lib.b2e_umma_selftest.restype = ctypes.c_int
    lib.b2e_umma_selftest.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
    return lib


@pytest.mark.parametrize("mode", [0, 1])
def test_umma_operand_layouts(mode):
    import torch
    lib = _lib()
    g = torch.Generator().manual_seed(3 + mode)
    if mode == 0:
        a = torch.randn(128, 64, generator=g).to(torch.bfloat16)
        b = torch.randn(64, 64, generator=g).to(torch.bfloat16)
        ref = a.double() @ b.double().T
    else:
        a = torch.randn(2, 128, 64, generator=g).to(torch.bfloat16)
        b = torch.randn(128, 64, generator=g).to(torch.bfloat16)
        at = torch.cat([a[0].double().T, a[1].double().T], dim=0)  # [128 m][128 k]
        ref = at @ b.double()
    da, db = a.cuda(), b.cuda()
    d = torch.full((128, 64), float("nan"), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.b2e_umma_selftest(mode, da.data_ptr(), db.data_ptr(), d.data_ptr(), stream)
    assert rc == 0
    torch.cuda.synchronize()
    out = d.cpu().double()
    err = (out - ref).abs().max().item()
    assert err < 1e-3 * ref.abs().max().item(), err


def test_bounded_wait_gives_up_and_frees_tensor_memory():
    """The timeout drill: a kernel whose load barrier never completes stops
    waiting after its poll limit, reports B2E_ERR_TIMEOUT through its status
    word, frees its tensor memory and exits -- no trap, and the context stays
    usable: the drill runs again, then a real tile computes correctly."""
    import torch
    lib = _lib()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        assert lib.b2e_umma_selftest(2, None, None, None, stream) == -6  # B2E_ERR_TIMEOUT
    torch.cuda.synchronize()
    g = torch.Generator().manual_seed(11)
    a = torch.randn(128, 64, generator=g).to(torch.bfloat16)
    b = torch.randn(64, 64, generator=g).to(torch.bfloat16)
    d = torch.full((128, 64), float("nan"), dtype=torch.float32, device="cuda")
    da, db = a.cuda(), b.cuda()
    assert lib.b2e_umma_selftest(0, da.data_ptr(), db.data_ptr(), d.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    ref = a.double() @ b.double().T
    assert (d.cpu().double() - ref).abs().max().item() < 1e-3 * ref.abs().max().item()


import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _profiles(n, nb, seed):
    rng = np.random.default_rng(seed)
    i = np.arange(nb)
    out = np.zeros((n, nb))
    for p in range(n):
        for _ in range(rng.integers(1, 5)):
            c, s, w = rng.uniform(0.2, 0.8) * nb, rng.uniform(0.01, 0.1) * nb, rng.uniform(0.2, 1)
            out[p] += w * np.exp(-0.5 * ((i - c) / s) ** 2)
        out[p] *= 1e5 / out[p].sum()
        out[p] += rng.normal(0, 1, nb) * np.sqrt(out[p] + 1)
        out[p] = np.maximum(out[p], 0)
    return out


@pytest.mark.parametrize("sg,trapz,steady", [(2, True, False), (0, True, False), (3, False, False), (2, True, True)])
def test_wake_batch_matches_oracle_bit_exact(sg, trapz, steady):
    import torch
    from elegant_b200.wakenet import library
    from reforacle import PortOracle
    lib, o = library(), PortOracle("b2e")
    nb, n = 600, 6
    counts = _profiles(n, nb, seed=sg + 7 * trapz)
    slip = np.array([0.3, 1.0, 2.7, 35.5, 400.0, 5000.0])
    dc, ds = torch.tensor(counts, device="cuda"), torch.tensor(slip, device="cuda")
    t1, h, d = (torch.empty((n, nb), dtype=torch.float64, device="cuda") for _ in range(3))
    rc = lib.b2e_csr_wake_batch(dc.data_ptr(), ds.data_ptr(), n, nb, sg, 1, 0, 0, int(trapz), int(steady),
                                t1.data_ptr(), h.data_ptr(), d.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    for p in range(n):
        rt1, rh, rd = o.wake_t1(counts[p], slip[p], sg_half=sg, sg_order=1, trapz=trapz, steady=steady)
        assert np.array_equal(h[p].cpu().numpy(), rh)
        assert np.array_equal(d[p].cpu().numpy(), rd)
        assert np.array_equal(t1[p].cpu().numpy(), rt1), p


def _net_case(seed, n=3, L=256):
    import wakenet_oracle as wo
    from elegant_b200.wakenet import init_params
    rng = np.random.default_rng(seed)
    params = init_params(seed, out_scale=1.0)
    params[wo.LAYERS * wo.WSIZE:] = rng.normal(0, 0.05, wo.LAYERS * wo.CH).astype(np.float32)
    params[wo.LAYERS * wo.WSIZE + 5 * 64 + 1:] = 0  # output channels 1..63 are not live
    inputs = rng.normal(0, 1, (n, 4, L)).astype(np.float32)
    targets = rng.normal(0, 1, (n, L)).astype(np.float32)
    return params, inputs, targets


def test_wakenet_forward_matches_oracle():
    import torch
    import wakenet_oracle as wo
    from elegant_b200.wakenet import init_params
    from elegant_b200.wakenet import WakeNet
    params, inputs, _ = _net_case(1)
    with WakeNet(bins=256, max_batch=4) as net:
        net.set_params(params)
        y = net.forward(torch.tensor(inputs, device="cuda")).cpu().numpy().astype(np.float64)
    ref, _ = wo.forward(params, inputs, net.dilations)
    rel = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert rel < 1e-2, rel


def test_wakenet_gradients_match_oracle():
    import torch
    import wakenet_oracle as wo
    from elegant_b200.wakenet import init_params
    from elegant_b200.wakenet import WakeNet
    params, inputs, targets = _net_case(2)
    with WakeNet(bins=256, max_batch=4) as net:
        net.set_params(params)
        loss = net.gradients(torch.tensor(inputs, device="cuda"), torch.tensor(targets, device="cuda"))
        g = net.grads().astype(np.float64)
    ref_loss, ref = wo.loss_and_gradients(params, inputs, targets, net.dilations)
    assert abs(loss - ref_loss) < 1e-2 * ref_loss
    for l in range(wo.LAYERS):
        sl = slice(l * wo.WSIZE, (l + 1) * wo.WSIZE)
        a, b = g[sl], ref[sl]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel < 3e-2, (l, rel)
    gb, rb = g[wo.LAYERS * wo.WSIZE:], ref[wo.LAYERS * wo.WSIZE:]
    assert np.linalg.norm(gb - rb) / np.linalg.norm(rb) < 3e-2


def test_wakenet_training_reduces_loss():
    import torch
    import wakenet_oracle as wo
    from elegant_b200.wakenet import init_params
    from elegant_b200.wakenet import WakeNet
    rng = np.random.default_rng(4)
    L, n = 256, 8
    x = rng.normal(0, 1, (n, 4, L)).astype(np.float32)
    # a fixed linear target: a smoothed, shifted copy of channel 1
    k = np.exp(-0.5 * (np.arange(-8, 9) / 3.0) ** 2)
    tgt = np.stack([np.convolve(x[p, 1], k / k.sum(), mode="same") for p in range(n)]).astype(np.float32)
    with WakeNet(bins=L, max_batch=n) as net:
        net.set_params(init_params(3))
        xi, ti = torch.tensor(x, device="cuda"), torch.tensor(tgt, device="cuda")
        first = net.train_step(xi, ti, 1e-3, want_loss=True)
        for _ in range(150):
            net.train_step(xi, ti, 1e-3)
        last = net.train_step(xi, ti, 1e-3, want_loss=True)
    assert last < 0.2 * first, (first, last)


def test_learned_wake_gains_over_the_method_without_it(capsys):
    """The trained wake network against the method without it -- the plain
    FP64 integral that it replaces, and the same network untrained -- on
    held-out profiles (a seed training never used), and in tracking.

    Accuracy: the trained network reproduces the plain wake to well under
    the 1 % gate on held-out profiles; untrained, the same network is off by
    its whole output.  Time: the wake stage of every kick of a 4-bunch
    chicane run (0.5-1.2 M particles per bunch), timed inside the engine with events around the plain wake
    kernel, or the learned wake's filter + network + combine kernels.  Both
    are reported; the learned stage is not asserted to be faster (it is
    not: the plain integral is a few microseconds per bunch on one CTA)."""
    import json as _json
    import torch
    from elegant_b200 import Beam, Tracker, workloads as w
    from elegant_b200.bunch_train import DEFAULT_NET
    from elegant_b200.wake_surrogate import WakeSurrogate, build_set, evaluate
    from elegant_b200.wakenet import init_params
    sur = WakeSurrogate.load(DEFAULT_NET, max_batch=256)
    held_out = build_set(2000, sur.features.bins, seed=9001)
    trained = evaluate(sur, held_out)
    raw = WakeSurrogate.load(DEFAULT_NET, max_batch=256)
    raw.net.set_params(init_params(5))
    untrained = evaluate(raw, held_out)
    assert trained["wake_rel_rms_mean"] < 0.01 and trained["wake_within_1pct"] > 0.95
    assert untrained["wake_rel_rms_mean"] > 20 * trained["wake_rel_rms_mean"]

    lat = w.chicane()
    parts, next_id = [], 1
    for k, (n, h) in enumerate(zip([500_000, 1_200_000, 700_000, 900_000], [-12.0, -7.0, -9.0, -14.0])):
        b = w.chicane_beam(n, seed=60 + k, chirp=h)
        parts.append(Beam(b.coords, np.arange(next_id, next_id + n)))
        next_id += n
    beam = Beam(np.concatenate([p.coords for p in parts]), np.concatenate([p.ids for p in parts]))
    offsets = np.concatenate([[0], np.cumsum([p.n for p in parts])]).astype(np.int64)
    stage, sigma = {}, {}
    net16 = WakeSurrogate.load(DEFAULT_NET, max_batch=16)
    for mode in ("plain", "learned"):
        with Tracker(lat, 1000 / 0.51099895, 1) as t:
            t.load_ensemble(offsets, [])
            if mode == "learned":
                t.set_csr_surrogate(net16, tolerance=0.01, gate_stride=16)
            t.track(beam)  # warm-up
            t.set_csr_timing(True)
            res = t.track(beam)
            stage[mode] = t.csr_wake_timing()
            if mode == "learned":
                stats = t.csr_surrogate_stats()
        sigma[mode] = [res.coords[offsets[b]:offsets[b + 1], 5].std() for b in range(4)]
    assert stage["plain"]["kicks"] == stage["learned"]["kicks"] == 80
    assert stage["plain"]["learned_kicks"] == 0 and stage["learned"]["learned_kicks"] == 80
    assert stats["evaluations"] == 320 and stats["fallbacks"] <= 0.1 * stats["evaluations"]
    assert max(abs(a - b) / b for a, b in zip(sigma["learned"], sigma["plain"])) < 1e-4
    summary = {"held_out_wake_rel_rms": {"trained": trained["wake_rel_rms_mean"],
                                         "untrained": untrained["wake_rel_rms_mean"], "plain": 0.0},
               "wake_stage_ms_per_kick_4_bunches": {"plain": stage["plain"]["ms_per_kick"],
                                                    "learned": stage["learned"]["ms_per_kick"]},
               "gate_error_p95": float(np.percentile(stats["gate_errors"], 95)),
               "fallbacks": [int(stats["fallbacks"]), int(stats["evaluations"])]}
    with capsys.disabled():
        print("\nlearned wake vs plain integral:", _json.dumps(summary))
    assert stage["plain"]["ms_per_kick"] > 0 and stage["learned"]["ms_per_kick"] > 0


def test_feature_kernels_match_the_feature_definition():
    """b2e_wake_features / b2e_wake_t1_from_output against the features'
    definition written in torch (elegant_b200.wake_surrogate.Features), on
    profiles with slippages from under one bin to beyond the window."""
    import torch
    from elegant_b200.wake_surrogate import Features, build_set
    from elegant_b200.wakenet import library
    lib = library()
    data = build_set(64, 256, seed=77)
    hist, deriv, slip = data["hist"], data["deriv"], data["slip"].clone()
    slip[:4] = torch.tensor([0.3, 1.0, 255.9, 900.0], dtype=torch.float64)
    f = Features(256, 1.7, 0.6, 2.3, shift_channel=True)
    ref = f.inputs(hist, deriv, slip)
    n = hist.shape[0]
    x = torch.empty_like(ref)
    scales = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.b2e_wake_features(hist.data_ptr(), deriv.data_ptr(), slip.data_ptr(), n, 256, 1.7, 0.6, 1,
                                 x.data_ptr(), scales.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert torch.allclose(x, ref, rtol=1e-5, atol=1e-6)
    y = torch.randn((n, 256), dtype=torch.float32, device="cuda")
    t1 = torch.empty((n, 256), dtype=torch.float64, device="cuda")
    assert lib.b2e_wake_t1_from_output(y.data_ptr(), scales.data_ptr(), slip.data_ptr(), n, 256, 2.3, t1.data_ptr(),
                                       stream) == 0
    torch.cuda.synchronize()
    want = f.t1_from_output(y, hist, deriv)
    want[slip < 1] = 0
    assert torch.allclose(t1, want, rtol=1e-10, atol=0)
