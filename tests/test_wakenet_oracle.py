"""CPU checks of the wake-network oracle (oracle/wakenet_oracle.py) and of the
standalone wake-integral restatement used to label its data."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import wakenet_oracle as wo  # noqa: E402
from elegant_b200.wakenet import init_params  # noqa: E402


def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(0).normal(0, 3, 10000) * 10.0 ** np.random.default_rng(1).integers(-20, 20, 10000)
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(wo.bf16(x), ref)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    dil = (1, 2, 3, 1, 2, 1)
    params = init_params(11, out_scale=1.0).astype(np.float64)
    params[wo.LAYERS * wo.WSIZE:] = rng.normal(0, 0.1, wo.LAYERS * wo.CH)
    inputs = rng.normal(0, 1, (2, 4, 24))
    targets = rng.normal(0, 1, (2, 24))
    loss, g = wo.loss_and_gradients(params, inputs, targets, dil, use_bf16=False)
    w_idx = [l * wo.WSIZE + (t * 64 + co) * 64 + ci for l, t, co, ci in
             [(0, 0, 5, 1), (0, 4, 63, 2), (1, 2, 7, 9), (2, 1, 30, 40), (3, 3, 1, 0), (4, 0, 60, 61),
              (5, 2, 0, 17), (5, 4, 0, 63)]]
    b_idx = [wo.LAYERS * wo.WSIZE + l * 64 + c for l, c in [(0, 3), (2, 50), (4, 0), (5, 0)]]
    for i in w_idx + b_idx:
        h = 1e-6
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        l1, _ = wo.loss_and_gradients(p1, inputs, targets, dil, use_bf16=False)
        l2, _ = wo.loss_and_gradients(p2, inputs, targets, dil, use_bf16=False)
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_wake_t1_restatement_properties():
    """Linear in the counts; zero for zero slippage; the steady-state integral
    equals the transient one once the slippage covers every bin."""
    from reforacle import PortOracle
    o = PortOracle("b2e")
    i = np.arange(256)
    counts = 1e4 * np.exp(-0.5 * ((i - 120) / 15.0) ** 2)
    t1, h, d = o.wake_t1(counts, 40.0, sg_half=2, sg_order=1)
    t1b, _, _ = o.wake_t1(3 * counts, 40.0, sg_half=2, sg_order=1)
    np.testing.assert_allclose(t1b, 3 * t1, rtol=1e-12, atol=1e-12 * np.abs(t1).max())
    z, _, _ = o.wake_t1(counts, 0.5, sg_half=2, sg_order=1)
    assert not z.any()
    s1, _, _ = o.wake_t1(counts, 1e6, sg_half=0, trapz=False)
    s2, _, _ = o.wake_t1(counts, 0.0, sg_half=0, trapz=False, steady=True)
    np.testing.assert_allclose(s1, s2, rtol=0, atol=1e-12 * np.abs(s2).max())
    assert abs(h.sum() - counts.sum()) < 1e-9 * counts.sum()
