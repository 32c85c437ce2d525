"""Learned CSR wake integral: data set, training driver and evaluation.

The surrogate replaces the O(bins x slippage) integral term T1 of the
CSRCSBEND kick wake (csbend.c:2623-2673); the boundary term T2 and the
smoothing / derivative filters stay exact.  In bin units (bin width 1, CSR
constant 1) the kick wake is

    W[i] = T1[i] - (hist[i + diS] - hist[i + diS4]) / s^(1/3),

s the slippage in bins, diS = floor(s), diS4 = floor(4 s); a kick of bin width
dct scales it by CSRConstant * L / N_KICKS * dct^(-4/3) (b2e_csr_wake_batch).
T1 is linear in the histogram and depends on the profile only through its
smoothed density and derivative and on the slippage only through diS.

Network inputs per bin (channels): density and derivative of the histogram
normalised to unit sum, both multiplied by k = 1 / rms(derivative) of that
profile and by fixed channel scales, the code log2(diS) / log2(bins), and the
density at bin i + diS (the far end of the integral, zero past the last bin)
scaled like the density.  The
target is T1 / N * k * target scale, so the squared error weighs every profile
by its relative error.  All compute runs in the engine's kernels; torch is the
driver's device-buffer and random-number plumbing.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import _native as nat
from .wakenet import DILATIONS, WakeNet, init_params, library

MM = 1e-3


# ---------------------------------------------------------------- profiles ----
def sample_profile_params(n: int, seed: int):
    """Gaussian mixtures (1-4 components), sigma 0.2-2 mm, centres within
    +-3 mm, Dirichlet(1) weights; bend radius 5-50 m; particle count
    log-uniform 0.5M-4M; slippage (in bins) log-uniform in [1, 2 * bins];
    binning window widened by a factor 1.2-2.2 (tracking bins a bunch on its
    own extent, and a histogram of fewer bins than the network's is padded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    k = rng.integers(1, 5, size=n)
    sig = rng.uniform(0.2, 2.0, size=(n, 4)) * MM
    cen = rng.uniform(-3.0, 3.0, size=(n, 4)) * MM
    w = rng.gamma(1.0, size=(n, 4))
    w[np.arange(4)[None, :] >= k[:, None]] = 0
    w /= w.sum(axis=1, keepdims=True)
    rho = rng.uniform(5.0, 50.0, size=n)
    npart = np.exp(rng.uniform(np.log(5e5), np.log(4e6), size=n))
    slip_u = rng.uniform(0, 1, size=n)
    widen = rng.uniform(1.2, 2.2, size=n)
    return dict(k=k, sigma=sig, centre=cen, weight=w, rho=rho, n_particles=npart, slip_u=slip_u, widen=widen)


def make_histograms(params: dict, bins: int, seed: int, device="cuda", chunk: int = 16384):
    """Bin-integrated mixture densities on each profile's own window (the
    +-4.5 sigma extent of its components, widened by the profile's factor),
    times the particle count, plus Gaussian shot noise
    of variance = count.  Returns (counts [n][bins] float64, slippage in bins,
    bin width in m).  Works in chunks of `chunk` profiles, each with its own
    seeded noise stream."""
    import torch
    n = len(params["k"])
    counts = torch.empty((n, bins), dtype=torch.float64, device=device)
    dct_all = torch.empty(n, dtype=torch.float64, device=device)
    ar = torch.arange(bins + 1, dtype=torch.float64, device=device)[None, :]
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        sig, cen, w = (torch.tensor(params[x][c0:c1], dtype=torch.float64, device=device)
                       for x in ("sigma", "centre", "weight"))
        live = w > 0
        lo = torch.where(live, cen - 4.5 * sig, torch.full_like(cen, 1e9)).min(dim=1).values
        hi = torch.where(live, cen + 4.5 * sig, torch.full_like(cen, -1e9)).max(dim=1).values
        widen = torch.tensor(params["widen"][c0:c1], dtype=torch.float64, device=device)
        mid, half = (lo + hi) / 2, (hi - lo) / 2 * widen
        lo = mid - half
        dct = 2 * half / bins
        edges = lo[:, None] + dct[:, None] * ar
        cdf = 0.5 * (1 + torch.erf((edges[:, :, None] - cen[:, None, :]) / (sig[:, None, :] * math.sqrt(2))))
        dens = ((cdf[:, 1:, :] - cdf[:, :-1, :]) * w[:, None, :]).sum(dim=2)
        npart = torch.tensor(params["n_particles"][c0:c1], dtype=torch.float64, device=device)
        cts = dens * npart[:, None]
        g = torch.Generator(device=device)
        g.manual_seed(seed * 1000003 + c0)
        noise = torch.randn(cts.shape, generator=g, dtype=torch.float64, device=device)
        counts[c0:c1] = torch.clamp(cts + noise * torch.sqrt(cts), min=0)
        dct_all[c0:c1] = dct
    slip_bins = torch.exp(torch.tensor(params["slip_u"], dtype=torch.float64, device=device) * math.log(2 * bins))
    return counts, slip_bins.contiguous(), dct_all


def wake_batch(counts, slip_bins, sg_half=2, sg_order=1, trapz=True, steady=False):
    """T1, smoothed density and derivative (engine FP64 kernel)."""
    import torch
    n, nb = counts.shape
    t1, h, d = (torch.empty((n, nb), dtype=torch.float64, device=counts.device) for _ in range(3))
    lib = library()
    for s in range(0, n, 65536):
        e = min(n, s + 65536)
        rc = lib.b2e_csr_wake_batch(counts[s:e].data_ptr(), slip_bins[s:e].data_ptr(), e - s, nb, sg_half, sg_order,
                                    0, 0, int(trapz), int(steady), t1[s:e].data_ptr(), h[s:e].data_ptr(),
                                    d[s:e].data_ptr(), torch.cuda.current_stream().cuda_stream)
        if rc != nat.B2E_OK:
            raise nat.EngineError(rc, "b2e_csr_wake_batch failed")
    return t1, h, d


def boundary_term(hist, slip_bins):
    """T2 part of the bin-unit wake: -(hist[i+diS] - hist[i+diS4]) / s^(1/3)."""
    import torch
    n, nb = hist.shape
    i = torch.arange(nb, device=hist.device)[None, :]
    dis = torch.clamp(torch.floor(slip_bins), 0, nb).long()[:, None]
    dis4 = torch.clamp(torch.floor(4 * slip_bins), 0, nb).long()[:, None]
    pad = torch.cat([hist, torch.zeros((n, 1), dtype=hist.dtype, device=hist.device)], dim=1)
    a = torch.gather(pad, 1, torch.clamp(i + dis, max=nb))
    b = torch.gather(pad, 1, torch.clamp(i + dis4, max=nb))
    return -(a - b) / torch.pow(slip_bins, 1.0 / 3.0)[:, None]


# --------------------------------------------------------------- features ----
class Features:
    """Maps (density, derivative, slippage) to network inputs and T1 to targets."""

    def __init__(self, bins: int, dens_scale=1.0, deriv_scale=1.0, target_scale=1.0, shift_channel=True):
        self.bins, self.dens_scale, self.deriv_scale, self.target_scale = bins, dens_scale, deriv_scale, target_scale
        self.shift_channel = shift_channel

    def sample_scale(self, hist, deriv):
        import torch
        total = hist.sum(dim=1, keepdim=True).clamp_min(1e-300)
        dnorm = deriv / total
        k = 1.0 / torch.sqrt((dnorm * dnorm).mean(dim=1, keepdim=True)).clamp_min(1e-300)
        return total, k

    def inputs(self, hist, deriv, slip_bins):
        import torch
        total, k = self.sample_scale(hist, deriv)
        n, nb = hist.shape
        x = torch.empty((n, 4, nb), dtype=torch.float32, device=hist.device)
        dn = hist / total * k * self.dens_scale
        x[:, 0] = dn.float()
        x[:, 1] = (deriv / total * k * self.deriv_scale).float()
        dis = torch.clamp(torch.floor(slip_bins), 1, nb)
        x[:, 2] = (torch.log2(dis) / math.log2(nb)).float()[:, None]
        if self.shift_channel:
            idx = torch.arange(nb, device=hist.device)[None, :] + dis.long()[:, None]
            pad = torch.cat([dn, torch.zeros((n, 1), dtype=dn.dtype, device=dn.device)], dim=1)
            x[:, 3] = torch.gather(pad, 1, torch.clamp(idx, max=nb)).float()
        else:
            x[:, 3] = 0
        return x

    def targets(self, t1, hist, deriv):
        total, k = self.sample_scale(hist, deriv)
        return (t1 / total * k * self.target_scale).float()

    def t1_from_output(self, y, hist, deriv):
        total, k = self.sample_scale(hist, deriv)
        return y.double() / self.target_scale / k * total

    def fit(self, hist, deriv, t1, slip_bins):
        """Channel scales giving unit RMS over a sample of the data."""
        import torch
        self.dens_scale = self.deriv_scale = self.target_scale = 1.0
        x = self.inputs(hist, deriv, slip_bins)
        t = self.targets(t1, hist, deriv)
        self.dens_scale = float(1.0 / torch.sqrt((x[:, 0].double() ** 2).mean()))
        self.deriv_scale = float(1.0 / torch.sqrt((x[:, 1].double() ** 2).mean()))
        self.target_scale = float(1.0 / torch.sqrt((t.double() ** 2).mean()))

    def state(self):
        return dict(bins=self.bins, dens_scale=self.dens_scale, deriv_scale=self.deriv_scale,
                    target_scale=self.target_scale, shift_channel=int(self.shift_channel))


class WakeSurrogate:
    """Trained network plus its feature scales."""

    def __init__(self, bins=1024, max_batch=256, dilations=DILATIONS, device=0):
        self.net = WakeNet(bins=bins, max_batch=max_batch, dilations=dilations, device=device)
        self.features = Features(bins)

    def save(self, path):
        np.savez(path, params=self.net.params(), dilations=np.array(self.net.dilations),
                 **{k: np.array(v) for k, v in self.features.state().items()})

    @classmethod
    def load(cls, path, max_batch=256, device=0):
        z = np.load(path)
        s = cls(bins=int(z["bins"]), max_batch=max_batch, dilations=tuple(int(d) for d in z["dilations"]),
                device=device)
        s.net.set_params(z["params"])
        s.features = Features(int(z["bins"]), float(z["dens_scale"]), float(z["deriv_scale"]),
                              float(z["target_scale"]), bool(int(z["shift_channel"])))
        return s

    def predict_t1(self, hist, deriv, slip_bins):
        """T1 of every profile by the network: the engine's feature kernel,
        the network, and its back-transform kernel, with no host-side glue."""
        import torch
        n, nb = hist.shape
        f = self.features
        lib = self.net.lib
        stream = torch.cuda.current_stream().cuda_stream
        x = torch.empty((n, 4, nb), dtype=torch.float32, device=hist.device)
        scales = torch.empty((n, 2), dtype=torch.float64, device=hist.device)
        t1 = torch.empty((n, nb), dtype=torch.float64, device=hist.device)
        hist, deriv, slip_bins = hist.contiguous(), deriv.contiguous(), slip_bins.contiguous()
        rc = lib.b2e_wake_features(hist.data_ptr(), deriv.data_ptr(), slip_bins.data_ptr(), n, nb, f.dens_scale,
                                   f.deriv_scale, int(f.shift_channel), x.data_ptr(), scales.data_ptr(), stream)
        if rc != nat.B2E_OK:
            raise nat.EngineError(rc, "b2e_wake_features failed")
        y = self.net.forward(x)
        rc = lib.b2e_wake_t1_from_output(y.data_ptr(), scales.data_ptr(), slip_bins.data_ptr(), n, nb,
                                         f.target_scale, t1.data_ptr(), stream)
        if rc != nat.B2E_OK:
            raise nat.EngineError(rc, "b2e_wake_t1_from_output failed")
        return t1


# ---------------------------------------------------------------- training ----
def build_set(n, bins, seed, sg_half=2):
    p = sample_profile_params(n, seed)
    counts, slip, dct = make_histograms(p, bins, seed + 1)
    t1, hist, deriv = wake_batch(counts, slip, sg_half=sg_half)
    return dict(counts=counts, slip=slip, dct=dct, t1=t1, hist=hist, deriv=deriv, params=p)


def rel_rms(a, b):
    import torch
    return torch.sqrt(((a - b) ** 2).mean(dim=1)) / torch.sqrt((b ** 2).mean(dim=1)).clamp_min(1e-300)


def evaluate(sur: WakeSurrogate, data: dict) -> dict:
    import torch
    t1p = sur.predict_t1(data["hist"], data["deriv"], data["slip"])
    t2 = boundary_term(data["hist"], data["slip"])
    w_ref, w_sur = data["t1"] + t2, t1p + t2
    e_w = rel_rms(w_sur, w_ref).cpu().numpy()
    e_t1 = rel_rms(t1p, data["t1"]).cpu().numpy()
    return {"profiles": int(len(e_w)),
            "wake_rel_rms_mean": float(e_w.mean()), "wake_rel_rms_median": float(np.median(e_w)),
            "wake_rel_rms_p95": float(np.percentile(e_w, 95)), "wake_within_1pct": float((e_w <= 0.01).mean()),
            "t1_rel_rms_mean": float(e_t1.mean()), "t1_rel_rms_median": float(np.median(e_t1)),
            "rms_wake_error": float(torch.sqrt(((w_sur - w_ref) ** 2).mean() / (w_ref ** 2).mean()))}


def timing(sur: WakeSurrogate, data: dict, n: int, reps: int = 5) -> dict:
    """Device time per profile: the plain FP64 wake (smoothing, derivative and
    integral) against the surrogate path (the same smoothing and derivative,
    then the feature kernel, the network and the back-transform kernel)."""
    import torch
    counts, slip = data["counts"][:n].contiguous(), data["slip"][:n].contiguous()
    zero = torch.zeros_like(slip)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    plain_ms = timed(lambda: wake_batch(counts, slip))

    def sur_fn():
        _, h, d = wake_batch(counts, zero)  # filters only: the integral loop is empty for diS = 0
        sur.predict_t1(h, d, slip)

    sur_ms = timed(sur_fn)
    return {"profiles": n, "plain_ms": plain_ms, "surrogate_ms": sur_ms, "speedup": plain_ms / sur_ms}


def train(args):
    import torch
    torch.cuda.set_device(0)
    t0 = time.time()
    train_set = build_set(args.train, args.bins, args.seed)
    test_set = build_set(args.test, args.bins, args.seed + 1000)
    t_data = time.time() - t0
    sur = WakeSurrogate(bins=args.bins, max_batch=args.batch,
                        dilations=tuple(int(x) for x in args.dilations.split(",")))
    sur.net.set_params(init_params(args.seed))
    f = sur.features
    f.shift_channel = not args.no_shift_channel
    f.fit(train_set["hist"][:4096], train_set["deriv"][:4096], train_set["t1"][:4096], train_set["slip"][:4096])
    x_all = f.inputs(train_set["hist"], train_set["deriv"], train_set["slip"])
    y_all = f.targets(train_set["t1"], train_set["hist"], train_set["deriv"])
    n = x_all.shape[0]
    steps_per_epoch = n // args.batch
    total = steps_per_epoch * args.epochs
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed)
    log = []
    step = 0
    torch.cuda.synchronize()
    t1 = time.time()
    for ep in range(args.epochs):
        perm = torch.randperm(n, generator=g, device="cuda")
        ep_loss = 0.0
        for s in range(steps_per_epoch):
            idx = perm[s * args.batch:(s + 1) * args.batch]
            xb, yb = x_all[idx].contiguous(), y_all[idx].contiguous()
            lr = args.lr_min + 0.5 * (args.lr - args.lr_min) * (1 + math.cos(math.pi * step / total))
            want = s == steps_per_epoch - 1
            l = sur.net.train_step(xb, yb, lr, want_loss=want)
            if want:
                ep_loss = l
            step += 1
        ev = evaluate(sur, {k: v[:2000] if hasattr(v, "shape") else v for k, v in test_set.items()})
        log.append({"epoch": ep + 1, "train_loss_last_batch": ep_loss, "test_wake_rel_rms_mean": ev["wake_rel_rms_mean"],
                    "test_t1_rel_rms_mean": ev["t1_rel_rms_mean"], "elapsed_s": time.time() - t1})
        print(json.dumps(log[-1]), flush=True)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    result = {"train_profiles": args.train, "test_profiles": args.test, "bins": args.bins, "epochs": args.epochs,
              "batch": args.batch, "steps": step, "data_s": t_data, "train_s": t_train,
              "train_step_ms": t_train / step * 1e3, "features": f.state(), "dilations": list(sur.net.dilations),
              "eval": evaluate(sur, test_set), "log": log}
    result["timing_batch"] = timing(sur, test_set, min(args.test, 8192))
    result["timing_single"] = timing(sur, test_set, 1, reps=50)
    if args.save:
        sur.save(args.save)
    return result


def main():
    ap = argparse.ArgumentParser(description="train the wake-network surrogate of the CSR wake integral")
    ap.add_argument("--train", type=int, default=200_000)
    ap.add_argument("--test", type=int, default=10_000)
    ap.add_argument("--bins", type=int, default=1024)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-min", type=float, default=1e-5)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--dilations", default=",".join(str(d) for d in DILATIONS))
    ap.add_argument("--no-shift-channel", action="store_true")
    ap.add_argument("--save", default="")
    ap.add_argument("--out", default="")
    args = ap.parse_args()
    res = train(args)
    txt = json.dumps(res, indent=1)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(txt)
    print(json.dumps({k: v for k, v in res.items() if k != "log"}))


if __name__ == "__main__":
    main()
