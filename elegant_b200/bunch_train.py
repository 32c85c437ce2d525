"""Bunch train through the CSR chicane: 16 bunches in one run, each with its
own histogram, wake and macro charge, the wake integral either plain (FP64)
or from the trained wake network with the per-kick gate and fallback.

The particles are generated on the device (torch as random-number plumbing)
with the distribution of workloads.chicane_beam: 6-D Gaussian, x/y matched to
beta = 10 m, normalised emittance 1 um, sigma_z = 1 mm, uncorrelated
sigma_delta = 1e-4 plus the bunch's linear chirp.  Tracking runs through
b2e_track_device on those device buffers (particles stay resident in HBM).
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import workloads as w
from .beam import p_central_from_momentum_mev
from .track import Tracker

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_NET = os.path.join(HERE, "data", "wakenet_1024.npz")


def make_train(n_bunches: int = 16, n_min: int = 500_000, n_max: int = 4_000_000, chirp=(-15.0, -5.0),
               seed: int = 4242, device="cuda"):
    """Per-bunch sizes and chirps, offsets, and the SoA columns on the device."""
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = rng.integers(n_min, n_max + 1, size=n_bunches)
    chirps = rng.uniform(chirp[0], chirp[1], size=n_bunches)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    n = int(offsets[-1])
    p = p_central_from_momentum_mev(w.CHICANE_P_MEV)
    eps, beta = 1e-6 / p, 10.0
    cols = [torch.empty(n, dtype=torch.float64, device=device) for _ in range(6)]
    g = torch.Generator(device=device)
    for b in range(n_bunches):
        g.manual_seed(seed * 1009 + b)
        sl = slice(int(offsets[b]), int(offsets[b + 1]))
        z = torch.randn((6, int(sizes[b])), generator=g, dtype=torch.float64, device=device)
        z -= z.mean(dim=1, keepdim=True)
        cols[0][sl] = math.sqrt(eps * beta) * z[0]
        cols[1][sl] = math.sqrt(eps / beta) * z[1]
        cols[2][sl] = math.sqrt(eps * beta) * z[2]
        cols[3][sl] = math.sqrt(eps / beta) * z[3]
        cols[4][sl] = 1e-3 * z[4]
        cols[5][sl] = 1e-4 * z[5] + chirps[b] * cols[4][sl]
    return sizes, chirps, offsets, cols


def bunch_moments(cols, lost, offsets):
    """Per bunch: survivors, rms energy spread, rms emittance in x (geometric)."""
    import torch
    out = []
    for b in range(len(offsets) - 1):
        sl = slice(int(offsets[b]), int(offsets[b + 1]))
        alive = lost[sl] < 0
        x, xp, d = cols[0][sl][alive], cols[1][sl][alive], cols[5][sl][alive]
        dx, dxp = x - x.mean(), xp - xp.mean()
        ex = torch.sqrt(torch.clamp((dx * dx).mean() * (dxp * dxp).mean() - (dx * dxp).mean() ** 2, min=0))
        out.append({"survivors": int(alive.sum()), "sigma_delta": float(d.std(unbiased=False)), "emit_x": float(ex)})
    return out


def run(n_bunches=16, n_min=500_000, n_max=4_000_000, net_path=DEFAULT_NET, tolerance=0.01, gate_stride=16,
        reps=2, warmup=1, seed=4242, bins=600, n_kicks=20):
    """Plain and learned-wake runs of the same bunch train; times are device
    time per run (CUDA events on the engine stream, particles resident)."""
    import torch
    from .wake_surrogate import WakeSurrogate
    sizes, chirps, offsets, init = make_train(n_bunches, n_min, n_max, seed=seed)
    n = int(offsets[-1])
    lat = w.chicane(bins=bins, n_kicks=n_kicks)
    p0 = p_central_from_momentum_mev(w.CHICANE_P_MEV)
    kicks = 4 * n_kicks
    cols = [torch.empty_like(c) for c in init]
    lost = torch.empty(n, dtype=torch.int32, device="cuda")
    lost_e = torch.empty(n, dtype=torch.int32, device="cuda")
    sur = WakeSurrogate.load(net_path, max_batch=max(16, n_bunches))
    result = {"bunches": n_bunches, "particles": n, "sizes": [int(x) for x in sizes],
              "chirps": [float(x) for x in chirps], "dipole_kicks": kicks, "bins": bins}
    for mode in ("plain", "surrogate"):
        with Tracker(lat, p0, 1) as t:
            t.load_ensemble(offsets, [])
            if mode == "surrogate":
                t.set_csr_surrogate(sur, tolerance=tolerance, gate_stride=gate_stride)
            stream = torch.cuda.ExternalStream(t.stream)
            times = []
            for it in range(warmup + reps):
                for c, c0 in zip(cols, init):
                    c.copy_(c0)
                lost.fill_(-1)
                lost_e.fill_(-1)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                t.track_device(cols, lost, lost_e)
                e1.record(stream)
                e1.synchronize()
                if it >= warmup:
                    times.append(e0.elapsed_time(e1))
            ms = sum(times) / len(times)
            r = {"run_ms": ms, "particle_kicks_per_s": n * kicks / (ms / 1e3), "per_bunch": bunch_moments(cols, lost,
                                                                                                      offsets)}
            # one more run with the wake stage of every kick bracketed by
            # events: the engine's own per-kick cost of this path's wake
            # (plain kernel, or filter + network + combine), all bunches
            for c, c0 in zip(cols, init):
                c.copy_(c0)
            lost.fill_(-1)
            lost_e.fill_(-1)
            t.set_csr_timing(True)
            t.track_device(cols, lost, lost_e)
            wt = t.csr_wake_timing()
            t.set_csr_timing(False)
            r["wake_stage_ms_per_kick"] = wt["ms_per_kick"]
            r["wake_stage_kicks"] = wt["kicks"]
            r["wake_stage_learned_kicks"] = wt["learned_kicks"]
            if mode == "surrogate":
                st = t.csr_surrogate_stats()
                errs = st["gate_errors"]
                r.update({"evaluations": st["evaluations"], "fallbacks": st["fallbacks"],
                          "gate_error_median": float(np.median(errs)) if errs.size else None,
                          "gate_error_p95": float(np.percentile(errs, 95)) if errs.size else None,
                          "tolerance": tolerance, "gate_stride": gate_stride})
            result[mode] = r
    pb, sb = result["plain"]["per_bunch"], result["surrogate"]["per_bunch"]
    result["sigma_delta_rel_diff_max"] = max(abs(s["sigma_delta"] - p["sigma_delta"]) / p["sigma_delta"]
                                             for p, s in zip(pb, sb))
    result["emit_x_rel_diff_max"] = max(abs(s["emit_x"] - p["emit_x"]) / p["emit_x"] for p, s in zip(pb, sb))
    result["surrogate_vs_plain_time"] = result["surrogate"]["run_ms"] / result["plain"]["run_ms"]
    result["wake_stage_learned_vs_plain_time"] = (result["surrogate"]["wake_stage_ms_per_kick"] /
                                                  result["plain"]["wake_stage_ms_per_kick"])
    return result


if __name__ == "__main__":
    import json
    print(json.dumps(run()))
