"""Throughput benchmark: particle-turns/s of FP64 ring tracking.

Workload (one GPU): the batched error ensemble -- 512 instances of the 8-cell
3 GeV FODO ring with seeded quadrupole offsets and quadrupole/sextupole
strength errors, 500-4000 particles per instance (~1.15 M particles), tracked
in one fused launch per step.  A step is ``--turns-per-step`` passes (100 by
default) continuing the same run; ``--steps`` steps are timed after
``--warmup`` untimed ones.

- value: particle-turns/s with particles resident in HBM (b2e_track),
  timed with CUDA events on the engine's stream, L2 flushed before each step.
- e2e: the same metric through the C ABI with host buffers (b2e_track_host:
  pinned-host -> device copy, tracking of a fresh run, device -> host copy,
  all inside the timed region).
- roofline: FP64; algorithmic FP64 operations per particle-turn (the
  reference's formulas for this lattice, each elementary-function call at a
  fixed weight: elegant_b200/flops.py) over the FP64 DGEMM rate measured on
  this GPU in the same run.
- cpu_baseline / --impl reference: elegant's own C tracking code
  (oracle/_ref, compiled from the reference sources) on the host cores.

Multi-GPU (torchrun): every rank tracks its own full ensemble (different
seed): weak scaling, no data-path collective; time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-turns/s (FP64)"
# dram__bytes_read.sum + dram__bytes_write.sum of one ring_kernel launch on the
# 512-instance ensemble (71.45 MB + 20.33 MB; the latest capture in profiles/)
RING_TRAFFIC_BYTES = 91_491_328
UNIT = "particle-turns/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--turns-per-step", type=int, default=100)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-csr", action="store_true")
    ap.add_argument("--no-history", action="store_true", help="do not record the per-instance pass history")
    ap.add_argument("--ring-variant", type=int, default=0, help="0 = autotune, else a fixed ring-kernel variant")
    ap.add_argument("--csr-particles", type=int, default=1_000_000)
    ap.add_argument("--no-surrogate", action="store_true", help="skip the wake-network evaluation")
    ap.add_argument("--no-bunch-train", action="store_true", help="skip the 16-bunch chicane")
    return ap.parse_args()


def csr_section(args, device, flush):
    """Secondary figure: CSR pass time on the single-pass chicane (
    1 GeV, 1 nC, 1e6 particles, 4 CSRCSBEND x 20 kicks, BINS=600,
    SG_HALFWIDTH=2, CSRDRIFT 5/1/5 m).  A run is the whole chicane; the CSR
    pass time is its device time divided by the 80 dipole kicks (each kick =
    slice integration + binning + smoothing + wake + kick)."""
    import torch

    from elegant_b200 import Tracker, workloads as w

    lat = w.chicane()
    beam = w.chicane_beam(args.csr_particles, seed=777)
    p0 = 1000 / 0.51099895
    tr = Tracker(lat, p0, 1, device=device)
    stream = torch.cuda.ExternalStream(tr.stream)
    times = []
    for it in range(3 + 3):
        tr.upload(beam)
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        tr.continue_tracking()
        e1.record(stream)
        e1.synchronize()
        if it >= 3:
            times.append(e0.elapsed_time(e1))
    kicks = sum(int(e.get("N_SLICES")) for e in lat.elements if e.type == "CSRCSBEND")
    ms = sum(times) / len(times)
    tr.close()
    return {"workload": "bunch-compressor chicane with CSR, 1 GeV, 1 nC", "particles": beam.n, "dipole_kicks": kicks,
            "run_ms": ms, "csr_pass_ms_per_kick": ms / kicks,
            "particle_kicks_per_s": beam.n * kicks / (ms / 1e3),
            "timing": "CUDA events on the engine stream; includes CSRDRIFT kicks and the one host sync per CSR element"}


def single_ring_section(args, flush):
    """Secondary figure: the single 8-cell ring, 10,000 particles, 1,000 turns
    in one run (one launch after the pass-0 RFCA fiducial)."""
    import torch

    from elegant_b200 import Tracker, workloads as w

    lat, beam = w.fodo_ring(), w.ring_beam(10000, seed=12345)
    with Tracker(lat, w.ring_p_central(), 1000) as t:
        stream = torch.cuda.ExternalStream(t.stream)
        times, eff = [], 0.0
        for it in range(2 + 3):
            t.upload(beam)
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eff = t.continue_tracking()
            e1.record(stream)
            e1.synchronize()
            if it >= 2:
                times.append(e0.elapsed_time(e1))
        res = t.download()
    ms = sum(times) / len(times)
    return {"workload": "single 8-cell FODO ring, 10,000 particles, 1,000 turns", "run_ms": ms,
            "particle_turns_per_s": eff / (ms / 1e3), "survivors": int(res.n_left),
            "note": "78 tiles of 128 particles occupy 78 of 148 SMs: the ensemble is the full-GPU figure"}


def surrogate_section(args):
    """Secondary figure: the shipped wake network (elegant_b200/data) on 10,000
    fresh profiles (a seed the training never used): rms wake error against
    the FP64 integral, and device time of the surrogate path against the
    plain integral (batched and one profile)."""
    import json as _json

    from elegant_b200 import wake_surrogate as ws
    from elegant_b200.bunch_train import DEFAULT_NET

    sur = ws.WakeSurrogate.load(DEFAULT_NET, max_batch=256)
    data = ws.build_set(10_000, sur.features.bins, seed=9001)
    ev = ws.evaluate(sur, data)
    meta = _json.load(open(DEFAULT_NET.replace(".npz", ".json")))
    return {"workload": "wake network, 1024 bins, 6 conv layers x 64 channels x 5 taps, BF16/FP32 on tcgen05",
            "eval": ev, "timing_batch": ws.timing(sur, data, 8192), "timing_single": ws.timing(sur, data, 1, reps=50),
            "training": {k: meta[k] for k in ("train_profiles", "epochs", "train_s", "train_step_ms", "steps")}}


def bunch_train_section(args):
    """Secondary figure: 16 bunches (0.5-4 M particles, chirp -15..-5 /m)
    through the CSR chicane in one run, plain FP64 wake against the learned
    wake with its per-kick gate (1 %)."""
    from elegant_b200 import bunch_train

    return bunch_train.run(reps=2, warmup=1)


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thr = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thr = threading.Thread(target=self._run, daemon=True)
        self._thr.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thr:
            self._thr.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        mx = max(float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


# ------------------------------------------------------------ CPU oracle ----
def _ref_worker(args):
    """Track a slice of ensemble instances with the reference's C code (libm)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from reforacle import RefOracle
    from elegant_b200 import workloads as w
    from elegant_b200.lattice import Element, Lattice

    inst_list, n_instances, turns, seed, max_particles = args
    lat, beam, offsets, overrides = w.ensemble(n_instances=n_instances, seed=seed)
    oracle = RefOracle("libm")
    effort = 0.0
    t0 = time.perf_counter()
    for i in inst_list:
        els = []
        for j, e in enumerate(lat.elements):
            params = dict(e.params)
            for (ie, name, vals) in overrides:
                if ie == j:
                    params[name] = float(vals[i])
            els.append(Element(e.name, e.type, params))
        sl = slice(offsets[i], min(offsets[i + 1], offsets[i] + max_particles))
        _, _, eff, _ = oracle.track(Lattice(els), beam.coords[sl], beam.ids[sl], w.ring_p_central(), turns)
        effort += eff
    return effort, time.perf_counter() - t0


def cpu_reference_rate(n_instances: int, seed: int, target_seconds: float, cores: int):
    """Particle-turns/s of the reference C code on `cores` host processes over a
    bounded sample: `cores` instances, each capped at a particle count sized
    so one process runs for about `target_seconds`."""
    rate_per_core = 1.6e4  # calibration guess, refined by the measurement itself
    turns = 100  # the GPU step's pass count
    max_particles = max(50, int(target_seconds * rate_per_core / turns))
    insts = [[i] for i in range(cores)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_worker, [(il, n_instances, turns, seed, max_particles) for il in insts])
    wall = time.perf_counter() - t0
    effort = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    return effort / busy, {"cores": cores, "turns": turns, "particles_per_instance_cap": max_particles,
                           "instances": cores, "effort": effort, "busy_s": busy, "wall_s": wall}


# ------------------------------------------------------------------ main ----
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, world, rank)

    import numpy as np
    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from elegant_b200 import Tracker, workloads as w
    from elegant_b200.flops import ELEMENTARY_WEIGHT, counts_per_particle_turn, flops_per_particle_turn

    seed = 2024 + 1000 * rank
    lat, beam, offsets, overrides = w.ensemble(n_instances=args.instances, seed=seed)
    n = beam.n
    tracker = Tracker(lat, w.ring_p_central(), args.turns_per_step, device=local_rank,
                      record_history=not args.no_history, ring_variant=args.ring_variant)
    tracker.load_ensemble(offsets, overrides)
    stream = torch.cuda.ExternalStream(tracker.stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # ---- device-resident run: upload once, then continue the run step by step
    tracker.upload(beam)
    for _ in range(args.warmup):
        tracker.continue_tracking()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = tracker.launches
    step_ms = []
    effort_total = 0.0
    with ClockSampler(local_rank) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            effort_total += tracker.continue_tracking()
            ev1.record(stream)
            ev1.synchronize()
            step_ms.append(ev0.elapsed_time(ev1))
    torch.cuda.synchronize()
    launches = tracker.launches - launches0
    variant, tune_ms = tracker.ring_tuning()
    history = None
    if not args.no_history:
        h = tracker.history()
        history = {"recorded": "per instance and pass: survivors, <x>, <y>, rms emittances",
                   "passes": int(h["ex"].shape[1]),
                   "final_survival": float(h["survivors"][:, -1].sum() / n),
                   "final_ex_median_m": float(np.median(h["ex"][:, -1])),
                   "final_ey_median_m": float(np.median(h["ey"][:, -1]))}
    t_total = sum(step_ms) / 1e3
    if dist:
        tt = torch.tensor([t_total, effort_total], dtype=torch.float64, device="cuda")
        tmax = tt.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        dist.all_reduce(tt, op=dist.ReduceOp.SUM)
        t_job, effort_job = float(tmax[0]), float(tt[1])
    else:
        t_job, effort_job = t_total, effort_total
    value = effort_job / t_job

    # ---- roofline: FP64 operations per particle-turn over measured DGEMM rate
    fpt = flops_per_particle_turn(lat)
    achieved_tflops = effort_total * fpt / t_total / 1e12
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.mm(a, a)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.mm(a, a)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    fp64_peak = 2 * 8192 ** 3 / best / 1e12
    del a

    # ---- e2e: host buffers through the C ABI, fresh run per step
    e2e = None
    if not args.no_e2e:
        pinned = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(6)]
        ids = torch.empty(n, dtype=torch.int64, pin_memory=True)
        lp = torch.empty(n, dtype=torch.int32, pin_memory=True)
        le = torch.empty(n, dtype=torch.int32, pin_memory=True)
        src = torch.from_numpy(beam.coords)
        src_ids = torch.from_numpy(beam.ids)

        def e2e_step():
            for c in range(6):
                pinned[c].copy_(src[:, c])
            ids.copy_(src_ids)
            return tracker.track_host_pointers([p.data_ptr() for p in pinned], ids.data_ptr(), n, lp.data_ptr(),
                                               le.data_ptr())

        e2e_step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e2e_ms = []
        e2e_eff = 0.0
        for _ in range(max(1, min(args.steps, 5))):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, eff = e2e_step()
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            e2e_eff += eff
        t_e2e = sum(e2e_ms) / 1e3
        if dist:
            tt = torch.tensor([t_e2e, e2e_eff], dtype=torch.float64, device="cuda")
            tmax = tt.clone()
            dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
            dist.all_reduce(tt, op=dist.ReduceOp.SUM)
            t_e2e, e2e_eff = float(tmax[0]), float(tt[1])
        e2e = {"value": e2e_eff / t_e2e, "unit": UNIT, "h2d_bytes_per_step": int(n * (6 * 8 + 8)),
               "d2h_bytes_per_step": int(n * (6 * 8 + 8 + 4 + 4)), "steps": len(e2e_ms),
               "ms_per_step": sum(e2e_ms) / len(e2e_ms), "timing": "host wall clock around the blocking C-ABI call"}

    csr = None if args.no_csr else csr_section(args, local_rank, flush)
    single = None if world > 1 else single_ring_section(args, flush)
    surrogate = None if (args.no_surrogate or world > 1) else surrogate_section(args)
    train = None if (args.no_bunch_train or world > 1) else bunch_train_section(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        rate, info = cpu_reference_rate(args.instances, 2024, args.cpu_seconds, cores)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
               "sample": f"elegant's own C tracking (oracle/_ref, glibc libm), {info['instances']} ensemble "
                         f"instances x <= {info['particles_per_instance_cap']} particles x {info['turns']} turns, "
                         f"one process per core; busy {info['busy_s']:.1f} s"}

    if dist:
        dist.barrier()
    tracker.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_job * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched error ensemble of the 8-cell FODO ring",
                       "instances_per_gpu": args.instances, "particles_per_gpu": n,
                       "history": history,
                       "turns_per_step": args.turns_per_step, "lattice_elements": len(lat),
                       "ring_variant": variant, "autotune_ms_per_pass": [round(x, 3) for x in tune_ms],
                       "l2": "flushed (256 MiB write) before every timed step"},
            "roofline": {"bound": "fp64", "achieved": achieved_tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": achieved_tflops / fp64_peak, "traffic": RING_TRAFFIC_BYTES,
                         "traffic_note": "DRAM read+write bytes of one ring launch (ncu, full-size ensemble: "
                                         "profiles/ring_kernel_ensemble.md); the coordinates once per launch",
                         "algorithmic_bytes_per_launch": int(n * 96),
                         "flops_per_particle_turn": fpt,
                         "flop_model": {"arithmetic": counts_per_particle_turn(lat)[0],
                                        "elementary_calls": counts_per_particle_turn(lat)[1],
                                        "elementary_weight": ELEMENTARY_WEIGHT,
                                        "source": "elegant_b200/flops.py: the reference's formulas, +-*/ and sqrt "
                                                  "1 each, each sin/cos/asin/tan call a fixed 20"},
                         "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 (torch.mm float64), best of 3"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks.summary(),
            "single_ring": single, "csr": csr, "wake_surrogate": surrogate, "bunch_train": train,
        }
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_reference(args, world, rank):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    steps = []
    effort_total = 0.0
    for _ in range(args.warmup):
        cpu_reference_rate(args.instances, 2024, min(2.0, args.cpu_seconds), cores)
    t_sum = 0.0
    info = None
    for _ in range(args.steps):
        rate, info = cpu_reference_rate(args.instances, 2024, args.cpu_seconds / 2, cores)
        effort_total += info["effort"]
        t_sum += info["busy_s"]
        steps.append(info["busy_s"] * 1e3)
    value = effort_total / t_sum
    sample = (f"elegant's own C tracking (oracle/_ref, glibc libm) on {cores} host processes; each step "
              f"{info['instances']} instances x <= {info['particles_per_instance_cap']} particles x "
              f"{info['turns']} turns of the ensemble ring")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum(steps) / len(steps), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batched error ensemble of the 8-cell FODO ring",
                   "instances_per_gpu": args.instances},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


if __name__ == "__main__":
    main()
