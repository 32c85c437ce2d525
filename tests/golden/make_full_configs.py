"""Golden results of elegant's own tracking code at the full sizes of the
benchmark cases, and the helpers that rebuild their inputs.

    python tests/golden/make_full_configs.py [ring] [edge] [chicane] [ensemble] [train]

runs oracle/_ref (elegant's multipole.c, csbend.c, simple_rfca.c, ... compiled
from the reference sources by oracle/Makefile.ref) on this host and writes
tests/golden/full_configs.json (+ full_ring_libm.npz, full_ensemble_history.npz:
per instance the survivors after every pass and <x>, <y>, ex, ey after every
tenth).  The GPU tests in
tests/test_gpu_full_configs.py rebuild the same inputs with the helpers below,
check the input digests, track them on the device and compare.

Cases (one per benchmark configuration that tracks particles):

- ring: 10,000 particles of the single 8-cell FODO ring, 1,000 turns.  The
  reference with the engine's elementary functions (shared maths) gives the
  bit-exact digest; the reference with glibc gives the coordinates stored in
  full_ring_libm.npz, and the same glibc run with every x moved by one ulp
  gives the ring's own sensitivity envelope.  Both runs are spread over
  particle slices with the whole beam's RFCA fiducial (reforacle.track_split).
- edge: 2,000 particles around the ring's dynamic-aperture boundary, 1,000
  turns: the loss pairs of both maths modes (and of glibc with x moved by one
  ulp), which carry the loss comparison that the matched beam (no losses)
  cannot.
- chicane: 1,000,000 particles through the four-dipole CSR chicane (BINS=600,
  SG_HALFWIDTH=2, 4 x 20 kicks, CSRDRIFT 5/1/5 m): final coordinates and the
  digest of every per-kick wake array (DeltaGamma of CSRCSBEND's OUTPUT_FILE).
- ensemble: the first 32 instances (500-4,000 particles each) of the
  512-instance error ensemble, 1,000 turns, with the per-pass history.
- train: two bunches of the bunch-train case, 500,000 and 4,000,000 particles
  with chirps -15 and -5 /m, plain wake, each tracked alone by the reference
  (a bunch's histogram and wake are its own).

Digests are SHA-256 over little-endian bytes, with -0.0 folded into +0.0
(the comparisons are of values): survivors' IDs and coordinates sorted by
ID; the sorted (ID, loss pass) pairs; each wake array.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

FIXTURE = os.path.join(HERE, "full_configs.json")
RING_LIBM = os.path.join(HERE, "full_ring_libm.npz")
ENSEMBLE_HISTORY = os.path.join(HERE, "full_ensemble_history.npz")
EDGE_LOSSES = os.path.join(HERE, "full_edge_losses.npz")
CHICANE_P0 = 1000 / 0.51099895
RING_TURNS = 1000
ENSEMBLE_INSTANCES = 32
TRAIN = {"sizes": [500_000, 4_000_000], "chirps": [-15.0, -5.0], "seeds": [4242, 4243]}


# ------------------------------------------------------------- digests ----
def _fold(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype="<f8") + 0.0


def digest_array(a) -> str:
    return hashlib.sha256(_fold(np.asarray(a, dtype=np.float64)).tobytes()).hexdigest()


def digest_beam(coords, ids) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ids, dtype="<i8").tobytes())
    h.update(_fold(coords).tobytes())
    return h.hexdigest()


def digest_survivors(coords, ids, lost_pass) -> str:
    """Survivors sorted by ID: IDs, then the six coordinates row by row."""
    order = np.argsort(ids, kind="stable")
    c, i, lp = coords[order], ids[order], lost_pass[order]
    alive = lp < 0
    return digest_beam(c[alive], i[alive])


def lost_pairs(ids, lost_pass) -> list:
    lost = lost_pass >= 0
    return sorted([int(a), int(b)] for a, b in zip(ids[lost], lost_pass[lost]))


def digest_lost(ids, lost_pass) -> str:
    return hashlib.sha256(np.asarray(lost_pairs(ids, lost_pass), dtype="<i8").tobytes()).hexdigest()


def rows_result(rows):
    """Reference rows -> (coords, ids, loss pass) in ID order."""
    order = np.argsort(rows[:, 6], kind="stable")
    r = rows[order]
    return r[:, :6].copy(), r[:, 6].astype(np.int64), r[:, 7].astype(np.int64)


# -------------------------------------------------------------- inputs ----
def twiss_from(fixture_twiss):
    from elegant_b200.optics import Twiss
    return Twiss(**fixture_twiss)


def ring_inputs(twiss):
    from elegant_b200 import workloads as w
    return w.fodo_ring(), w.ring_beam(10000, seed=12345, twiss=twiss)


def edge_inputs():
    """2,000 particles around the ring's dynamic-aperture boundary (x 12-13.3
    mm, |y| <= 3 mm, |delta| <= 0.5 %): most are lost between the first
    pass and the thousandth."""
    from elegant_b200 import workloads as w
    from elegant_b200.beam import Beam
    rng = np.random.Generator(np.random.PCG64(4711))
    n = 2000
    c = np.zeros((n, 6))
    c[:, 0] = rng.uniform(0.012, 0.0133, n) * rng.choice([-1.0, 1.0], n)
    c[:, 2] = rng.uniform(-0.003, 0.003, n)
    c[:, 5] = rng.uniform(-0.005, 0.005, n)
    c[:, 4] = rng.uniform(-0.003, 0.003, n)
    return w.fodo_ring(), Beam(c, np.arange(1, n + 1))


def chicane_inputs():
    from elegant_b200 import workloads as w
    return w.chicane(), w.chicane_beam(1_000_000, seed=777)


def ensemble_inputs(twiss):
    """The 512-instance ensemble of the benchmark; its first instances."""
    from elegant_b200 import workloads as w
    lat, beam, offsets, overrides = w.ensemble(n_instances=512, seed=2024, twiss=twiss)
    k = ENSEMBLE_INSTANCES
    n = int(offsets[k])
    from elegant_b200.beam import Beam
    sub = Beam(beam.coords[:n], beam.ids[:n])
    ovr = [(ie, name, np.asarray(vals[:k])) for ie, name, vals in overrides]
    return lat, sub, offsets[: k + 1].copy(), ovr


def instance_lattice(lat, overrides, i):
    from elegant_b200.lattice import Element, Lattice
    els = []
    for j, e in enumerate(lat.elements):
        params = dict(e.params)
        for (ie, name, vals) in overrides:
            if ie == j:
                params[name] = float(vals[i])
        els.append(Element(e.name, e.type, params))
    return Lattice(els)


def train_inputs():
    """Two bunches of the bunch-train case, IDs running on across bunches."""
    from elegant_b200 import workloads as w
    from elegant_b200.beam import Beam
    parts, next_id = [], 1
    for n, h, s in zip(TRAIN["sizes"], TRAIN["chirps"], TRAIN["seeds"]):
        b = w.chicane_beam(n, seed=s, chirp=h)
        parts.append(Beam(b.coords, np.arange(next_id, next_id + n)))
        next_id += n
    offsets = np.concatenate([[0], np.cumsum(TRAIN["sizes"])]).astype(np.int64)
    return w.chicane(), Beam(np.concatenate([p.coords for p in parts]), np.concatenate([p.ids for p in parts])), \
        offsets


def load_fixture() -> dict:
    with open(FIXTURE) as f:
        return json.load(f)


# ---------------------------------------------------------- generation ----
def _rel(a, b):
    """Per coordinate: max |a-b| / max(|a|, std of the column)."""
    scale = np.maximum(np.abs(a), a.std(axis=0) + 1e-300)
    return (np.abs(a - b) / scale).max(axis=0)


def make_ring(out):
    from elegant_b200 import workloads as w
    from elegant_b200.optics import periodic_twiss
    from reforacle import track_split
    tw = periodic_twiss(w.fodo_ring(rf=False))
    twd = {k: float(getattr(tw, k)) for k in ("beta_x", "alpha_x", "beta_y", "alpha_y", "eta_x", "etap_x")}
    lat, beam = ring_inputs(twiss_from(twd))
    p0 = w.ring_p_central()
    res = {"twiss": twd, "input": digest_beam(beam.coords, beam.ids), "turns": RING_TURNS}
    t = time.time()
    rows, nl, eff, t0 = track_split("b2e", lat, beam.coords, beam.ids, p0, RING_TURNS)
    c, ids, lp = rows_result(rows)
    res["b2e"] = {"n_left": int(nl), "effort": float(eff), "t0": t0, "survivors": digest_survivors(c, ids, lp),
                  "lost": lost_pairs(ids, lp), "seconds": time.time() - t}
    t = time.time()
    rows, nl, eff, t0l = track_split("libm", lat, beam.coords, beam.ids, p0, RING_TURNS)
    cl, idl, lpl = rows_result(rows)
    pert = beam.coords.copy()
    pert[:, 0] = np.nextafter(pert[:, 0], np.inf)
    rows, nlp, _, _ = track_split("libm", lat, pert, beam.ids, p0, RING_TURNS)
    cp, _, lpp = rows_result(rows)
    alive = (lpl < 0) & (lp < 0) & (lpp < 0)
    res["libm"] = {"n_left": int(nl), "effort": float(eff), "t0": t0l, "lost": lost_pairs(idl, lpl),
                   "envelope": _rel(cl[alive], cp[alive]).tolist(),
                   "b2e_vs_libm": _rel(cl[alive], c[alive]).tolist(),
                   "lost_one_ulp": lost_pairs(idl, lpp), "seconds": time.time() - t}
    np.savez_compressed(RING_LIBM, coords=cl, ids=idl, lost_pass=lpl.astype(np.int32))
    out["ring"] = res


def make_edge(out):
    """The dynamic-aperture edge beam, 1,000 turns: loss pairs of the
    reference in both maths modes and of the glibc build with x moved by one
    ulp, and the shared-maths survivors' digest."""
    from elegant_b200 import workloads as w
    from reforacle import track_split
    lat, beam = edge_inputs()
    p0 = w.ring_p_central()
    t = time.time()
    res = {"input": digest_beam(beam.coords, beam.ids), "turns": RING_TURNS}
    pairs = {}
    for math in ("b2e", "libm"):
        rows, nl, eff, t0 = track_split(math, lat, beam.coords, beam.ids, p0, RING_TURNS)
        c, ids, lp = rows_result(rows)
        pairs[math] = np.asarray(lost_pairs(ids, lp), dtype=np.int64)
        res[math] = {"n_left": int(nl), "effort": float(eff), "lost": digest_lost(ids, lp),
                     "survivors": digest_survivors(c, ids, lp)}
    pert = beam.coords.copy()
    pert[:, 0] = np.nextafter(pert[:, 0], np.inf)
    rows, _, _, _ = track_split("libm", lat, pert, beam.ids, p0, RING_TURNS)
    _, ids, lp = rows_result(rows)
    pairs["libm_one_ulp"] = np.asarray(lost_pairs(ids, lp), dtype=np.int64)
    res["libm_one_ulp_lost"] = digest_lost(ids, lp)
    np.savez_compressed(EDGE_LOSSES, **pairs)
    res["seconds"] = time.time() - t
    out["edge"] = res


def make_chicane(out):
    from reforacle import RefOracle
    lat, beam = chicane_inputs()
    t = time.time()
    rows, nl, eff, wakes = RefOracle("b2e", private=True).track(lat, beam.coords, beam.ids, CHICANE_P0, 1,
                                                               capture_wakes=True)
    c, ids, lp = rows_result(rows)
    bins = 600
    wk = wakes.reshape(-1, bins)
    out["chicane"] = {"input": digest_beam(beam.coords, beam.ids), "n_left": int(nl), "bins": bins,
                      "survivors": digest_survivors(c, ids, lp), "lost": lost_pairs(ids, lp),
                      "kicks": int(wk.shape[0]), "wakes": [digest_array(k) for k in wk],
                      "seconds": time.time() - t}


def make_ensemble(out):
    from elegant_b200 import workloads as w
    from reforacle import track_instances
    twd = out["ring"]["twiss"]
    lat, beam, offsets, overrides = ensemble_inputs(twiss_from(twd))
    p0 = w.ring_p_central()
    jobs = []
    for i in range(ENSEMBLE_INSTANCES):
        sl = slice(int(offsets[i]), int(offsets[i + 1]))
        jobs.append((instance_lattice(lat, overrides, i), beam.coords[sl], beam.ids[sl], p0, RING_TURNS, True))
    t = time.time()
    res = track_instances("b2e", jobs)
    inst, surv, mom = [], [], []
    keep = np.arange(9, RING_TURNS, 10)
    for (rows, nl, eff, hist) in res:
        c, ids, lp = rows_result(rows)
        inst.append({"n_left": int(nl), "effort": float(eff), "survivors": digest_survivors(c, ids, lp),
                     "lost": digest_lost(ids, lp), "n_lost": int((lp >= 0).sum())})
        surv.append(hist[:, 0].astype(np.int64))
        mom.append(hist[keep, 1:])
    np.savez_compressed(ENSEMBLE_HISTORY, survivors=np.asarray(surv), passes=keep, moments=np.asarray(mom))
    out["ensemble"] = {"input": digest_beam(beam.coords, beam.ids), "instances": inst,
                       "offsets": [int(x) for x in offsets], "seconds": time.time() - t}


def _train_bunch(args):
    lat, coords, ids = args
    from reforacle import RefOracle
    rows, nl, eff, wakes = RefOracle("b2e", private=True).track(lat, coords, ids, CHICANE_P0, 1,
                                                               capture_wakes=True)
    return rows, nl, wakes


def make_train(out):
    import concurrent.futures
    import multiprocessing as mp
    lat, beam, offsets = train_inputs()
    t = time.time()
    jobs = [(lat, beam.coords[offsets[b]:offsets[b + 1]], beam.ids[offsets[b]:offsets[b + 1]])
            for b in range(len(offsets) - 1)]
    with concurrent.futures.ProcessPoolExecutor(len(jobs), mp_context=mp.get_context("spawn")) as pool:
        res = list(pool.map(_train_bunch, jobs))
    bunches = []
    for rows, nl, wakes in res:
        c, ids, lp = rows_result(rows)
        wk = wakes.reshape(-1, 600)
        bunches.append({"n_left": int(nl), "survivors": digest_survivors(c, ids, lp), "lost": lost_pairs(ids, lp),
                        "wakes": [digest_array(k) for k in wk]})
    out["train"] = {"input": digest_beam(beam.coords, beam.ids), "offsets": [int(x) for x in offsets],
                    "bunches": bunches, "seconds": time.time() - t, **TRAIN}


def main(which):
    out = load_fixture() if os.path.exists(FIXTURE) else {}
    for name, fn in (("ring", make_ring), ("edge", make_edge), ("chicane", make_chicane),
                     ("ensemble", make_ensemble), ("train", make_train)):
        if name in which:
            t = time.time()
            fn(out)
            print(f"{name}: {time.time() - t:.1f} s", flush=True)
            with open(FIXTURE, "w") as f:
                json.dump(out, f, indent=1)
                f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:] or ["ring", "edge", "chicane", "ensemble", "train"])
