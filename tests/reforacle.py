"""Test-side wrappers around the CPU oracles in oracle/.

- ``RefOracle``: elegant's own hot-path C sources compiled through a shim
  (oracle/_ref/libb2e_ref*.so, built by oracle/Makefile.ref), driven by
  oracle/ref_driver.c.  ``math="libm"`` uses glibc's elementary functions like
  the reference build; ``math="b2e"`` routes sin/cos/tan/asin to the shared
  implementations of elegant_b200/csrc/b2e_math.h that the CUDA engine uses.
- ``PortOracle``: the restatement in oracle/b2e_oracle.c (same math switch).

Only tests, the graft smoke check and the benchmark's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def lattice_spec(lattice) -> str:
    """Element list in the driver's 'NAME:TYPE KEY=VALUE ...;' syntax."""
    from elegant_b200.lattice import FIDUCIAL_MODES
    fid = {c: n for n, c in FIDUCIAL_MODES}
    items = []
    for e in lattice.elements:
        kv = " ".join(f"{k}={fid[int(v)]}" if (k == "FIDUCIAL" and e.type == "RFCA") else f"{k}={v!r}"
                      for k, v in e.params.items())
        items.append(f"{e.name}:{e.type} {kv}".strip())
    return ";".join(items)


class RefOracle:
    def __init__(self, math: str = "libm", private: bool = False):
        """private=True loads a fresh copy of the library, so that file-static
        state of the reference (SolveForPhiStupakov's start value, which
        carries over from one call to the next for the life of an elegant
        process) starts as in a new process."""
        name = "libb2e_ref.so" if math == "libm" else "libb2e_ref_b2emath.so"
        path = os.path.join(REF_DIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        if private:
            import shutil
            import tempfile
            fd, tmp = tempfile.mkstemp(prefix="b2e_ref_", suffix=".so")
            os.close(fd)
            shutil.copyfile(path, tmp)
            try:
                self.lib = ctypes.CDLL(tmp)
            finally:
                os.unlink(tmp)  # the mapping stays valid
        else:
            self.lib = ctypes.CDLL(path)
        self.lib.b2e_ref_track.restype = ctypes.c_long
        self.lib.b2e_ref_last_fiducial_t0.restype = ctypes.c_double
        self.math = math
        self.last_history = None

    def last_fiducial_t0(self) -> float:
        """Fiducial time the last run's zero-length RFCA computed on its first
        pass (findFiducialTime on the particles it received); -1 if none."""
        return float(self.lib.b2e_ref_last_fiducial_t0())

    def watch_rows(self):
        """The rows the last run's WATCH elements were handed (set_watch):
        array [k][9] = element index, pass, particleID, x, xp, y, yp, s, delta."""
        self.lib.b2e_ref_watch_rows.restype = ctypes.c_long
        k = self.lib.b2e_ref_watch_rows()
        return self._watch[:k].copy()

    def set_watch(self, capacity_rows: int):
        """Capture the coordinate-mode WATCH rows of the following runs (up to
        capacity_rows rows); 0 turns it off."""
        self._watch = np.zeros((max(capacity_rows, 1), 9))
        self.lib.b2e_ref_set_watch(self._watch.ctypes.data_as(ctypes.c_void_p) if capacity_rows else None,
                                   ctypes.c_long(capacity_rows))

    def track(self, lattice, coords, ids, p_central, n_passes, wake_capacity=0, capture_wakes=False,
              history=False):
        """Returns (rows, n_left, effort, wakes); rows are the reference's final
        particle array (x, xp, y, yp, s, delta, id, lossPass), survivors first.
        With capture_wakes, every CSRCSBEND writes its per-kick DeltaGamma through
        the reference's own OUTPUT_FILE path (captured in memory), returned as wakes.
        With history, ``last_history`` holds [pass][survivors, <x>, <y>, ex, ey]
        of the survivors after every pass."""
        hist = np.zeros((max(n_passes, 1), 5)) if history else None
        self.lib.b2e_ref_set_history(hist.ctypes.data_as(ctypes.c_void_p) if history else None,
                                     ctypes.c_long(n_passes if history else 0))
        try:
            return self._track(lattice, coords, ids, p_central, n_passes, wake_capacity, capture_wakes)
        finally:
            self.lib.b2e_ref_set_history(None, ctypes.c_long(0))
            self.last_history = hist[:n_passes] if history else None

    def _track(self, lattice, coords, ids, p_central, n_passes, wake_capacity, capture_wakes):
        n = coords.shape[0]
        rows = np.zeros((n, 7))
        rows[:, :6] = coords
        rows[:, 6] = ids
        out = np.zeros((max(n, 1), 8))
        nl = ctypes.c_long()
        eff = ctypes.c_double()
        err = ctypes.create_string_buffer(512)
        ww = ctypes.c_long()
        wakes = np.zeros(max(wake_capacity, 1))
        spec = lattice_spec(lattice)
        if capture_wakes:
            spec = spec.replace(":CSRCSBEND", ":CSRCSBEND OUTPUT_FILE=capture")
        rc = self.lib.b2e_ref_track(spec.encode(), ctypes.c_double(p_central),
                                    rows.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(n), ctypes.c_long(n_passes),
                                    out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nl), ctypes.byref(eff),
                                    wakes.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(wake_capacity),
                                    ctypes.byref(ww), err, ctypes.c_long(512))
        if rc != 0:
            raise RuntimeError(f"reference oracle failed: {err.value.decode()}")
        if capture_wakes:
            self.lib.b2e_ref_capture_get.restype = ctypes.c_long
            k = self.lib.b2e_ref_capture_get(0, None, ctypes.c_long(0))
            buf = np.zeros(max(k, 1))
            self.lib.b2e_ref_capture_get(0, buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(k))
            return out[:n], nl.value, eff.value, buf[:k]
        return out[:n], nl.value, eff.value, wakes[: ww.value]


CAPTURE_COLUMNS = ["DeltaGamma", "LinearDensity", "LinearDensityDeriv", "DeltaGammaT1", "DeltaGammaT2", "s",
                   "GammaDeriv"]
CAPTURE_PARAMS = ["Pass", "Kick", "dsKick", "pCentral", "Angle", "SlippageLength", "TotalBunchLength", "BinSize",
                  "DerbenevRatio"]


def captured_pages(ref: "RefOracle") -> dict:
    """What the last capture_wakes run's CSRCSBEND OUTPUT_FILE writer was given:
    every column (all pages concatenated) and the parameters, one row per page."""
    lib = ref.lib
    lib.b2e_ref_capture_get.restype = ctypes.c_long
    lib.b2e_ref_capture_params.restype = ctypes.c_long
    out = {}
    for i, name in enumerate(CAPTURE_COLUMNS):
        k = lib.b2e_ref_capture_get(i, None, ctypes.c_long(0))
        buf = np.zeros(max(k, 1))
        lib.b2e_ref_capture_get(i, buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(k))
        out[name] = buf[:k]
    k = lib.b2e_ref_capture_params(None, ctypes.c_long(0))
    buf = np.zeros(max(k, 1))
    lib.b2e_ref_capture_params(buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(k))
    out["parameters"] = buf[:k].reshape(-1, len(CAPTURE_PARAMS))
    return out


def with_fiducial(lattice, t0: float):
    """The lattice with T_REFERENCE = t0 on its RFCA elements."""
    from elegant_b200.lattice import Element, Lattice
    return Lattice([Element(e.name, e.type, dict(e.params, T_REFERENCE=t0)) if e.type == "RFCA" else e
                    for e in lattice.elements])


def _pool(processes):
    """Spawned worker processes (never forked: the parent may hold a CUDA
    context); a worker that dies raises BrokenProcessPool instead of hanging."""
    import concurrent.futures
    import multiprocessing as mp
    return concurrent.futures.ProcessPoolExecutor(processes, mp_context=mp.get_context("spawn"))


def _split_worker(args):
    math, lattice, coords, ids, p_central, n_passes, history = args
    ref = RefOracle(math)
    rows, nl, eff, _ = ref.track(lattice, coords, ids, p_central, n_passes, history=history)
    return rows, nl, eff, ref.last_history


def track_split(math, lattice, coords, ids, p_central, n_passes, processes=None):
    """The reference's tracking of one beam, spread over particle slices in
    spawned processes.  Particles of a ring are independent except through the
    RFCA's TMEAN fiducial (the Kahan mean over the whole beam on the first
    pass, simple_rfca.c:179-230), so the whole beam is tracked for one pass
    first, its fiducial time is read back and every slice is given it as
    T_REFERENCE.  Returns (rows by slice, concatenated; n_left; effort; t0)."""
    n = coords.shape[0]
    ref = RefOracle(math)
    ref.track(lattice, coords, ids, p_central, 1)
    t0 = ref.last_fiducial_t0()
    lat = with_fiducial(lattice, t0) if t0 != -1 else lattice
    processes = processes or os.cpu_count() or 1
    bounds = np.linspace(0, n, processes + 1).astype(int)
    jobs = [(math, lat, coords[a:b], ids[a:b], p_central, n_passes, False) for a, b in zip(bounds[:-1], bounds[1:])
            if b > a]
    with _pool(len(jobs)) as pool:
        res = list(pool.map(_split_worker, jobs))
    rows = np.concatenate([r[0] for r in res])
    return rows, sum(r[1] for r in res), sum(r[2] for r in res), t0


def track_instances(math, jobs, processes=None):
    """Independent reference runs in spawned processes: jobs are
    (lattice, coords, ids, p_central, n_passes, history) tuples; returns
    [(rows, n_left, effort, history)] in job order."""
    processes = min(processes or os.cpu_count() or 1, len(jobs))
    with _pool(processes) as pool:
        return list(pool.map(_split_worker, [(math, *j) for j in jobs]))


def by_id(rows):
    """Sort reference rows by particle ID; returns (coords[n,6], ids, loss_pass)."""
    order = np.argsort(rows[:, 6], kind="stable")
    r = rows[order]
    return r[:, :6], r[:, 6].astype(np.int64), r[:, 7].astype(np.int64)


class PortOracle:
    """The C restatement in oracle/b2e_oracle.c (oracle/_build)."""

    def __init__(self, math: str = "b2e"):
        name = "libb2e_oracle.so" if math == "b2e" else "libb2e_oracle_libm.so"
        path = os.path.join(ROOT, "oracle", "_build", name)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.b2e_oracle_track.restype = ctypes.c_long
        for f in ("sin", "cos", "tan", "asin"):
            fn = getattr(self.lib, f"b2e_oracle_{f}")
            fn.restype = ctypes.c_double
            fn.argtypes = [ctypes.c_double]
        self.math = math
        self.set_isr(0, 3.0)

    def set_isr(self, seed: int, limit: float = 3.0):
        """Seed and truncation of the ISR deviates (the engine's generator)."""
        self.lib.b2e_oracle_set_isr.argtypes = [ctypes.c_uint64, ctypes.c_double]
        self.lib.b2e_oracle_set_isr(ctypes.c_uint64(seed), ctypes.c_double(limit))

    def wake_t1(self, counts, slippage_bins, sg_half=0, sg_order=1, sgd_half=0, sgd_order=0, trapz=True,
                steady=False):
        """T1 wake integral of one histogram in bin units: (t1, density, derivative)."""
        c = np.ascontiguousarray(counts, dtype=np.float64)
        nb = c.size
        t1, h, d = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        dp = ctypes.POINTER(ctypes.c_double)
        f = self.lib.b2e_oracle_wake_t1
        f.restype = None
        f.argtypes = [dp, ctypes.c_long, ctypes.c_double] + [ctypes.c_int] * 6 + [dp, dp, dp]
        f(c.ctypes.data_as(dp), nb, float(slippage_bins), sg_half, sg_order, sgd_half, sgd_order, int(trapz),
          int(steady), t1.ctypes.data_as(dp), h.ctypes.data_as(dp), d.ctypes.data_as(dp))
        return t1, h, d

    def track(self, lattice, coords, ids, p_central, n_passes, default_order=2, capture_wakes=False):
        """Returns (rows, n_left, effort) like RefOracle.track, plus the per-kick
        CSR wakes as a fourth item when capture_wakes is set."""
        n = coords.shape[0]
        rows = np.zeros((max(n, 1), 8))
        rows[:n, :6] = coords
        rows[:n, 6] = ids
        rows[:n, 7] = -1
        elems = lattice.to_ctypes()
        eff = ctypes.c_double()
        self.lib.b2e_oracle_track_csr.restype = ctypes.c_long
        cap = 4_000_000 if capture_wakes else 0
        wakes = np.zeros(max(cap, 1))
        nw = ctypes.c_long()
        nl = self.lib.b2e_oracle_track_csr(elems, ctypes.c_int(len(lattice)), ctypes.c_double(p_central),
                                           ctypes.c_int(n_passes), ctypes.c_int(default_order),
                                           rows.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(n), ctypes.byref(eff),
                                           wakes.ctypes.data_as(ctypes.c_void_p) if capture_wakes else None,
                                           ctypes.c_long(cap), ctypes.byref(nw))
        if nl < 0:
            raise RuntimeError("port oracle failed: No available particle for RF cavity fiducialization")
        if capture_wakes:
            return rows[:n], nl, eff.value, wakes[: nw.value]
        return rows[:n], nl, eff.value
