"""Host-side mirror of elegant's tracking entry (&run_setup + &track ->
do_tracking, do_tracking.c:144) for the supported element subset, calling
the CUDA engine through its C ABI.

    trk = Tracker(lattice, p_central, n_passes)
    result = trk.track(beam)        # host buffers in, host buffers out

Results keep the input particle order; ``lost_pass`` is -1 for survivors,
else the pass on which the particle was lost (elegant's lossPass column).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .beam import Beam
from .lattice import SLOTS, TYPES, Lattice


@dataclass
class TrackResult:
    coords: np.ndarray       # (n, 6), input order
    ids: np.ndarray          # (n,)
    lost_pass: np.ndarray    # (n,) int32, -1 = survived
    lost_element: np.ndarray  # (n,) int32, -1 = survived
    n_left: int
    effort: float            # particle-passes (do_tracking.c:2758-2764)

    @property
    def survived(self) -> np.ndarray:
        return self.lost_pass < 0


class Tracker:
    """One engine context bound to a lattice and run options."""

    def __init__(self, lattice: Lattice, p_central: float, n_passes: int, device: int = 0, default_order: int = 2,
                 passes_per_launch: int = 0, ring_variant: int = 0, record_history: bool = False,
                 compact_every: int = 0, isr_seed: int = 0, sr_gaussian_limit: float = 3.0,
                 record_tbt: bool = False, fiducial_particles: int = 0):
        self.lib = nat.load_library()
        self.lattice = lattice
        self._ctx = ctypes.c_void_p()
        rc = self.lib.b2e_create(ctypes.byref(self._ctx), device)
        if rc != nat.B2E_OK:
            raise nat.EngineError(rc, "b2e_create failed (is a CUDA device visible?)")
        self.options = nat.RunOptions(p_central=p_central, n_passes=n_passes, default_order=default_order,
                                      coord_limit=10.0, slope_limit=1.0, passes_per_launch=passes_per_launch,
                                      ring_variant=ring_variant, record_history=int(record_history),
                                      compact_every=compact_every, sr_gaussian_limit=sr_gaussian_limit,
                                      isr_seed=isr_seed, record_tbt=int(record_tbt),
                                      fiducial_particles=fiducial_particles)
        self._elems = lattice.to_ctypes()
        self._check(self.lib.b2e_load_lattice(self._ctx, self._elems, len(lattice), ctypes.byref(self.options)))
        self.n_instances = 1

    # -- helpers ---------------------------------------------------------
    def _check(self, rc: int):
        if rc != nat.B2E_OK:
            raise nat.EngineError(rc, self.lib.b2e_last_error(self._ctx).decode())

    def close(self):
        if self._ctx:
            self.lib.b2e_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- ensembles -------------------------------------------------------
    def load_ensemble(self, offsets, overrides):
        """offsets: n_instances+1 particle offsets; overrides: (element_index, PARAM, values)."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n_inst = len(offsets) - 1
        self._ov_values = []
        arr = (nat.Override * max(len(overrides), 1))()
        for k, (ie, name, values) in enumerate(overrides):
            e = self.lattice.elements[ie]
            slot = SLOTS[TYPES[e.type]][name.upper()]
            v = np.ascontiguousarray(values, dtype=np.float64)
            if v.shape != (n_inst,):
                raise ValueError("override values must have one entry per instance")
            self._ov_values.append(v)
            arr[k].element = ie
            arr[k].slot = slot
            arr[k].values = v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self._offsets = offsets
        self._check(self.lib.b2e_load_ensemble(self._ctx, n_inst, offsets.ctypes.data_as(ctypes.c_void_p), arr,
                                               len(overrides)))
        self.n_instances = n_inst

    # -- tracking --------------------------------------------------------
    def track(self, beam: Beam) -> TrackResult:
        """Upload, track all passes, download (b2e_track_host).  The input beam is not modified."""
        cols = [np.array(beam.coords[:, i], dtype=np.float64, copy=True) for i in range(6)]
        ids = beam.ids.copy()
        n = beam.n
        lost_pass = np.empty(n, dtype=np.int32)
        lost_elem = np.empty(n, dtype=np.int32)
        n_left = ctypes.c_int64()
        effort = ctypes.c_double()
        ptrs = nat.pointer_array([c.ctypes.data for c in cols])
        self._check(self.lib.b2e_track_host(self._ctx, ptrs, ids.ctypes.data, n, lost_pass.ctypes.data,
                                            lost_elem.ctypes.data, ctypes.byref(n_left), ctypes.byref(effort)))
        self._n = n
        return TrackResult(np.stack(cols, axis=1), ids, lost_pass, lost_elem, int(n_left.value), effort.value)

    def upload(self, beam: Beam):
        """Copy a beam to the device (starts a new run at pass 0)."""
        cols = [np.array(beam.coords[:, i], dtype=np.float64, copy=True) for i in range(6)]
        self._n = beam.n
        ptrs = nat.pointer_array([c.ctypes.data for c in cols])
        self._check(self.lib.b2e_upload_particles(self._ctx, ptrs, beam.ids.ctypes.data, beam.n))

    def continue_tracking(self) -> float:
        """Track the resident particles for n_passes more passes; returns the effort."""
        effort = ctypes.c_double()
        self._check(self.lib.b2e_track(self._ctx, ctypes.byref(effort)))
        return effort.value

    def download(self) -> TrackResult:
        n = self._n if hasattr(self, "_n") else 0
        cols = [np.empty(n) for _ in range(6)]
        ids = np.empty(n, dtype=np.int64)
        lost_pass = np.empty(n, dtype=np.int32)
        lost_elem = np.empty(n, dtype=np.int32)
        n_left = ctypes.c_int64()
        ptrs = nat.pointer_array([c.ctypes.data for c in cols])
        self._check(self.lib.b2e_download(self._ctx, ptrs, ids.ctypes.data, lost_pass.ctypes.data,
                                          lost_elem.ctypes.data, ctypes.byref(n_left)))
        return TrackResult(np.stack(cols, axis=1), ids, lost_pass, lost_elem, int(n_left.value), float("nan"))

    def ring_tuning(self):
        """(variant in use, per-variant ms of one pass) from the autotuner."""
        chosen = ctypes.c_int32()
        ms = (ctypes.c_float * nat.RING_VARIANTS)()
        self._check(self.lib.b2e_ring_tuning(self._ctx, ctypes.byref(chosen), ms))
        return int(chosen.value), [float(x) for x in ms]

    @property
    def launches(self) -> int:
        """Kernels launched by this context so far."""
        return int(self.lib.b2e_kernel_launches(self._ctx))

    def track_host_pointers(self, col_ptrs, ids_ptr: int, n: int, lost_pass_ptr: int, lost_elem_ptr: int):
        """b2e_track_host on caller-owned (e.g. pinned) host buffers; returns (n_left, effort)."""
        n_left = ctypes.c_int64()
        effort = ctypes.c_double()
        ptrs = nat.pointer_array(list(col_ptrs))
        self._check(self.lib.b2e_track_host(self._ctx, ptrs, ids_ptr, n, lost_pass_ptr, lost_elem_ptr,
                                            ctypes.byref(n_left), ctypes.byref(effort)))
        self._n = n
        return int(n_left.value), effort.value

    @property
    def stream(self) -> int:
        """cudaStream_t of this context (as an integer handle)."""
        return self.lib.b2e_stream(self._ctx) or 0

    def track_device(self, columns, lost_pass, lost_element) -> float:
        """Track device-resident columns in place (six CUDA float64 tensors or raw
        pointers, lost_pass/lost_element int32 initialised to -1).  Returns the effort."""
        def ptr(t):
            return t if isinstance(t, int) else t.data_ptr()
        n = columns[0].numel() if hasattr(columns[0], "numel") else None
        if n is None:
            raise ValueError("pass tensors so the particle count is known")
        effort = ctypes.c_double()
        ptrs = nat.pointer_array([ptr(c) for c in columns])
        self._check(self.lib.b2e_track_device(self._ctx, ptrs, None, n, ptr(lost_pass), ptr(lost_element),
                                              ctypes.byref(effort)))
        return effort.value

    def history(self) -> dict:
        """Per-instance, per-pass survivors, centroids and rms emittances of the
        run so far: arrays of shape (n_instances, n_passes)."""
        n_pass = int(self.lib.b2e_history_passes(self._ctx))
        shape = (self.n_instances, max(n_pass, 0))
        out = {"survivors": np.zeros(shape, dtype=np.int64)}
        for k in ("cx", "cy", "ex", "ey"):
            out[k] = np.zeros(shape, dtype=np.float64)
        self._check(self.lib.b2e_ensemble_history(self._ctx, *(out[k].ctypes.data for k in
                                                                ("survivors", "cx", "cy", "ex", "ey"))))
        return out

    def tbt(self) -> np.ndarray:
        """Turn-by-turn x, x', y, y' of the last call with record_tbt:
        array [records][4][n]; record 0 is the call's start."""
        n = ctypes.c_int64()
        self._check(self.lib.b2e_tbt(self._ctx, None, 0, ctypes.byref(n)))
        out = np.empty(n.value, dtype=np.float64)
        self._check(self.lib.b2e_tbt(self._ctx, out.ctypes.data, n.value, ctypes.byref(n)))
        return out.reshape(-1, 4, self._n)

    def set_watch(self, max_bytes: int):
        """Record WATCH elements (coordinate mode) in the following calls,
        within max_bytes of device memory (b2e_set_watch); 0 turns it off."""
        self._check(self.lib.b2e_set_watch(self._ctx, int(max_bytes)))

    def watch(self) -> list:
        """The WATCH records of the last call, in WATCH (lattice) order then
        pass order: dicts with element (index), pass, ids and coords (n, 6)
        of the particles alive at the element, by ascending ID."""
        nr = ctypes.c_int32()
        rows = ctypes.c_int64()
        self._check(self.lib.b2e_watch_records(self._ctx, ctypes.byref(nr), ctypes.byref(rows), None, None, 0))
        elems = np.empty(nr.value, dtype=np.int32)
        passes = np.empty(nr.value, dtype=np.int32)
        self._check(self.lib.b2e_watch_records(self._ctx, ctypes.byref(nr), ctypes.byref(rows), elems.ctypes.data,
                                               passes.ctypes.data, nr.value))
        out = []
        buf = np.empty((7, rows.value), dtype=np.float64)
        for r in range(nr.value):
            self._check(self.lib.b2e_watch_data(self._ctx, r, buf.ctypes.data))
            live = ~np.isnan(buf[6])
            ids = buf[6, live].astype(np.int64)
            order = np.argsort(ids, kind="stable")
            out.append({"element": int(elems[r]), "pass": int(passes[r]), "ids": ids[order],
                        "coords": buf[:6, live].T[order].copy()})
        return out

    def tbt_tunes(self, first_record: int, n_records: int) -> dict:
        """Tunes (NAFF + half-plane from the x/x' phases) of every row over
        records [first_record, first_record + n_records); -1 where the
        particle was lost before the window's end."""
        out = {k: np.empty(self._n) for k in ("nux", "nuy", "ax", "ay")}
        self._check(self.lib.b2e_tbt_tunes(self._ctx, first_record, n_records, *(out[k].ctypes.data for k in
                                                                                 ("nux", "nuy", "ax", "ay"))))
        return out

    def set_csr_reducer(self, fn):
        """Spread bunches over several ranks: fn(op, device_ptr, count, stream)
        all-reduces an engine buffer in place (see elegant_b200.parallel);
        None for single-GPU bunches."""
        if fn is None:
            self._reducer = None
            self._check(self.lib.b2e_set_csr_reducer(self._ctx, None, None))
            return

        def cb(user, op, ptr, count, stream):
            try:
                return int(fn(int(op), int(ptr or 0), int(count), int(stream or 0)) or 0)
            except Exception:  # an exception must not cross into C
                return -1

        self._reducer = nat.REDUCE_FN(cb)  # kept alive while registered
        self._check(self.lib.b2e_set_csr_reducer(self._ctx, self._reducer, None))

    def set_csr_surrogate(self, surrogate, tolerance: float = 0.01, gate_stride: int = 16):
        """Use a trained wake surrogate (elegant_b200.wake_surrogate.WakeSurrogate)
        for the CSRCSBEND wake integral, gated by the plain integral on every
        gate_stride-th bin with fallback above `tolerance`; None switches back."""
        if surrogate is None:
            self._check(self.lib.b2e_set_csr_surrogate(self._ctx, None, None, 0.0, 1))
            self._surrogate = None
            return
        f = surrogate.features
        sc = (ctypes.c_double * 3)(f.dens_scale, f.deriv_scale, f.target_scale)
        self._check(self.lib.b2e_set_csr_surrogate(self._ctx, surrogate.net._h, sc, tolerance, gate_stride))
        self._surrogate = surrogate  # keeps the network alive while bound

    def csr_surrogate_stats(self) -> dict:
        ev, fb, wr = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.b2e_csr_surrogate_stats(self._ctx, ctypes.byref(ev), ctypes.byref(fb), None, 0,
                                                     ctypes.byref(wr)))
        errs = np.zeros(max(wr.value, 1))
        self._check(self.lib.b2e_csr_surrogate_stats(self._ctx, ctypes.byref(ev), ctypes.byref(fb),
                                                     errs.ctypes.data, wr.value, ctypes.byref(wr)))
        return {"evaluations": ev.value, "fallbacks": fb.value, "gate_errors": errs[: wr.value]}

    def set_csr_timing(self, on: bool = True):
        """Time the wake stage of every CSRCSBEND kick of later runs with CUDA
        events (see csr_wake_timing)."""
        self._check(self.lib.b2e_set_csr_timing(self._ctx, int(on)))

    def csr_wake_timing(self) -> dict:
        """Summed device time of the last run's timed wake stages: ms, kicks,
        learned_kicks (kicks that took the learned wake), ms_per_kick."""
        ms, k, lk = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.b2e_csr_timing(self._ctx, ctypes.byref(ms), ctypes.byref(k), ctypes.byref(lk)))
        return {"ms": ms.value, "kicks": k.value, "learned_kicks": lk.value,
                "ms_per_kick": ms.value / k.value if k.value else float("nan")}

    def set_csr_pages(self, record: bool = True):
        """Keep, for every plain-integral CSRCSBEND kick of later runs, what the
        element's OUTPUT_FILE page holds (see csr_pages)."""
        self._check(self.lib.b2e_set_csr_pages(self._ctx, int(record)))

    def csr_pages(self) -> list[dict]:
        """The page records of the last run, in kick order (bunches within a
        kick): element index, kick, bunch, bins, the binned range (ct_lower,
        ct_upper), dct, slippage, angle (phiBend), ds_kick, p_central,
        macro_charge, and the arrays hist (line density per unit c*t), deriv
        (its derivative), t1 and t2 (the wake terms), dgamma (the kick's
        wake, from the wake log).  Kicks of a bunch without CSR are left out.
        Plain-integral kicks only: with the learned wake bound, no pages."""
        written = ctypes.c_int64()
        self._check(self.lib.b2e_csr_pages(self._ctx, None, 0, ctypes.byref(written)))
        buf = np.empty(max(written.value, 1), dtype=np.float64)
        self._check(self.lib.b2e_csr_pages(self._ctx, buf.ctypes.data, written.value, ctypes.byref(written)))
        nw = ctypes.c_int64()
        self._check(self.lib.b2e_csr_wakes(self._ctx, None, 0, ctypes.byref(nw)))
        wakes = self.csr_wakes(max(nw.value, 1))
        pages, pos, wpos, h = [], 0, 0, nat.CSR_PAGE_HEADER
        while pos < written.value:
            head = buf[pos:pos + h]
            bins = int(head[3])
            if head[0] >= 0:  # else a bunch without CSR on this kick
                a = buf[pos + h:pos + h + 4 * bins].reshape(4, bins)
                pages.append({"element": int(head[0]), "kick": int(head[1]), "bunch": int(head[2]), "bins": bins,
                              "ct_lower": head[4], "ct_upper": head[5], "dct": head[6], "slippage": head[7],
                              "angle": head[8], "ds_kick": head[9], "p_central": head[10],
                              "macro_charge": head[11], "hist": a[0].copy(), "deriv": a[1].copy(),
                              "t1": a[2].copy(), "t2": a[3].copy(), "dgamma": wakes[wpos:wpos + bins].copy()})
            pos += h + 4 * bins
            wpos += bins  # the wake log holds every bunch of every kick in the same order
        return pages

    def csr_wakes(self, capacity: int) -> np.ndarray:
        buf = np.empty(capacity, dtype=np.float64)
        written = ctypes.c_int64()
        self._check(self.lib.b2e_csr_wakes(self._ctx, buf.ctypes.data, capacity, ctypes.byref(written)))
        return buf[: written.value]


def track(lattice: Lattice, beam: Beam, p_central: float, n_passes: int, **kw) -> TrackResult:
    with Tracker(lattice, p_central, n_passes, **kw) as t:
        return t.track(beam)
