"""SDDS output of tracking results, in the layouts elegant writes, for its
post-processing tools (sddsplot, sddsanalyzebeam, ...).

- `write_phase_space`: the &run_setup `final` / `output` file
  (dump_phase_space, sdds_support.c:1531-1604): columns x, xp, y, yp,
  t = s / (c beta), p = P0 (1 + delta), particleID; parameters Step,
  pCentral, Charge, Particles, IDSlotsPerBunch (sdds_support.c:150-170).
- `write_losses`: the `losses` file (sdds_support.c:199-212): x, xp, y, yp, s,
  p, particleID, Pass.
- `write_momentum_aperture`, `write_frequency_map`, `write_aperture`: the
  outputs of &momentum_aperture (output_mode 0), &frequency_map and the
  line modes of &find_aperture, in their column layouts.  s is the end position of the element where the
  particle was lost (elegant additionally extrapolates aperture losses into
  the preceding drift); the coordinates are those at the loss.

Files are protocol-1 SDDS, binary (little-endian) or ASCII.  particleID is
written as `long` (32-bit), which every SDDS reader accepts; elegant itself
uses ulong64.  `read_sdds` reads what this module writes (for tests and
round trips), not arbitrary SDDS.
"""
from __future__ import annotations

import math
import os
import struct

import numpy as np

C_MKS = 2.99792458e8
# SDDS type -> (struct code, numpy dtype); strings are (int32 length, bytes)
_FMT = {"double": ("d", np.float64), "long": ("i", np.int32), "short": ("h", np.int16), "string": (None, None)}


def _quote(v: str) -> str:
    return '"' + v.replace('"', '\\"') + '"'


def write_sdds(path, parameters, columns, mode="binary", description=None, append=False):
    """parameters: [(name, type, value, attrs)], columns: [(name, type,
    values, attrs)], types 'double' | 'long' | 'short' | 'string'; attrs:
    dict of units, symbol, description.  Binary data are written row by row
    (SDDS's row-major layout), so string columns work too.  One page;
    append=True adds it to an existing file of the same layout (elegant's
    one page per step)."""
    write_sdds_pages(path, [(p[0], p[1], p[3]) for p in parameters], [(c[0], c[1], c[3]) for c in columns],
                     [([p[2] for p in parameters], [c[2] for c in columns])], mode, description, append)


def write_sdds_pages(path, parameters, columns, pages, mode="binary", description=None, append=False):
    """Several pages of one layout: parameters [(name, type, attrs)], columns
    [(name, type, attrs)], pages [(parameter values, column arrays)] in the
    definition orders.  append=True and an existing file: the pages are
    added after its last page (the caller keeps the layout the same)."""
    if mode not in ("binary", "ascii"):
        raise ValueError("mode must be 'binary' or 'ascii'")
    for c in columns:
        if c[1] not in _FMT:
            raise ValueError(f"unsupported SDDS type {c[1]}")
    for _, cols in pages:
        n = len(cols[0]) if cols else 0
        if any(len(v) != n for v in cols):
            raise ValueError("columns of different lengths")
    lines = ["SDDS1"]
    if mode == "binary":
        lines.append("!# little-endian")
    if description:
        lines.append(f"&description text={_quote(description)}, &end")

    def attrs_text(a):
        return "".join(f" {k}={_quote(str(v))}," for k, v in (a or {}).items())

    for name, typ, a in parameters:
        lines.append(f"&parameter name={name},{attrs_text(a)} type={typ}, &end")
    for name, typ, a in columns:
        lines.append(f"&column name={name},{attrs_text(a)} type={typ}, &end")
    lines.append(f"&data mode={mode}, &end")
    adding = append and os.path.exists(path)
    with open(path, "ab" if adding else "wb") as fh:
        if not adding:
            fh.write(("\n".join(lines) + "\n").encode())
        for values, cols in pages:
            n = len(cols[0]) if cols else 0
            if mode == "binary":
                fh.write(struct.pack("<i", n))
                for (_, typ, _), v in zip(parameters, values):
                    fh.write(_pack(typ, v))
                if n and all(c[1] != "string" for c in columns):
                    rec = np.dtype([(c[0], "<" + np.dtype(_FMT[c[1]][1]).str[1:]) for c in columns])
                    rows = np.empty(n, dtype=rec)
                    for c, v in zip(columns, cols):
                        rows[c[0]] = v
                    fh.write(rows.tobytes())
                else:
                    for i in range(n):
                        fh.write(b"".join(_pack(c[1], v[i]) for c, v in zip(columns, cols)))
            else:
                out = []
                for (_, typ, _), v in zip(parameters, values):
                    out.append(_text(typ, v))
                out.append(f"\t{n}")
                for i in range(n):
                    out.append(" ".join(_text(c[1], v[i]) for c, v in zip(columns, cols)))
                fh.write(("\n".join(out) + "\n").encode())


def _pack(typ, v):
    if typ == "string":
        b = str(v).encode()
        return struct.pack("<i", len(b)) + b
    return struct.pack("<" + _FMT[typ][0], float(v) if typ == "double" else int(v))


def _text(typ, v):
    if typ == "string":
        return _quote(str(v))
    return repr(float(v)) if typ == "double" else str(int(v))


def _split_ascii(line):
    """Tokens of an ASCII data line, double-quoted strings kept whole."""
    out, i = [], 0
    while i < len(line):
        if line[i].isspace():
            i += 1
        elif line[i] == '"':
            j, buf = i + 1, []
            while j < len(line) and line[j] != '"':
                if line[j] == "\\" and j + 1 < len(line):
                    j += 1
                buf.append(line[j])
                j += 1
            out.append("".join(buf))
            i = j + 1
        else:
            j = i
            while j < len(line) and not line[j].isspace():
                j += 1
            out.append(line[i:j])
            i = j
    return out


def read_sdds(path):
    """(parameters dict, columns dict) of a single-page file written by
    write_sdds (numeric columns as arrays, string columns as lists)."""
    with open(path, "rb") as fh:
        data = fh.read()
    pos, params, cols, mode = 0, [], [], None
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].decode()
        pos = end + 1
        if line.startswith("&parameter") or line.startswith("&column"):
            fields = dict(kv.strip().split("=", 1) for kv in line.split(" ", 1)[1].rsplit("&end", 1)[0].split(",")
                          if "=" in kv)
            (params if line.startswith("&parameter") else cols).append((fields["name"], fields["type"]))
        elif line.startswith("&data"):
            mode = "binary" if "binary" in line else "ascii"
            break

    def conv(typ, v):
        return v if typ == "string" else (float(v) if typ == "double" else int(v))

    if mode == "binary":
        n = struct.unpack_from("<i", data, pos)[0]
        pos += 4

        def take(typ):
            nonlocal pos
            if typ == "string":
                k = struct.unpack_from("<i", data, pos)[0]
                v = data[pos + 4:pos + 4 + k].decode()
                pos += 4 + k
                return v
            f = _FMT[typ][0]
            v = struct.unpack_from("<" + f, data, pos)[0]
            pos += struct.calcsize(f)
            return v
        pv = {name: take(typ) for name, typ in params}
        rows = [[take(typ) for _, typ in cols] for _ in range(n)]
    else:
        toks = data[pos:].decode().split("\n")
        pv = {}
        for (name, typ), t in zip(params, toks):
            pv[name] = conv(typ, t.strip().strip('"'))
        n = int(toks[len(params)])
        rows = [[conv(typ, v) for (_, typ), v in zip(cols, _split_ascii(t))]
                for t in toks[len(params) + 1:len(params) + 1 + n]]
    out = {}
    for j, (name, typ) in enumerate(cols):
        vals = [r[j] for r in rows]
        out[name] = vals if typ == "string" else np.array(vals, dtype=_FMT[typ][1])
    return pv, out


def write_phase_space(path, result, p_central, step=1, charge=0.0, mode="binary", append=False):
    """elegant's `final`/`output` file for the survivors of a TrackResult."""
    alive = result.lost_pass < 0
    c = result.coords[alive]
    p = p_central * (1 + c[:, 5])
    t = c[:, 4] / (C_MKS * p / np.sqrt(p * p + 1))
    params = [("Step", "long", step, {"description": "Simulation step"}),
              ("pCentral", "double", p_central, {"symbol": "p$bcen$n", "units": "m$be$nc",
                                                  "description": "Reference beta*gamma"}),
              ("Charge", "double", charge, {"units": "C", "description": "Bunch charge before sampling"}),
              ("Particles", "long", int(alive.sum()), {"description": "Number of particles before sampling"}),
              ("IDSlotsPerBunch", "long", 0, {"description": "Number of particle ID slots reserved to a bunch"})]
    cols = [("x", "double", c[:, 0], {"units": "m"}), ("xp", "double", c[:, 1], {"symbol": "x'"}),
            ("y", "double", c[:, 2], {"units": "m"}), ("yp", "double", c[:, 3], {"symbol": "y'"}),
            ("t", "double", t, {"units": "s"}), ("p", "double", p, {"units": "m$be$nc"}),
            ("particleID", "long", result.ids[alive].astype(np.int64), {})]
    write_sdds(path, params, cols, mode, description="elegant_b200 phase-space output", append=append)


def watch_pass_central_times(passes, z, length, p_central, reference_frequency=-1.0):
    """PassCentralTime of a WATCH on each of `passes` (ascending) of one step,
    as dump_watch_particles carries it (sdds_support.c:714-736): z beta^-1/c on
    pass 0, then one revolution time per pass added with Kahan's compensated
    sum, each rounded to the RF bucket when reference_frequency > 0."""
    root = math.sqrt(p_central * p_central + 1)
    t0 = z * root / (C_MKS * (p_central + 1e-32))
    err = 0.0
    last, out = 0, []
    for q in passes:
        for _ in range(q - last):
            dt = length * root / (C_MKS * (p_central + 1e-32))
            if reference_frequency > 0:
                dt = float(int(dt * reference_frequency + 0.5)) / reference_frequency
            y = dt + err
            total = t0 + y
            err = y - (total - t0)
            t0 = total
        last = q
        out.append(t0)
    return out


ME_MEV = 0.51099895000  # electron rest energy (particleMassMV), CODATA 2018
# the second moments accumulate_beam_sums forms with BEAM_SUMS_SPARSE
# (compute_centroids.c:300-307): the diagonal blocks and the correlations
# with delta (and s with t)
_SPARSE = [(0, 0), (0, 1), (0, 5), (1, 1), (1, 5), (2, 2), (2, 3), (2, 5), (3, 3), (3, 5), (4, 4), (4, 5), (4, 6),
           (5, 5), (6, 6)]


def watch_statistics(coords, ids, p_central, start_pid=-1, end_pid=-1):
    """The beam statistics of one WATCH record in parameter/centroid mode
    (dump_watch_parameters, sdds_support.c:881-1160): centroids of x..delta
    and of t = s sqrt(P^2+1)/(c P) (computeTimeCoordinates, trwake.c:532),
    the sparse second-moment matrix about them (accumulate_beam_sums,
    compute_centroids.c:286-490), the emittances (computeEmitTwissFromSigma-
    Matrix, sdds_support.c:2303-2340; rms_longitudinal_emittance,
    final_props.c:944-990), and Ct, pAverage, KAverage.  Particles in the
    START_PID/END_PID window only.  Sums here are numpy's (pairwise), where
    elegant sums in its array order with Kahan's compensation: the results
    agree to rounding, not bit for bit."""
    c = np.asarray(coords, dtype=np.float64)
    ids = np.asarray(ids)
    win = np.ones(len(ids), dtype=bool) if (start_pid < 0 and end_pid < 0) else (ids >= start_pid) & (ids <= end_pid)
    x = c[win]
    n = len(x)
    out = {"n": n}
    if n == 0:
        out.update(centroid=np.zeros(7), sigma=np.zeros((7, 7)), Ct=0.0, pAverage=float("nan"),
                   KAverage=float("nan"), ex=0.0, ey=0.0, ecx=0.0, ecy=0.0, el=0.0)
        return out
    P = p_central * (x[:, 5] + 1)
    t = x[:, 4] * np.sqrt(P * P + 1) / (C_MKS * P)
    cols = [x[:, k] for k in range(6)] + [t]
    cen = np.array([v.sum() / n for v in cols])
    dev = [cols[k] - cen[k] for k in range(7)]
    sig = np.zeros((7, 7))
    for i, j in _SPARSE:
        sig[i, j] = sig[j, i] = (dev[i] * dev[j]).sum() / n
    out["centroid"], out["sigma"] = cen, sig

    def emit(plane):
        e = sig[plane, plane] * sig[plane + 1, plane + 1] - sig[plane, plane + 1] ** 2
        e = math.sqrt(e) if e > 0 else 0.0
        if sig[5, 5]:
            ec = e * e - (sig[plane, 5] ** 2 * sig[plane + 1, plane + 1]
                          - 2 * sig[plane, plane + 1] * sig[plane, 5] * sig[plane + 1, 5]
                          + sig[plane + 1, 5] ** 2 * sig[plane, plane]) / sig[5, 5]
            ec = math.sqrt(ec) if ec > 0 else 0.0
        else:
            ec = e
        return e, ec

    out["ex"], out["ecx"] = emit(0)
    out["ey"], out["ecy"] = emit(2)
    # rms_longitudinal_emittance: its own window test (startPID >= endPID is
    # "every particle") and t = s / (beta c)
    lwin = np.ones(len(ids), dtype=bool) if start_pid >= end_pid else (ids >= start_pid) & (ids <= end_pid)
    xl = c[lwin]
    Pl = p_central * (1 + xl[:, 5])
    tl = xl[:, 4] / (Pl / np.sqrt(Pl * Pl + 1) * C_MKS)
    dt, dd = tl - tl.mean(), xl[:, 5] - xl[:, 5].mean()
    e2 = (dt * dt).sum() * (dd * dd).sum() - (dt * dd).sum() ** 2
    out["el"] = (math.sqrt(e2) if e2 > 0 else 0.0) / len(xl) if len(xl) else 0.0
    # Ct, pAverage, KAverage (sdds_support.c:1075-1130): t = s / (p/sqrt(p^2+1) c)
    tt = x[:, 4] / (P / np.sqrt(P * P + 1) * C_MKS)
    out["Ct"] = tt.sum() / n
    out["pAverage"] = P.sum() / n
    out["KAverage"] = (np.sqrt(P * P + 1).sum() / n - 1) * ME_MEV
    return out


_WATCH_PARAM_COLS = [("Step", "long", {}), ("Pass", "long", {}), ("ElapsedTime", "double", {"units": "s"}),
                     ("ElapsedCoreTime", "double", {"units": "s"}), ("MemoryUsage", "long", {"units": "kB"}),
                     ("Cx", "double", {"symbol": "<x>", "units": "m"}), ("Cxp", "double", {"symbol": "<x'>"}),
                     ("Cy", "double", {"symbol": "<y>", "units": "m"}), ("Cyp", "double", {"symbol": "<y'>"}),
                     ("Cs", "double", {"symbol": "<s>", "units": "m"}), ("Cdelta", "double", {"symbol": "<$gd$r>"}),
                     ("Ct", "double", {"symbol": "<t>", "units": "s"}),
                     ("dCt", "double", {"symbol": "$gD$r<t>", "units": "s"}), ("Particles", "long", {}),
                     ("Charge", "double", {"units": "C"}), ("Transmission", "double", {}),
                     ("pCentral", "double", {"symbol": "p$bcen$n", "units": "m$be$nc"}),
                     ("pAverage", "double", {"symbol": "p$bave$n", "units": "m$be$nc"}),
                     ("KAverage", "double", {"symbol": "K$bave$n", "units": "MeV"}),
                     ("Sx", "double", {"units": "m"}), ("Sxp", "double", {}), ("Sy", "double", {"units": "m"}),
                     ("Syp", "double", {}), ("Ss", "double", {"units": "m"}), ("Sdelta", "double", {}),
                     ("St", "double", {"units": "s"}), ("ex", "double", {"units": "m"}),
                     ("ey", "double", {"units": "m"}), ("el", "double", {"units": "s"}),
                     ("ecx", "double", {"units": "m"}), ("ecy", "double", {"units": "m"})]


def _write_watch_parameters(path, records, p_central, z, length, step, charge, w, mode, append, original_particles,
                            previous_element):
    """Parameter (31 columns) or centroid (the first 19) mode: one page per
    step, one row per recorded pass (sdds_support.c:359-393, :538-585,
    :881-1160)."""
    centroid_only = int(w.get("MODE", 1)) == 2
    cols_def = _WATCH_PARAM_COLS[:19] if centroid_only else _WATCH_PARAM_COLS
    times = watch_pass_central_times([r["pass"] for r in records], z, length, p_central,
                                     w.get("REFERENCE_FREQUENCY", -1.0))
    rows = {name: [] for name, _, _ in cols_def}
    for r, t0 in zip(records, times):
        st = watch_statistics(r["coords"], r["ids"], p_central, w.get("START_PID", -1), w.get("END_PID", -1))
        cen, sig = st["centroid"], st["sigma"]
        vals = {"Step": step, "Pass": r["pass"], "ElapsedTime": 0.0, "ElapsedCoreTime": 0.0, "MemoryUsage": 0,
                "Cx": cen[0], "Cxp": cen[1], "Cy": cen[2], "Cyp": cen[3], "Cs": cen[4], "Cdelta": cen[5],
                "Ct": st["Ct"], "dCt": st["Ct"] - t0, "Particles": st["n"], "Charge": charge * st["n"],
                "Transmission": len(r["ids"]) / original_particles if original_particles else 0.0,
                "pCentral": p_central, "pAverage": st["pAverage"], "KAverage": st["KAverage"],
                "Sx": math.sqrt(sig[0, 0]), "Sxp": math.sqrt(sig[1, 1]), "Sy": math.sqrt(sig[2, 2]),
                "Syp": math.sqrt(sig[3, 3]), "Ss": math.sqrt(sig[4, 4]), "Sdelta": math.sqrt(sig[5, 5]),
                "St": math.sqrt(sig[6, 6]), "ex": st["ex"], "ey": st["ey"], "el": st["el"], "ecx": st["ecx"],
                "ecy": st["ecy"]}
        for name, _, _ in cols_def:
            rows[name].append(vals[name])
    params_def = [("Step", "long", {"description": "Simulation step"}), ("s", "double", {"units": "m"}),
                  ("PreviousElementName", "string", {})]
    write_sdds_pages(path, params_def, cols_def,
                     [([step, z, previous_element or "_BEG_"], [rows[name] for name, _, _ in cols_def])],
                     mode, description="watch-point " + ("centroids" if centroid_only else "parameters"),
                     append=append)


def write_watch(path, records, p_central, z, length, step=1, charge=0.0, watch=None, mode="binary", append=False,
                original_particles=0, previous_element=None):
    """A WATCH file.  Parameter and centroid modes: one page per step with a
    row per recorded pass (_write_watch_parameters; original_particles, the
    step's initial count, gives Transmission).  Coordinate mode
    (SDDS_WatchPointSetup, sdds_support.c:403-520;
    dump_watch_particles :703-860), one page per recorded pass, from the
    records of one WATCH (elegant_b200.track.Tracker.watch entries of that
    element, in pass order): columns x, xp, y, yp (X_DATA, Y_DATA; slopes
    left out with EXCLUDE_SLOPES), t = s/(c beta), p = P0 (1 + delta) and
    dt = t - PassCentralTime (LONGIT_DATA), particleID; parameters Step,
    pCentral, Charge (macro charge x particles), Particles, IDSlotsPerBunch,
    SampledCharge, SampledParticles, Pass, PassLength, PassCentralTime, s.
    watch: the element's numeric parameters (X_DATA, START_PID, ...).
    Rows are the particles by ascending ID (elegant keeps its array order);
    START_PID/END_PID select rows."""
    w = dict(watch or {})
    if int(w.get("MODE", 0)) in (1, 2):
        _write_watch_parameters(path, records, p_central, z, length, step, charge, w, mode, append,
                                original_particles, previous_element)
        return
    if int(w.get("MODE", 0)) != 0:
        raise ValueError("WATCH fft mode is not written by this module")
    get = lambda k, d: w.get(k, d)
    x_data, y_data, longit = get("X_DATA", 1), get("Y_DATA", 1), get("LONGIT_DATA", 1)
    slopes = not get("EXCLUDE_SLOPES", 0)
    s_pid, e_pid = get("START_PID", -1), get("END_PID", -1)
    cols_def = []
    if x_data:
        cols_def += [("x", "double", {"units": "m"})] + ([("xp", "double", {})] if slopes else [])
    if y_data:
        cols_def += [("y", "double", {"units": "m"})] + ([("yp", "double", {})] if slopes else [])
    if longit:
        cols_def += [("t", "double", {"units": "s"}), ("p", "double", {"units": "m$be$nc"}),
                     ("dt", "double", {"units": "s"})]
    cols_def += [("particleID", "long", {})]
    params_def = [("Step", "long", {"description": "Simulation step"}),
                  ("pCentral", "double", {"symbol": "p$bcen$n", "units": "m$be$nc",
                                          "description": "Reference beta*gamma"}),
                  ("Charge", "double", {"units": "C", "description": "Bunch charge before sampling"}),
                  ("Particles", "long", {"description": "Number of particles before sampling"}),
                  ("IDSlotsPerBunch", "long", {"description": "Number of particle ID slots reserved to a bunch"}),
                  ("SampledCharge", "double", {"units": "C", "description": "Sampled charge"}),
                  ("SampledParticles", "long", {"description": "Sampled number of particles"}),
                  ("Pass", "long", {}), ("PassLength", "double", {"units": "m"}),
                  ("PassCentralTime", "double", {"units": "s"}), ("s", "double", {"units": "m"})]
    times = watch_pass_central_times([r["pass"] for r in records], z, length, p_central,
                                     get("REFERENCE_FREQUENCY", -1.0))
    pages = []
    for r, t0 in zip(records, times):
        c, ids = r["coords"], r["ids"]
        if s_pid >= 0 or e_pid >= 0:
            keep = (ids >= s_pid) & (ids <= e_pid)
            c, ids = c[keep], ids[keep]
        p = p_central * (1 + c[:, 5])
        t = c[:, 4] / (C_MKS * p / np.sqrt(p * p + 1))
        by = {"x": c[:, 0], "xp": c[:, 1], "y": c[:, 2], "yp": c[:, 3], "t": t, "p": p, "dt": t - t0,
              "particleID": ids.astype(np.int64)}
        n = len(ids)
        pages.append(([step, p_central, charge * n, n, 0, charge * n, n, r["pass"], length, t0, z],
                      [by[name] for name, _, _ in cols_def]))
    write_sdds_pages(path, params_def, cols_def, pages, mode, description="watch-point phase space", append=append)


def write_losses(path, result, lattice, p_central, step=1, mode="binary", append=False):
    """elegant's `losses` file for the lost particles of a TrackResult."""
    lost = result.lost_pass >= 0
    c = result.coords[lost]
    z_end = np.cumsum([e.length for e in lattice.elements])
    s = z_end[result.lost_element[lost].clip(0, len(z_end) - 1)]
    params = [("Step", "long", step, {"description": "Simulation step"})]
    cols = [("x", "double", c[:, 0], {"units": "m"}), ("xp", "double", c[:, 1], {"symbol": "x'"}),
            ("y", "double", c[:, 2], {"units": "m"}), ("yp", "double", c[:, 3], {"symbol": "y'"}),
            ("s", "double", s, {"units": "m"}), ("p", "double", p_central * (1 + c[:, 5]), {"units": "m$be$nc"}),
            ("particleID", "long", result.ids[lost].astype(np.int64), {}),
            ("Pass", "long", result.lost_pass[lost].astype(np.int64), {})]
    write_sdds(path, params, cols, mode, description="elegant_b200 loss output", append=append)


def write_momentum_aperture(path, rows, step=1, mode="binary", output_mode=0, append=False):
    """elegant's &momentum_aperture output from elegant_b200.momentum_aperture
    rows: output_mode 0, one row per element with both sides
    (momentumAperture.c:189-212, :692-714), or output_mode 1, one row per
    element and side, negative (direction -1) first (:141-160, :715-731);
    output_mode 2 from local_momentum_acceptance rows, the two limits per
    element (:163-180).  nuxLost/nuyLost are the last survivor's tunes
    (-1 where rows carry none)."""
    n = len(rows)
    occ = [r["occurrence"] for r in rows] if rows and "occurrence" in rows[0] else _occurrences(rows)
    if output_mode == 1:
        sides = [(r, o, d, side) for r, o in zip(rows, occ) for d, side in ((-1, "negative"), (1, "positive"))]
        cols = [("ElementName", "string", [r["name"] for r, _, _, _ in sides], {}),
                ("s", "double", [r["s"] for r, _, _, _ in sides], {"units": "m"}),
                ("ElementType", "string", [r["type"] for r, _, _, _ in sides], {}),
                ("ElementOccurence", "long", [o for _, o, _, _ in sides], {}),
                ("direction", "short", [d for _, _, d, _ in sides], {}),
                ("deltaFound", "short", [int(r[sd]["found"]) for r, _, _, sd in sides], {}),
                ("delta", "double", [r[sd]["delta"] for r, _, _, sd in sides], {"symbol": "$gd$R$blimit$n"}),
                ("lostOnPass", "long", [r[sd]["lost_on_pass"] for r, _, _, sd in sides], {}),
                ("sLost", "double", [r[sd]["s_lost"] for r, _, _, sd in sides], {"units": "m"}),
                ("xLost", "double", [r[sd]["x_lost"] for r, _, _, sd in sides], {"units": "m"}),
                ("yLost", "double", [r[sd]["y_lost"] for r, _, _, sd in sides], {"units": "m"}),
                ("deltaLost", "double", [r[sd]["delta_when_lost"] for r, _, _, sd in sides], {}),
                ("nuxLost", "double", [r[sd].get("nux", -1.0) for r, _, _, sd in sides], {}),
                ("nuyLost", "double", [r[sd].get("nuy", -1.0) for r, _, _, sd in sides], {})]
        write_sdds(path, [("Step", "long", step, {})], cols, mode, description="Momentum aperture search",
                   append=append)
        return
    if output_mode == 2:
        # multiparticleLocalMomentumAcceptance's page (momentumAperture.c:163-180, :1084-1099)
        cols = [("ElementName", "string", [r["name"] for r in rows], {}),
                ("s", "double", [r["s"] for r in rows], {"units": "m"}),
                ("ElementType", "string", [r["type"] for r in rows], {}),
                ("ElementOccurence", "long", occ, {}),
                ("deltaPositive", "double", [r["positive"]["delta"] for r in rows], {"symbol": "$gd$R$bpos$n"}),
                ("deltaNegative", "double", [r["negative"]["delta"] for r in rows], {"symbol": "$gd$R$bneg$n"})]
        write_sdds(path, [("Step", "long", step, {})], cols, mode, description="Momentum aperture search",
                   append=append)
        return
    if output_mode != 0:
        raise ValueError("output_mode must be 0, 1 or 2")
    cols = [("ElementName", "string", [r["name"] for r in rows], {}),
            ("s", "double", [r["s"] for r in rows], {"units": "m"}),
            ("ElementType", "string", [r["type"] for r in rows], {}),
            ("ElementOccurence", "long", occ, {})]
    for label, side in (("Positive", "positive"), ("Negative", "negative")):
        cols += [(f"delta{label}Found", "short", [int(r[side]["found"]) for r in rows], {}),
                 (f"delta{label}", "double", [r[side]["delta"] for r in rows],
                  {"symbol": "$gd$R$b" + side[:3] + "$n"}),
                 (f"lostOnPass{label}", "long", [r[side]["lost_on_pass"] for r in rows], {}),
                 (f"sLost{label}", "double", [r[side]["s_lost"] for r in rows], {"units": "m"}),
                 (f"xLost{label}", "double", [r[side]["x_lost"] for r in rows], {"units": "m"}),
                 (f"yLost{label}", "double", [r[side]["y_lost"] for r in rows], {"units": "m"}),
                 (f"deltaLost{label}", "double", [r[side]["delta_when_lost"] for r in rows], {}),
                 (f"nuxLost{label}", "double", [r[side].get("nux", -1.0) for r in rows], {}),
                 (f"nuyLost{label}", "double", [r[side].get("nuy", -1.0) for r in rows], {})]
    write_sdds(path, [("Step", "long", step, {})], cols, mode, description="Momentum aperture search",
                   append=append)


def _occurrences(rows):
    seen, out = {}, []
    for r in rows:
        seen[r["name"]] = seen.get(r["name"], 0) + 1
        out.append(seen[r["name"]])
    return out


def write_frequency_map(path, rows, step=1, include_changes=False, mode="binary", append=False):
    """elegant's &frequency_map output (frequencyMap.c:30-60) from
    elegant_b200.frequency_map rows."""
    names = ["x", "y", "delta", "nux", "nuy", "s"]
    if include_changes:
        names += ["dnux", "dnuy", "dnu", "dx", "dy", "diffusion", "diffusionRate"]
    units = {"x": "m", "y": "m", "s": "m/pass", "dx": "m", "dy": "m"}
    cols = [(k, "double", [r[k] for r in rows], {"units": units[k]} if k in units else {}) for k in names]
    write_sdds(path, [("Step", "long", step, {})], cols, mode, description="Frequency map analysis", append=append)


def write_aperture(path, result, step=1, mode="binary", append=False):
    """elegant's &find_aperture output for the line modes
    (aperture_search.c:20-55, :1160-1215) from
    elegant_b200.aperture.find_aperture_lines: the last survivor of each
    line, the clipped limits, the loss point, and the Area parameter."""
    lines = result["lines"]
    if result.get("slope"):
        # slope mode's columns and parameter (aperture_search.c:32-39, :53-57)
        head = [("xp", "double", [l["x"] for l in lines], {}),
                ("yp", "double", [l["y"] for l in lines], {}),
                ("xpClipped", "double", result["x_limit"], {}),
                ("ypClipped", "double", result["y_limit"], {})]
        area_attrs = {}
    else:
        head = [("x", "double", [l["x"] for l in lines], {"symbol": "x", "units": "m"}),
                ("y", "double", [l["y"] for l in lines], {"symbol": "y", "units": "m"}),
                ("xClipped", "double", result["x_limit"], {"symbol": "xClipped", "units": "m"}),
                ("yClipped", "double", result["y_limit"], {"symbol": "yClipped", "units": "m"})]
        area_attrs = {"units": "m$a2$n"}
    cols = head + [
            ("sLost", "double", [l.get("s_lost", 0.0) for l in lines], {"units": "m"}),
            ("xLost", "double", [l["x_lost"] if l["x_lost"] is not None else 1.7976931348623157e308
                                 for l in lines], {"units": "m"}),
            ("yLost", "double", [l["y_lost"] if l["y_lost"] is not None else 1.7976931348623157e308
                                 for l in lines], {"units": "m"})]
    write_sdds(path, [("Step", "long", step, {}), ("Area", "double", result["area"], area_attrs)], cols,
               mode, description="Dynamic aperture search", append=append)


def write_aperture_mp(path, result, step=1, mode="binary", append=False):
    """elegant's &find_aperture output for mode = "many-particle"
    (aperture_search.c:520-552) from one elegant_b200.aperture.find_aperture_mp
    result: the boundary points (left scan, then right scan from the top) in
    x and y; the other columns of the layout and the Area are zero there."""
    pts = result["boundary"]
    n = len(pts)
    cols = [("x", "double", [p[0] for p in pts], {"symbol": "x", "units": "m"}),
            ("y", "double", [p[1] for p in pts], {"symbol": "y", "units": "m"}),
            ("xClipped", "double", [0.0] * n, {"symbol": "xClipped", "units": "m"}),
            ("yClipped", "double", [0.0] * n, {"symbol": "yClipped", "units": "m"}),
            ("sLost", "double", [0.0] * n, {"units": "m"}),
            ("xLost", "double", [0.0] * n, {"units": "m"}),
            ("yLost", "double", [0.0] * n, {"units": "m"})]
    write_sdds(path, [("Step", "long", step, {}), ("Area", "double", 0.0, {"units": "m$a2$n"})], cols, mode,
               description="Dynamic aperture search", append=append)


def csr_wake_columns(page):
    """The OUTPUT_FILE columns of one CSRCSBEND kick from its page record
    (elegant_b200.track.Tracker.csr_pages), with the reference's expressions
    (csbend.c:2762-2806): LinearDensity = ctHist * (q c), LinearDensityDeriv
    = ctHistDeriv * (q c^2 / dct), s = ctLower - (ctLower + ctUpper)/2 + dct
    (i + 1/2), GammaDeriv = DeltaGamma / (L / N_KICKS)."""
    q, dct, lo, hi = page["macro_charge"], page["dct"], page["ct_lower"], page["ct_upper"]
    dgamma = page["dgamma"]
    return {"s": (lo - (lo + hi) / 2.0) + dct * (np.arange(page["bins"]) + 0.5),
            "LinearDensity": page["hist"] * (q * C_MKS),
            "LinearDensityDeriv": page["deriv"] * ((q * (C_MKS * C_MKS)) / dct),
            "DeltaGamma": dgamma, "GammaDeriv": dgamma / page["ds_kick"],
            "DeltaGammaT1": page["t1"], "DeltaGammaT2": page["t2"]}


CSR_WAKE_PARAMETERS = [("SVNVersion", "string", {"description": "SVN version number"}),
                       ("Pass", "long", {}), ("Kick", "long", {}), ("pCentral", "double", {"units": "m$be$nc"}),
                       ("Angle", "double", {}), ("SlippageLength", "double", {"units": "m"}),
                       ("TotalBunchLength", "double", {"units": "m"}), ("BinSize", "double", {"units": "m"}),
                       ("dsKick", "double", {"units": "m"}), ("DerbenevRatio", "double", {})]
CSR_WAKE_COLUMNS = [("s", "double", {"units": "m"}), ("LinearDensity", "double", {"units": "C/s"}),
                    ("LinearDensityDeriv", "double", {"units": "C/s$a2$n"}), ("DeltaGamma", "double", {}),
                    ("GammaDeriv", "double", {"units": "1/m"}), ("DeltaGammaT1", "double", {}),
                    ("DeltaGammaT2", "double", {})]


def write_csr_wake(path, pages, mode="binary", append=False):
    """CSRCSBEND's OUTPUT_FILE (csbend.c:2227-2249 layout, one page per kick,
    :2762-2806) for the page records of one element, in the order given (a
    bunch train: bunch by bunch, as elegant writes consecutive bunches).
    Pass is -1 and DerbenevRatio 0, as the reference writes them with its
    Derbenev criterion off (the default)."""
    out = []
    for pg in pages:
        cols = csr_wake_columns(pg)
        values = ["elegant_b200", -1, pg["kick"], pg["p_central"], pg["angle"], pg["slippage"],
                  pg["ct_upper"] - pg["ct_lower"], pg["dct"], pg["ds_kick"], 0.0]
        out.append((values, [cols[c[0]] for c in CSR_WAKE_COLUMNS]))
    write_sdds_pages(path, CSR_WAKE_PARAMETERS, CSR_WAKE_COLUMNS, out, mode, description="CSR wake output",
                     append=append)


# ---------------------------------------------------------------- input ----
# SDDS type -> numpy dtype code (the byte order is added per file)
_NP = {"double": "f8", "float": "f4", "long": "i4", "ulong": "u4", "long64": "i8", "ulong64": "u8", "short": "i2",
       "ushort": "u2", "char": "S1"}


def _fields(body: str) -> dict:
    """key=value pairs of one namelist body; values may be double-quoted
    (with backslash escapes) and are separated by commas or white space."""
    out, i, n = {}, 0, len(body)
    while i < n:
        if body[i] in " \t\r\n,":
            i += 1
            continue
        eq = body.find("=", i)
        if eq < 0:
            break
        key = body[i:eq].strip().lower()
        i = eq + 1
        while i < n and body[i] in " \t":
            i += 1
        if i < n and body[i] == '"':
            j, buf = i + 1, []
            while j < n and body[j] != '"':
                if body[j] == "\\" and j + 1 < n:
                    j += 1
                buf.append(body[j])
                j += 1
            out[key] = "".join(buf)
            i = j + 1
        else:
            j = i
            while j < n and body[j] not in " \t\r\n,":
                j += 1
            out[key] = body[i:j]
            i = j
    return out


def _ascii_tokens(text: str):
    """White-space separated tokens; double-quoted ones kept whole."""
    toks, i, n = [], 0, len(text)
    while i < n:
        c = text[i]
        if c.isspace():
            i += 1
        elif c == '"':
            j, buf = i + 1, []
            while j < n and text[j] != '"':
                if text[j] == "\\" and j + 1 < n:
                    j += 1
                buf.append(text[j])
                j += 1
            toks.append("".join(buf))
            i = j + 1
        else:
            j = i
            while j < n and not text[j].isspace():
                j += 1
            toks.append(text[i:j])
            i = j
    return toks


def _scalar(typ, tok):
    if typ == "string":
        return tok
    if typ == "char":
        return tok[:1]
    return float(tok) if typ in ("double", "float") else int(tok)


def read_sdds_pages(path):
    """Every page of an SDDS file as a list of (parameters, columns) dicts,
    numeric columns as numpy arrays (native byte order), string columns as
    lists; fixed_value parameters included.  Handles protocol versions 1-5,
    binary data of either byte order (the "!# big-endian" meta-comment),
    row- or column-major binary pages, 64-bit row counts, and ASCII data with
    or without row counts.  Arrays (&array) are not supported."""
    with open(path, "rb") as fh:
        raw = fh.read()
    nl = raw.index(b"\n")
    first = raw[:nl].decode("latin-1").strip()
    if not (first.startswith("SDDS") and first[4:].isdigit()):
        raise ValueError(f"{path}: not an SDDS file")
    pos, order, pending = nl + 1, "<", ""
    params, cols, data = [], [], None
    while data is None:
        nl = raw.find(b"\n", pos)
        if nl < 0:
            raise ValueError(f"{path}: header without &data")
        line = raw[pos:nl].decode("latin-1").strip()
        pos = nl + 1
        if line.startswith("!"):
            order = ">" if "big-endian" in line else ("<" if "little-endian" in line else order)
            continue
        pending = f"{pending} {line}".strip()
        while "&end" in pending:
            k = pending.index("&end")
            cmd, pending = pending[:k].strip(), pending[k + 4:].strip()
            name, _, body = cmd.partition(" ")
            f = _fields(body)
            if name == "&parameter":
                params.append(f)
            elif name == "&column":
                cols.append(f)
            elif name == "&array":
                raise ValueError(f"{path}: SDDS arrays are not supported")
            elif name == "&data":
                data = f
                break
    mode = data.get("mode", "ascii").lower()
    for f in params + cols:
        f["type"] = f.get("type", "double").lower()
    stored = [p for p in params if "fixed_value" not in p]
    fixed = {p["name"]: _scalar(p["type"], p["fixed_value"]) for p in params if "fixed_value" in p}
    pages = []
    if mode == "binary":
        col_major = data.get("column_major_order", "0") not in ("0", "")
        numeric = all(c["type"] != "string" for c in cols)
        while pos + 4 <= len(raw):
            n = int(np.frombuffer(raw, order + "i4", 1, pos)[0])
            pos += 4
            if n == -2 ** 31:
                n = int(np.frombuffer(raw, order + "i8", 1, pos)[0])
                pos += 8
            pv = dict(fixed)
            for p in stored:
                pv[p["name"]], pos = _binary_value(raw, pos, order, p["type"])
            cv = {}
            if col_major:
                for c in cols:
                    if c["type"] == "string":
                        vals = []
                        for _ in range(n):
                            v, pos = _binary_value(raw, pos, order, "string")
                            vals.append(v)
                        cv[c["name"]] = vals
                    else:
                        dt = np.dtype(order + _NP[c["type"]])
                        cv[c["name"]] = np.frombuffer(raw, dt, n, pos).astype(dt.newbyteorder("="))
                        pos += n * dt.itemsize
            elif numeric:
                dt = np.dtype([(c["name"], order + _NP[c["type"]]) for c in cols])
                rows = np.frombuffer(raw, dt, n, pos)
                pos += n * dt.itemsize
                for c in cols:
                    cv[c["name"]] = rows[c["name"]].astype(rows[c["name"]].dtype.newbyteorder("="))
            else:
                vals = {c["name"]: [] for c in cols}
                for _ in range(n):
                    for c in cols:
                        v, pos = _binary_value(raw, pos, order, c["type"])
                        vals[c["name"]].append(v)
                cv = {c["name"]: (vals[c["name"]] if c["type"] == "string" else
                                  np.array(vals[c["name"]], dtype=_NP[c["type"]])) for c in cols}
            pages.append((pv, cv))
    else:
        lines = raw[pos:].decode("latin-1").split("\n")
        skip = int(data.get("additional_header_lines", "0") or 0)
        li = skip
        no_counts = data.get("no_row_counts", "0") not in ("0", "")
        while True:
            while li < len(lines) and (not lines[li].strip() or lines[li].lstrip().startswith("!")):
                li += 1
            if li >= len(lines):
                break
            pv = dict(fixed)
            for p in stored:
                t = lines[li].strip()
                li += 1
                pv[p["name"]] = _scalar(p["type"], t[1:-1] if p["type"] == "string" and t.startswith('"') else t)
            if no_counts:
                body = []
                while li < len(lines) and lines[li].strip():
                    body.append(lines[li])
                    li += 1
            else:
                while li < len(lines) and not lines[li].strip():
                    li += 1
                n = int(lines[li].split()[0])
                li += 1
                body = lines[li:li + n * int(data.get("lines_per_row", "1") or 1)]
                li += len(body)
            toks = _ascii_tokens(" ".join(body))
            k = len(cols)
            n = len(toks) // k if k else 0
            cv = {}
            for j, c in enumerate(cols):
                vals = [_scalar(c["type"], t) for t in toks[j::k][:n]]
                cv[c["name"]] = vals if c["type"] == "string" else np.array(vals, dtype=_NP[c["type"]])
            pages.append((pv, cv))
    return pages


def _binary_value(raw, pos, order, typ):
    if typ == "string":
        k = int(np.frombuffer(raw, order + "i4", 1, pos)[0])
        return raw[pos + 4:pos + 4 + k].decode("latin-1"), pos + 4 + k
    dt = np.dtype(order + _NP[typ])
    v = np.frombuffer(raw, dt, 1, pos)[0]
    return (v.decode("latin-1") if typ == "char" else v.item()), pos + dt.itemsize


def beam_from_sdds(path, p_central, page=0, sample_interval=1, p_lower=0.0, p_upper=0.0, t_offset=0.0):
    """The particles of one page of an elegant phase-space file (columns x,
    xp, y, yp, t, p and optionally particleID), as &sdds_beam reads point
    particles (sdds_beam.c:408-440): s = (t_offset + t) c p / gamma with
    gamma = sqrt(p^2 + 1), delta = (p - p_central) / p_central, every
    sample_interval-th row, rows with p outside [p_lower, p_upper] dropped
    when p_lower is set; IDs from particleID, else the row numbers 1, 2, ...
    of the page."""
    from .beam import Beam
    pages = read_sdds_pages(path)
    if page >= len(pages):
        raise ValueError(f"{path}: page {page} requested, {len(pages)} in the file")
    _, c = pages[page]
    for name in ("x", "xp", "y", "yp", "t", "p"):
        if name not in c:
            raise ValueError(f"{path}: column {name} missing (sdds_beam.c:840-870)")
    n = len(c["x"])
    rows = np.arange(0, n, max(1, int(sample_interval)))
    p = np.asarray(c["p"], dtype=np.float64)[rows]
    keep = np.ones(rows.size, dtype=bool)
    if p_lower:
        keep = ~((p_lower > p) | (p_upper < p))
    rows, p = rows[keep], p[keep]
    gamma = np.sqrt(p * p + 1)
    coords = np.empty((rows.size, 6))
    for j, name in enumerate(("x", "xp", "y", "yp")):
        coords[:, j] = np.asarray(c[name], dtype=np.float64)[rows]
    coords[:, 4] = (t_offset + np.asarray(c["t"], dtype=np.float64)[rows]) * C_MKS * p / gamma
    coords[:, 5] = (p - p_central) / p_central
    if not np.isfinite(coords).all():
        raise ValueError(f"{path}: NaN or Infinity detected in initial particle data (sdds_beam.c:441-448)")
    # without a particleID column the reader numbers the rows as it reads
    # them, before sampling (sdds_beam.c:1005-1007)
    ids = np.asarray(c["particleID"], dtype=np.int64)[rows] if "particleID" in c else (rows + 1).astype(np.int64)
    return Beam(coords, ids)
