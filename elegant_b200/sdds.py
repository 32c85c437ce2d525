"""SDDS output of tracking results, in the layouts elegant writes, for its
post-processing tools (sddsplot, sddsanalyzebeam, ...).

- `write_phase_space`: the &run_setup `final` / `output` file
  (dump_phase_space, sdds_support.c:1531-1604): columns x, xp, y, yp,
  t = s / (c beta), p = P0 (1 + delta), particleID; parameters Step,
  pCentral, Charge, Particles, IDSlotsPerBunch (sdds_support.c:150-170).
- `write_losses`: the `losses` file (sdds_support.c:199-212): x, xp, y, yp, s,
  p, particleID, Pass.  s is the end position of the element where the
  particle was lost (elegant additionally extrapolates aperture losses into
  the preceding drift); the coordinates are those at the loss.

Files are protocol-1 SDDS, binary (little-endian) or ASCII.  particleID is
written as `long` (32-bit), which every SDDS reader accepts; elegant itself
uses ulong64.  `read_sdds` reads what this module writes (for tests and
round trips), not arbitrary SDDS.
"""
from __future__ import annotations

import struct

import numpy as np

C_MKS = 2.99792458e8
_FMT = {"double": ("d", np.float64), "long": ("i", np.int32), "string": (None, None)}


def _quote(v: str) -> str:
    return '"' + v.replace('"', '\\"') + '"'


def write_sdds(path, parameters, columns, mode="binary", description=None):
    """parameters: [(name, type, value, attrs)], columns: [(name, type, array,
    attrs)], types 'double' | 'long' | 'string'; attrs: dict of units,
    symbol, description."""
    if mode not in ("binary", "ascii"):
        raise ValueError("mode must be 'binary' or 'ascii'")
    n = len(columns[0][2]) if columns else 0
    for c in columns:
        if len(c[2]) != n:
            raise ValueError("columns of different lengths")
    lines = ["SDDS1"]
    if mode == "binary":
        lines.append("!# little-endian")
    if description:
        lines.append(f"&description text={_quote(description)}, &end")

    def attrs_text(a):
        return "".join(f" {k}={_quote(str(v))}," for k, v in (a or {}).items())

    for name, typ, _, a in parameters:
        lines.append(f"&parameter name={name},{attrs_text(a)} type={typ}, &end")
    for name, typ, _, a in columns:
        lines.append(f"&column name={name},{attrs_text(a)} type={typ}, &end")
    lines.append(f"&data mode={mode}, &end")
    with open(path, "wb") as fh:
        fh.write(("\n".join(lines) + "\n").encode())
        if mode == "binary":
            fh.write(struct.pack("<i", n))
            for _, typ, v, _ in parameters:
                if typ == "string":
                    b = str(v).encode()
                    fh.write(struct.pack("<i", len(b)) + b)
                else:
                    fh.write(struct.pack("<" + _FMT[typ][0], v))
            if n:
                rec = np.dtype([(c[0], "<" + ("f8" if c[1] == "double" else "i4")) for c in columns])
                rows = np.empty(n, dtype=rec)
                for c in columns:
                    rows[c[0]] = c[2]
                fh.write(rows.tobytes())
        else:
            out = []
            for _, typ, v, _ in parameters:
                out.append(_quote(str(v)) if typ == "string" else repr(float(v)) if typ == "double" else str(int(v)))
            out.append(f"\t{n}")
            cols = [np.asarray(c[2]) for c in columns]
            for i in range(n):
                out.append(" ".join(repr(float(c[i])) if col[1] == "double" else str(int(c[i]))
                                    for c, col in zip(cols, columns)))
            fh.write(("\n".join(out) + "\n").encode())


def read_sdds(path):
    """(parameters dict, columns dict of arrays) of a single-page file written
    by write_sdds."""
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
    if mode == "binary":
        n = struct.unpack_from("<i", data, pos)[0]
        pos += 4
        pv = {}
        for name, typ in params:
            if typ == "string":
                k = struct.unpack_from("<i", data, pos)[0]
                pv[name] = data[pos + 4:pos + 4 + k].decode()
                pos += 4 + k
            else:
                f = _FMT[typ][0]
                pv[name] = struct.unpack_from("<" + f, data, pos)[0]
                pos += struct.calcsize(f)
        rec = np.dtype([(c[0], "<" + ("f8" if c[1] == "double" else "i4")) for c in cols])
        rows = np.frombuffer(data, dtype=rec, count=n, offset=pos)
        return pv, {c[0]: np.array(rows[c[0]]) for c in cols}
    toks = data[pos:].decode().split("\n")
    pv = {}
    for (name, typ), t in zip(params, toks):
        pv[name] = t.strip().strip('"') if typ == "string" else (float(t) if typ == "double" else int(t))
    n = int(toks[len(params)])
    body = [t.split() for t in toks[len(params) + 1:len(params) + 1 + n]]
    out = {}
    for j, (name, typ) in enumerate(cols):
        out[name] = np.array([float(r[j]) if typ == "double" else int(r[j]) for r in body],
                             dtype=np.float64 if typ == "double" else np.int32)
    return pv, out


def write_phase_space(path, result, p_central, step=1, charge=0.0, mode="binary"):
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
    write_sdds(path, params, cols, mode, description="elegant_b200 phase-space output")


def write_losses(path, result, lattice, p_central, step=1, mode="binary"):
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
    write_sdds(path, params, cols, mode, description="elegant_b200 loss output")
