"""A reader of SDDS files written from the protocol's description (version 1
to 5 headers; ASCII and binary data, either byte order, row- or
column-major), kept apart from elegant_b200.sdds so that the writer is not
checked by its own reader.  Test infrastructure.

Header: the first line is "SDDSn"; then namelist commands -- &description,
&parameter, &column, &array, &associate, &include, &data -- each "&name
key=value ... &end", fields separated by commas or white space (values
optionally double-quoted, quotes escaped by a backslash); lines starting
with "!" are comments, and the meta-comment "!# big-endian" /
"!# little-endian" states the byte order of binary data.
&data sets mode (ascii | binary), lines_per_row, no_row_counts,
column_major_order and additional_header_lines.

Binary page: the row count (int32; the value INT32_MIN announces an int64
count), the parameters without fixed_value in definition order, then the
columns -- row by row, or column by column when column_major_order is set.
Strings are an int32 length and that many bytes.

ASCII page: one line per parameter without fixed_value, then (unless
no_row_counts) a line with the row count, then the rows, values separated by
white space, strings double-quoted when they contain white space.
"""
from __future__ import annotations

import struct

import numpy as np

_SIZES = {"double": "d", "float": "f", "long": "i", "ulong": "I", "long64": "q", "ulong64": "Q", "short": "h",
          "ushort": "H", "char": "c"}


def _namelist(text):
    """'&name k=v, k="v, w", &end' -> (name, {k: v})."""
    text = text.strip()
    assert text.startswith("&") and text.endswith("&end"), text
    body = text[1:-4]
    name, _, rest = body.partition(" ")
    fields, i, n = {}, 0, len(rest)
    while i < n:
        while i < n and rest[i] in " \t,":
            i += 1
        if i >= n:
            break
        j = rest.index("=", i)
        key = rest[i:j].strip().lower()
        i = j + 1
        while i < n and rest[i] in " \t":
            i += 1
        if i < n and rest[i] == '"':
            buf, i = [], i + 1
            while rest[i] != '"':
                if rest[i] == "\\":
                    i += 1
                buf.append(rest[i])
                i += 1
            value, i = "".join(buf), i + 1
        else:
            j = i
            while j < n and rest[j] not in ", \t":
                j += 1
            value, i = rest[i:j], j
        fields[key] = value
    return name.strip().lower(), fields


def _tokens(line):
    out, i = [], 0
    while i < len(line):
        c = line[i]
        if c.isspace():
            i += 1
        elif c == '"':
            buf, i = [], i + 1
            while line[i] != '"':
                if line[i] == "\\":
                    i += 1
                buf.append(line[i])
                i += 1
            out.append("".join(buf))
            i += 1
        else:
            j = i
            while j < len(line) and not line[j].isspace():
                j += 1
            out.append(line[i:j])
            i = j
    return out


def _convert(typ, token):
    if typ == "string":
        return token
    if typ == "char":
        return token[:1]
    if typ in ("double", "float"):
        return float(token)
    return int(token)


class SddsFile:
    """parameters: [{name, type, fixed_value, ...}]; columns: [{name, type,
    ...}]; pages: [{"parameters": {name: value}, "columns": {name: array}}]."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            raw = fh.read()
        self.parameters, self.columns, self.arrays, self.description = [], [], [], {}
        self.endian = "<"
        pos = 0
        first = True
        data = None
        pending = ""
        while data is None:
            end = raw.index(b"\n", pos)
            line = raw[pos:end].decode("latin-1").rstrip("\r")
            pos = end + 1
            if first:
                assert line.startswith("SDDS") and line[4:].strip().isdigit(), line
                self.version = int(line[4:].strip())
                first = False
                continue
            if line.startswith("!"):
                if "big-endian" in line:
                    self.endian = ">"
                elif "little-endian" in line:
                    self.endian = "<"
                continue
            pending = (pending + " " + line).strip() if pending else line.strip()
            while "&end" in pending:
                k = pending.index("&end") + 4
                cmd, pending = pending[:k], pending[k:].strip()
                name, fields = _namelist(cmd)
                if name == "parameter":
                    self.parameters.append(fields)
                elif name == "column":
                    self.columns.append(fields)
                elif name == "array":
                    self.arrays.append(fields)
                elif name == "description":
                    self.description = fields
                elif name == "data":
                    data = fields
        self.mode = data.get("mode", "binary").lower()
        self.column_major = int(data.get("column_major_order", "0") or 0) != 0
        self.no_row_counts = int(data.get("no_row_counts", "0") or 0) != 0
        for _ in range(int(data.get("additional_header_lines", "0") or 0)):
            pos = raw.index(b"\n", pos) + 1
        if self.arrays:
            raise NotImplementedError("arrays")
        self.pages = self._binary(raw, pos) if self.mode == "binary" else self._ascii(raw[pos:].decode("latin-1"))

    # -- binary ---------------------------------------------------------
    def _binary(self, raw, pos):
        e = self.endian
        pages = []

        def scalar(typ):
            nonlocal pos
            if typ == "string":
                (k,) = struct.unpack_from(e + "i", raw, pos)
                pos += 4
                v = raw[pos:pos + k].decode("latin-1")
                pos += k
                return v
            code = _SIZES[typ]
            (v,) = struct.unpack_from(e + code, raw, pos)
            pos += struct.calcsize(code)
            return v.decode("latin-1") if typ == "char" else v

        while pos < len(raw):
            (rows,) = struct.unpack_from(e + "i", raw, pos)
            pos += 4
            if rows == -(2 ** 31):
                (rows,) = struct.unpack_from(e + "q", raw, pos)
                pos += 8
            params = {}
            for p in self.parameters:
                params[p["name"]] = _convert(p["type"], p["fixed_value"]) if "fixed_value" in p else scalar(p["type"])
            cols = {c["name"]: [None] * rows for c in self.columns}
            if self.column_major:
                for c in self.columns:
                    for r in range(rows):
                        cols[c["name"]][r] = scalar(c["type"])
            else:
                for r in range(rows):
                    for c in self.columns:
                        cols[c["name"]][r] = scalar(c["type"])
            pages.append({"parameters": params, "columns": {k: self._array(k, v) for k, v in cols.items()}})
        assert pos == len(raw), "trailing bytes after the last page"
        return pages

    # -- ascii ----------------------------------------------------------
    def _ascii(self, text):
        lines = [ln for ln in text.split("\n") if not ln.startswith("!")]
        i, pages = 0, []
        while True:
            while i < len(lines) and not lines[i].strip():
                i += 1
            if i >= len(lines):
                break
            params = {}
            for p in self.parameters:
                if "fixed_value" in p:
                    params[p["name"]] = _convert(p["type"], p["fixed_value"])
                    continue
                line = lines[i]
                i += 1
                tok = _tokens(line) if p["type"] != "string" or line.strip().startswith('"') else [line.strip()]
                params[p["name"]] = _convert(p["type"], tok[0] if tok else "")
            if self.no_row_counts:
                rows_text = []
                while i < len(lines) and lines[i].strip():
                    rows_text.append(lines[i])
                    i += 1
            else:
                while not lines[i].strip():
                    i += 1
                rows = int(lines[i].split()[0])
                i += 1
                rows_text = lines[i:i + rows]
                i += rows
            cols = {c["name"]: [] for c in self.columns}
            for line in rows_text:
                tok = _tokens(line)
                assert len(tok) == len(self.columns), (line, self.columns)
                for c, t in zip(self.columns, tok):
                    cols[c["name"]].append(_convert(c["type"], t))
            pages.append({"parameters": params, "columns": {k: self._array(k, v) for k, v in cols.items()}})
        return pages

    def _array(self, name, values):
        typ = next(c["type"] for c in self.columns if c["name"] == name)
        if typ in ("string", "char"):
            return list(values)
        return np.asarray(values, dtype=np.float64 if typ in ("double", "float") else np.int64)
