"""Lattice description for the tracking engine: elegant's element types,
parameter names and defaults for the supported subset, plus a reader for the
matching subset of elegant's ``.lte`` syntax.

Parameter names and defaults follow the reference's tables (track_data.c):
``drift_param`` :450, ``edrift_param`` :3174, ``kquad_param`` :1222,
``ksext_param`` :1120, ``csbend_param`` :1893, ``csrcsbend_param`` :1982,
``rfca_param`` :576, ``maxamp_param`` :990, ``charge_param`` :2488,
``csrdrift_param`` :2543.  The .lte grammar handled here is the part of
elegant's parser (get_beamline.c:117, mad_parse.c:886) that lattices of
these element types use: ``NAME: TYPE, P=V, ...``, ``NAME: LINE=(...)`` with
repetition ``n*X`` and reversal ``-X``, ``&`` continuation, ``!`` comments and
``USE``.  Anything outside the subset raises ``LatticeError``.
"""
from __future__ import annotations

import ctypes
import re
from dataclasses import dataclass, field

from . import _native as nat


class LatticeError(ValueError):
    """The lattice uses an element type or parameter the engine does not support."""


# elegant type name -> engine type code; aliases are elegant's synonyms
TYPES = {
    "DRIF": nat.DRIF, "DRIFT": nat.DRIF, "EDRIFT": nat.EDRIFT, "KQUAD": nat.KQUAD, "KSEXT": nat.KSEXT,
    "CSBEND": nat.CSBEND, "RFCA": nat.RFCA, "MAXAMP": nat.MAXAMP, "MARK": nat.MARK, "MARKER": nat.MARK,
    "CHARGE": nat.CHARGE, "CSRCSBEND": nat.CSRCSBEND, "CSRDRIFT": nat.CSRDRIFT, "MALIGN": nat.MALIGN,
    "WATCH": nat.WATCH,
}
TYPE_NAMES = {nat.DRIF: "DRIF", nat.EDRIFT: "EDRIFT", nat.KQUAD: "KQUAD", nat.KSEXT: "KSEXT",
              nat.CSBEND: "CSBEND", nat.RFCA: "RFCA", nat.MAXAMP: "MAXAMP", nat.MARK: "MARK",
              nat.CHARGE: "CHARGE", nat.CSRCSBEND: "CSRCSBEND", nat.CSRDRIFT: "CSRDRIFT", nat.MALIGN: "MALIGN",
              nat.WATCH: "WATCH"}

_KMULT = {"L": 0, "TILT": 2, "DX": 3, "DY": 4, "DZ": 5, "FSE": 6, "N_KICKS": 7, "N_SLICES": 8,
          "INTEGRATION_ORDER": 9, "SYNCH_RAD": 12, "ISR": 13, "ISR1PART": 14, "HKICK": 15, "VKICK": 16,
          "HCALIBRATION": 17, "VCALIBRATION": 18, "BORE": 19, "B": 20}
_BEND = {"L": 0, "ANGLE": 1, "E1": 2, "E2": 3, "TILT": 4, "ETILT": 5, "DX": 6, "DY": 7, "DZ": 8, "FSE": 9,
         "HGAP": 10, "FINT": 11, "N_SLICES": 12, "N_KICKS": 12, "INTEGRATION_ORDER": 13, "EDGE1_EFFECTS": 14,
         "EDGE2_EFFECTS": 15, "EDGE_ORDER": 16, "K1": 17, "K2": 18, "NONLINEAR": 19, "SYNCH_RAD": 35, "ISR": 36,
         "ISR1PART": 37, "XKICK": 38, "YKICK": 39}
_CSRBEND = dict(_BEND, BINS=20, BIN_RANGE_FACTOR=21, SG_HALFWIDTH=22, SG_ORDER=23, SGDERIV_HALFWIDTH=24,
                SGDERIV_ORDER=25, TRAPAZOID_INTEGRATION=26, STEADY_STATE=27, CSR=28, CLIP_NEGATIVE_BINS=29, IGF=30,
                LOW_FREQUENCY_CUTOFF0=31, LOW_FREQUENCY_CUTOFF1=32, HIGH_FREQUENCY_CUTOFF0=33,
                HIGH_FREQUENCY_CUTOFF1=34)

# parameter name -> slot, per engine type
SLOTS = {
    nat.DRIF: {"L": 0, "ORDER": 1},
    nat.EDRIFT: {"L": 0},
    nat.KQUAD: dict(_KMULT, K1=1, EDGE1_EFFECTS=21, EDGE2_EFFECTS=22, EDGE1_LINEAR=23, EDGE2_LINEAR=24,
                    EDGE1_NONLINEAR_FACTOR=25, EDGE2_NONLINEAR_FACTOR=26, I0P=27, I1P=28, I2P=29, I3P=30,
                    LAMBDA2P=31, I0M=32, I1M=33, I2M=34, I3M=35, LAMBDA2M=36, LEFFECTIVE=37),
    nat.KSEXT: dict(_KMULT, K2=1, K1=10, J1=11),
    nat.CSBEND: _BEND,
    nat.CSRCSBEND: _CSRBEND,
    nat.RFCA: {"L": 0, "VOLT": 1, "PHASE": 2, "FREQ": 3, "DX": 4, "DY": 5, "T_REFERENCE": 6, "N_KICKS": 7,
               "FIDUCIAL": 8, "PHASE_REFERENCE": 9},
    nat.MAXAMP: {"X_MAX": 0, "Y_MAX": 1, "ELLIPTICAL": 2, "EXPONENT": 3, "YEXPONENT": 4},
    nat.MARK: {},
    nat.CHARGE: {"TOTAL": 0, "PER_PARTICLE": 1},
    nat.CSRDRIFT: {"L": 0, "N_KICKS": 1, "DZ": 2, "CSR": 3, "USE_STUPAKOV": 4},
    nat.MALIGN: {"DXP": 0, "DYP": 1, "DX": 2, "DY": 3, "DZ": 4, "DT": 5, "DP": 6, "DE": 7, "ON_PASS": 8,
                 "START_PID": 9, "END_PID": 10},
    # WATCH: slots 0-8 are the engine's (include/elegant_b200.h); 9-17 only
    # shape the output file (elegant_b200.sdds.write_watch)
    nat.WATCH: {"START_PASS": 0, "END_PASS": 1, "INTERVAL": 2, "DISABLE": 3, "MODE": 4, "FRACTION": 5,
                "START_PID": 6, "END_PID": 7, "SPARSE_INTERVAL": 8, "X_DATA": 9, "Y_DATA": 10, "LONGIT_DATA": 11,
                "EXCLUDE_SLOPES": 12, "FLUSH_INTERVAL": 13, "USE_DISCONNECT": 14, "INDEX_OFFSET": 15,
                "REFERENCE_FREQUENCY": 16, "AUTO_REFERENCE": 17},
}
# parameters the reference's tracking of these elements never reads (optimizer
# flags, matrix-only options, PITCH/YAW under MALIGN_METHOD 0, malign_mat.c:494-505):
# accepted and kept, without an engine slot
_KMULT_IGNORED = ("HSTEERING", "VSTEERING", "SQRT_ORDER", "PITCH", "YAW")
IGNORED = {nat.KQUAD: _KMULT_IGNORED + ("SR_IN_ORDINARY_MATRIX", "TRACKING_MATRIX"), nat.KSEXT: _KMULT_IGNORED}
# string-valued parameters, kept beside the numeric slots
STRING_PARAMS = {nat.WATCH: ("FILENAME", "LABEL")}
# WATCH MODE strings (matched by prefix, as elegant's match_string) -> B2E_WATCH_MODE codes
WATCH_MODES = (("coord", 0), ("param", 1), ("centroid", 2), ("fft", 3))
# RFCA FIDUCIAL strings (simple_rfca.c:22-27; exact name or unique prefix) -> B2E_FIDUCIAL_* codes
FIDUCIAL_MODES = (("light", 1), ("tmean", 0), ("first", None), ("pmaximum", 2))


def _fiducial_code(name: str, element: str) -> int:
    m = name.strip('"').strip().lower()
    hits = [c for n, c in FIDUCIAL_MODES if n == m] or [c for n, c in FIDUCIAL_MODES if m and n.startswith(m)]
    if len(hits) != 1:
        raise LatticeError(f"RFCA {element}: invalid fiducial mode {name!r} (light, tmean, first, pmaximum)")
    if hits[0] is None:
        raise LatticeError(f"RFCA {element}: FIDUCIAL=first ends every serial elegant run "
                           "(simple_rfca.c:103-111); use tmean, light or pmaximum")
    return hits[0]

# defaults from the reference's parameter tables (only nonzero ones listed)
DEFAULTS = {
    nat.KQUAD: {"N_SLICES": 1, "INTEGRATION_ORDER": 4, "ISR1PART": 1, "HCALIBRATION": 1, "VCALIBRATION": 1,
                "EDGE1_LINEAR": 1, "EDGE2_LINEAR": 1, "EDGE1_NONLINEAR_FACTOR": 1, "EDGE2_NONLINEAR_FACTOR": 1},
    nat.KSEXT: {"N_SLICES": 1, "INTEGRATION_ORDER": 4, "ISR1PART": 1, "HCALIBRATION": 1, "VCALIBRATION": 1},
    nat.CSBEND: {"FINT": 0.5, "N_SLICES": 4, "INTEGRATION_ORDER": 4, "EDGE1_EFFECTS": 1, "EDGE2_EFFECTS": 1,
                 "EDGE_ORDER": 1, "NONLINEAR": 1, "ISR1PART": 1},
    nat.CSRCSBEND: {"FINT": 0.5, "N_SLICES": 4, "INTEGRATION_ORDER": 4, "EDGE1_EFFECTS": 1, "EDGE2_EFFECTS": 1,
                    "EDGE_ORDER": 1, "NONLINEAR": 1, "ISR1PART": 1, "BIN_RANGE_FACTOR": 1.2, "SG_ORDER": 1, "TRAPAZOID_INTEGRATION": 1, "CSR": 1,
                    "CLIP_NEGATIVE_BINS": 1, "LOW_FREQUENCY_CUTOFF0": -1, "LOW_FREQUENCY_CUTOFF1": -1,
                    "HIGH_FREQUENCY_CUTOFF0": -1, "HIGH_FREQUENCY_CUTOFF1": -1},
    nat.RFCA: {"FREQ": 500e6, "T_REFERENCE": -1},
    nat.MAXAMP: {"EXPONENT": 2},
    nat.CSRDRIFT: {"N_KICKS": 1, "CSR": 1},
    nat.MALIGN: {"ON_PASS": -1, "START_PID": -1, "END_PID": -1},
    nat.WATCH: {"END_PASS": -1, "INTERVAL": 1, "FRACTION": 1, "START_PID": -1, "END_PID": -1, "SPARSE_INTERVAL": 1,
                "X_DATA": 1, "Y_DATA": 1, "LONGIT_DATA": 1, "FLUSH_INTERVAL": 100, "REFERENCE_FREQUENCY": -1},
}

LENGTH_TYPES = {nat.DRIF, nat.EDRIFT, nat.KQUAD, nat.KSEXT, nat.CSBEND, nat.RFCA, nat.CSRCSBEND, nat.CSRDRIFT}


@dataclass
class Element:
    """One lattice element: elegant type name, element name and parameters."""

    name: str
    type: str
    params: dict = field(default_factory=dict)
    strings: dict = field(default_factory=dict)

    def __post_init__(self):
        self.type = self.type.upper()
        if self.type not in TYPES:
            raise LatticeError(f"element type {self.type} is not supported by the engine")
        code = TYPES[self.type]
        self.type = TYPE_NAMES[code]
        clean = {}
        strings = {k.upper(): str(v) for k, v in self.strings.items()}
        for k, v in self.params.items():
            k = k.upper()
            if k in STRING_PARAMS.get(code, ()):
                strings[k] = str(v).strip('"')
                continue
            if k == "MODE" and code == nat.WATCH and isinstance(v, str):
                m = v.strip('"').strip().lower()
                codes = [c for prefix, c in WATCH_MODES if m and (prefix.startswith(m) or m.startswith(prefix))]
                if not codes:
                    raise LatticeError(f"WATCH {self.name}: unknown MODE {v!r}")
                v = codes[0]
            if k == "FIDUCIAL" and code == nat.RFCA and isinstance(v, str):
                v = _fiducial_code(v, self.name)
            if k not in SLOTS[code] and k not in IGNORED.get(code, ()):
                raise LatticeError(f"parameter {k} of {self.type} {self.name} is not supported by the engine")
            if k == "N_KICKS" and code in (nat.CSBEND, nat.CSRCSBEND):
                k = "N_SLICES"  # alias sharing storage (track_data.c:1925, :2006)
            clean[k] = float(v)
        self.params = clean
        self.strings = strings

    @property
    def code(self) -> int:
        return TYPES[self.type]

    def get(self, key: str) -> float:
        key = key.upper()
        if key in self.params:
            return self.params[key]
        return float(DEFAULTS.get(self.code, {}).get(key, 0.0))

    @property
    def length(self) -> float:
        return self.get("L") if self.code in LENGTH_TYPES else 0.0

    def slots(self) -> list[float]:
        p = [0.0] * nat.MAX_PARAMS
        for k, v in DEFAULTS.get(self.code, {}).items():
            p[SLOTS[self.code][k]] = float(v)
        for k, v in self.params.items():
            if k in SLOTS[self.code]:
                p[SLOTS[self.code][k]] = v
        return p

    def to_lte(self) -> str:
        names = {c: n for n, c in (("coordinates", 0), ("parameters", 1), ("centroids", 2), ("fft", 3))}
        fid = {c: n for n, c in FIDUCIAL_MODES}
        items = [f'{k}="{names.get(int(v), "coordinates")}"' if (k == "MODE" and self.code == nat.WATCH)
                 else f'{k}="{fid[int(v)]}"' if (k == "FIDUCIAL" and self.code == nat.RFCA)
                 else f"{k}={v!r}" for k, v in self.params.items()]
        items += [f'{k}="{v}"' for k, v in self.strings.items()]
        return f"{self.name}: {self.type}" + ("".join(", " + i for i in items))


class Lattice:
    """An expanded beamline (list of Elements in tracking order)."""

    def __init__(self, elements: list[Element]):
        if not elements:
            raise LatticeError("empty beamline")
        self.elements = list(elements)

    def __len__(self):
        return len(self.elements)

    @property
    def total_length(self) -> float:
        return sum(e.length for e in self.elements)

    def index(self, name: str) -> list[int]:
        return [i for i, e in enumerate(self.elements) if e.name == name]

    def to_ctypes(self) -> ctypes.Array:
        arr = (nat.Element * len(self.elements))()
        for i, e in enumerate(self.elements):
            arr[i].type = e.code
            arr[i].name = e.name.encode()[:31]
            for j, v in enumerate(e.slots()):
                arr[i].p[j] = v
        return arr

    def to_lte(self, line_name: str = "RING") -> str:
        """Write the expanded line as .lte text (one definition per element occurrence)."""
        defs, seen, names = [], {}, []
        for e in self.elements:
            key = e.name
            if key in seen and seen[key] != e.to_lte():
                key = f"{e.name}_{len(seen)}"
                e = Element(key, e.type, dict(e.params))
            if key not in seen:
                seen[key] = e.to_lte()
                defs.append(seen[key])
            names.append(key)
        body = ",".join(names)
        return "\n".join(defs) + f"\n{line_name}: LINE=({body})\nUSE,{line_name}\n"


_TOKEN_NUM = re.compile(r"^[-+]?(\d+\.?\d*|\.\d+)([eEdD][-+]?\d+)?$")


def _value(text: str) -> float:
    t = text.strip().strip('"').strip()
    if _TOKEN_NUM.match(t):
        return float(t.replace("d", "e").replace("D", "e"))
    # elegant accepts RPN expressions in quotes; the subset handled here is
    # plain arithmetic on numbers and the constant pi
    expr = t.replace("pi", "3.141592653589793").replace("PI", "3.141592653589793")
    if re.fullmatch(r"[0-9eE.+\-*/() ]+", expr):
        return float(eval(expr, {"__builtins__": {}}, {}))  # noqa: S307 - digits and operators only
    raise LatticeError(f"cannot evaluate parameter value {text!r}")


def _split_params(s: str) -> list[str]:
    out, depth, cur, quote = [], 0, "", False
    for ch in s:
        if ch == '"':
            quote = not quote
        if ch == "(" and not quote:
            depth += 1
        if ch == ")" and not quote:
            depth -= 1
        if ch == "," and depth == 0 and not quote:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [x.strip() for x in out if x.strip()]


def parse_lte(text: str, use: str | None = None, outputs: dict | None = None) -> Lattice:
    """Read the supported subset of elegant's .lte format and expand the used line.

    outputs: if given, receives CSRCSBEND OUTPUT_FILE names by element name
    (the file is written from the engine's page records, not by the engine
    itself); without it such a parameter is an error."""
    stmts, cur = [], ""
    for raw in text.splitlines():
        line = raw.split("!")[0].rstrip()
        if not line.strip():
            continue
        if line.endswith("&"):
            cur += line[:-1] + " "
            continue
        cur += line
        stmts.append(cur.strip())
        cur = ""
    if cur.strip():
        stmts.append(cur.strip())
    elements: dict[str, Element] = {}
    lines: dict[str, list[str]] = {}
    last_line = None
    for st in stmts:
        up = st.upper()
        if up.startswith("USE"):
            use = use or _split_params(st.split(",", 1)[1] if "," in st else st.split(None, 1)[1])[0].upper()
            continue
        if up.startswith("RETURN"):
            break
        if ":" not in st:
            raise LatticeError(f"cannot parse statement {st!r}")
        name, rest = st.split(":", 1)
        name = name.strip().strip('"').upper()
        rest = rest.strip()
        m = re.match(r"^LINE\s*=\s*\((.*)\)\s*$", rest, flags=re.I | re.S)
        if m:
            lines[name] = _split_params(m.group(1))
            last_line = name
            continue
        parts = _split_params(rest)
        etype = parts[0].upper()
        params = {}
        for p in parts[1:]:
            if "=" not in p:
                raise LatticeError(f"cannot parse parameter {p!r} of {name}")
            k, v = p.split("=", 1)
            if k.strip().upper() == "OUTPUT_FILE" and etype == "CSRCSBEND":
                if outputs is None:
                    raise LatticeError(f"OUTPUT_FILE of {name}: pass outputs= to collect it (elegant_b200.ele)")
                outputs[name] = v.strip().strip('"')
                continue
            if (etype == "WATCH" and k.strip().upper() in ("FILENAME", "LABEL", "MODE")) or \
                    (etype == "RFCA" and k.strip().upper() == "FIDUCIAL"):
                params[k.strip().upper()] = v.strip().strip('"')
                continue
            params[k.strip().upper()] = _value(v)
        if etype in elements:
            base = elements[etype]
            merged = dict(base.params)
            merged.update(base.strings)
            merged.update(params)
            elements[name] = Element(name, base.type, merged)
        else:
            elements[name] = Element(name, etype, params)

    def expand(item: str, depth: int = 0) -> list[Element]:
        if depth > 64:
            raise LatticeError("beamline nesting too deep")
        item = item.strip()
        rep = 1
        m = re.match(r"^(\d+)\s*\*\s*(.+)$", item)
        if m:
            rep, item = int(m.group(1)), m.group(2).strip()
        reverse = item.startswith("-")
        if reverse:
            item = item[1:].strip()
        if item.startswith("(") and item.endswith(")"):
            seq = []
            for sub in _split_params(item[1:-1]):
                seq += expand(sub, depth + 1)
        else:
            key = item.upper()
            if key in lines:
                seq = []
                for sub in lines[key]:
                    seq += expand(sub, depth + 1)
            elif key in elements:
                seq = [elements[key]]
            else:
                raise LatticeError(f"undefined element or line {item}")
        if reverse:
            seq = seq[::-1]
        return seq * rep

    target = (use or last_line or "").upper()
    if not target:
        raise LatticeError("no beamline to use")
    return Lattice(expand(target))
