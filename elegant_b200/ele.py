"""The subset of elegant's run file (.ele) that drives tracking on the engine.

elegant reads namelist commands (namelist.h syntax: ``&name key = value,
key[1] = value, key[0] = 3*value, ... &end``) and runs them in order
(elegant.c, main command loop).  For a tracking job the commands on this
path are

- &run_setup (elegant.nl:21-61): lattice, use_beamline, rootname,
  p_central / p_central_mev, default_order, random_number_seed, and the
  phase-space files final and output (both written with the beam at the end
  of the step: this runner has no per-pass output) and losses; ``%s`` in a
  file name is the rootname (the .ele file's name without extension, as
  elegant's compose_filename forms it);
- &run_control (vary.nl:8-19): n_steps, n_passes;
- &bunched_beam (bunched_beam.nl:9-60): Gaussian beams matched to the given
  Twiss parameters, emittances (geometric, or normalised emit_n / beta
  gamma), sigma_dp, sigma_s, dp_s_coupling, momentum_chirp, centroid,
  distribution_cutoff (a Gaussian truncated at that many sigma, values
  redrawn), enforce_rms_values (the sample's emittance made exact; its
  Twiss parameters always are, as generate_bunch does), symmetrize (each
  particle with its mirror images, so odd moments vanish),
  n_particles_per_bunch;
- &sdds_beam (sdds_beam.nl): an elegant phase-space file (x, xp, y, yp, t,
  p, optionally particleID), one page per step after n_tables_to_skip (the
  first with reuse_bunch), sample_interval, p_lower/p_upper, converted as
  elegant converts point particles (elegant_b200.sdds.beam_from_sdds);
- &twiss_output with matched = 1 and &bunched_beam use_twiss_command_values
  = 1: the beam is matched to the periodic Twiss parameters of the line;
- &track: runs n_steps steps of n_passes passes;
- &find_aperture (aperture_search.nl): the many-particle mode, the one- to
  eleven-line modes and n-line, slope mode (xmin == xmax) and
  optimization_mode (the area only, no file), with setup_aperture_search's
  checks; the output file per step;
- &momentum_aperture (momentumAperture.nl): every key, fiducialize and
  forbid_resonance_crossing included; output_mode 0, 1, and 2 (Pelegant's
  grid search, run here on the batched engine).

A command outside this list, or a key of these commands away from its
default that the engine does not implement, raises EleError naming it: the
job belongs to elegant, not to this engine.  elegant's random-number streams
(the SDDS toolkit's generators) are not in the reference tree, so beams are
drawn from numpy's PCG64 seeded with random_number_seed: the same
distribution, not the same particles.

CSRCSBEND OUTPUT_FILE (a string parameter of the .lte) is written through
the engine's page records (Tracker.set_csr_pages, sdds.write_csr_wake);
coordinate-mode WATCH elements (FILENAME) through the engine's WATCH records
(Tracker.set_watch, sdds.write_watch), one page per recorded pass.
"""
from __future__ import annotations

import math
import os
import re

import numpy as np

from .beam import Beam, ME_MEV
from .lattice import parse_lte


class EleError(ValueError):
    """A run file the engine does not run."""


# ------------------------------------------------------------------ parsing ----
def _strip_comments(text: str) -> str:
    """Drop everything from an unquoted "!" to the end of its line."""
    out = []
    for line in text.splitlines():
        quote, cut = False, len(line)
        i = 0
        while i < len(line):
            ch = line[i]
            if ch == "\\" and quote:
                i += 2
                continue
            if ch == '"':
                quote = not quote
            elif ch == "!" and not quote:
                cut = i
                break
            i += 1
        out.append(line[:cut])
    return "\n".join(out)


def _quoted(body: str, pos: int):
    """The string starting at the quote at pos (backslash escapes kept as
    the escaped character) and the position after its closing quote."""
    out, i = [], pos + 1
    while i < len(body) and body[i] != '"':
        if body[i] == "\\" and i + 1 < len(body):
            i += 1
        out.append(body[i])
        i += 1
    if i >= len(body):
        raise EleError("unterminated string in a namelist")
    return "".join(out), i + 1


def _tokens(body: str):
    """Split a namelist body into (key, index, values) assignments."""
    pos, n = 0, len(body)
    items = []
    while pos < n:
        m = re.compile(r"\s*,?\s*([A-Za-z_][A-Za-z0-9_]*)\s*(\[\s*(\d+)\s*\])?\s*=\s*").match(body, pos)
        if not m:
            rest = body[pos:].strip(" \t\r\n,")
            if rest:
                raise EleError(f"cannot parse namelist text near {rest[:40]!r}")
            break
        key, index = m.group(1).lower(), int(m.group(3)) if m.group(3) else 0
        pos = m.end()
        values = []
        while True:
            while pos < n and body[pos] in " \t\r\n":
                pos += 1
            rep = 1
            mr = re.compile(r"(\d+)\*").match(body, pos)
            if mr:
                rep, pos = int(mr.group(1)), mr.end()
            if pos < n and body[pos] == '"':
                v, pos = _quoted(body, pos)
            else:
                j = pos
                while j < n and body[j] not in ", \t\r\n":
                    j += 1
                v, pos = body[pos:j], j
            values += [v] * rep
            k = pos
            while k < n and body[k] in " \t\r\n":
                k += 1
            if k < n and body[k] == ",":
                # another value of the same key follows unless a new
                # assignment or the end of the command does
                if re.compile(r",\s*[A-Za-z_][A-Za-z0-9_]*\s*(\[\s*\d+\s*\])?\s*=").match(body, k) or \
                        not body[k + 1:].strip():
                    pos = k + 1
                    break
                pos = k + 1
                continue
            pos = k
            break
        items.append((key, index, values))
    return items


def _commands(text: str):
    """(name, body) of every "&name ... &end", skipping quoted text."""
    i, n = 0, len(text)
    while True:
        i = text.find("&", i)
        if i < 0:
            return
        m = re.compile(r"&([A-Za-z_][A-Za-z0-9_]*)").match(text, i)
        if not m or m.group(1).lower() == "end":
            i += 1
            continue
        j, quote = m.end(), False
        while j < n:
            if text[j] == "\\" and quote:
                j += 2
                continue
            if text[j] == '"':
                quote = not quote
            elif not quote and text.startswith("&end", j):
                break
            j += 1
        yield m.group(1).lower(), text[m.end():j]
        i = j + 4


def parse_namelists(text: str):
    """[(command, {key: value or [values]})] in file order; values are
    strings, converted by the consumer against the command's defaults."""
    text = _strip_comments(text)
    out = []
    for name, body in _commands(text):
        fields = {}
        for key, index, values in _tokens(body):
            if index == 0 and len(values) == 1 and key not in fields:
                fields[key] = values[0]
            else:
                cur = fields.get(key)
                arr = list(cur) if isinstance(cur, list) else ([cur] if cur is not None else [])
                while len(arr) < index + len(values):
                    arr.append(None)
                arr[index:index + len(values)] = values
                fields[key] = arr
        out.append((name, fields))
    return out


# ----------------------------------------------------------------- commands ----
RUN_SETUP = {"lattice": None, "use_beamline": None, "rootname": None, "output": None, "final": None,
             "losses": None, "default_order": 2, "random_number_seed": 987654321, "p_central": 0.0,
             "p_central_mev": 0.0, "print_statistics": 0, "concat_order": 0, "wrap_around": 1,
             "tracking_updates": 1, "echo_lattice": 0, "show_element_timing": 0, "monitor_memory_usage": 0,
             "semaphore_file": None, "search_path": None, "final_pass": 0, "always_change_p0": 0,
             "back_tracking": 0, "element_divisions": 0, "s_start": 0.0, "load_balancing_on": 0,
             "random_sequence_no": 1, "correction_iterations": 1, "suppress_parameter_defaults": 0,
             "combine_bunch_statistics": 0, "losses_include_global_coordinates": 0, "expand_for": None}
RUN_SETUP_UNSUPPORTED_FILES = ("centroid", "bpm_centroid", "sigma", "acceptance", "magnets", "parameters",
                               "rfc_reference_output")
RUN_CONTROL = {"n_steps": 1, "n_passes": 1, "bunch_frequency": 0.0, "n_indices": 0, "n_passes_fiducial": 0,
               "terminate_on_failure": 0, "reset_rf_for_each_step": 1, "first_is_fiducial": 0,
               "restrict_fiducialization": 0, "reset_scattering_seed": 0}
BUNCHED_BEAM = {"bunch": None, "n_particles_per_bunch": 1, "time_start": 0.0, "matched_to_cell": None,
                "emit_x": 0.0, "emit_nx": 0.0, "beta_x": 1.0, "alpha_x": 0.0, "eta_x": 0.0, "etap_x": 0.0,
                "emit_y": 0.0, "emit_ny": 0.0, "beta_y": 1.0, "alpha_y": 0.0, "eta_y": 0.0, "etap_y": 0.0,
                "use_twiss_command_values": 0, "use_moments_output_values": 0, "po": 0.0, "sigma_dp": 0.0,
                "sigma_s": 0.0, "dp_s_coupling": 0.0, "emit_z": 0.0, "beta_z": 0.0, "alpha_z": 0.0,
                "momentum_chirp": 0.0, "one_random_bunch": 1, "save_initial_coordinates": 1,
                "limit_invariants": 0, "symmetrize": 0, "halton_sequence": [0, 0, 0], "optimized_halton": 0,
                "randomize_order": [0, 0, 0], "limit_in_4d": 0, "enforce_rms_values": [0, 0, 0],
                "distribution_cutoff": [2.0, 2.0, 2.0],
                "distribution_type": ["gaussian", "gaussian", "gaussian"],
                "centroid": [0.0] * 6, "first_is_fiducial": 0, "multiply_np_by_cores": 0,
                "halton_radix": [0] * 6}
TRACK = {"center_on_orbit": 0, "center_momentum_also": 1, "offset_by_orbit": 0, "offset_momentum_also": 1,
         "soft_failure": 1, "use_linear_chromatic_matrix": 0, "longitudinal_ring_only": 0, "ibs_only": 0,
         "stop_tracking_particle_limit": -1, "check_beam_structure": 0, "interrupt_file": "%s.interrupt"}
TWISS_OUTPUT = {"matched": 1, "filename": None, "output_at_each_step": 0, "statistics": 0, "radiation_integrals": 0,
                "beta_x": 1.0, "alpha_x": 0.0, "eta_x": 0.0, "etap_x": 0.0, "beta_y": 1.0, "alpha_y": 0.0,
                "eta_y": 0.0, "etap_y": 0.0, "concat_order": 0}
SDDS_BEAM = {"input": None, "input_list": None, "input_type": "elegant", "selection_parameter": None,
             "selection_string": None, "one_random_bunch": 0, "n_particles_per_ring": 0, "reuse_bunch": 0,
             "prebunched": -1, "track_pages_separately": 0, "use_bunched_mode": 0, "fiducialization_bunch": 0,
             "sample_interval": 1, "n_tables_to_skip": 0, "center_transversely": 0, "center_arrival_time": 0,
             "reverse_t_sign": 0, "sample_fraction": 1.0, "p_lower": 0.0, "p_upper": 0.0,
             "save_initial_coordinates": 1, "n_duplicates": 0, "duplicate_stagger": [0.0] * 6}
FIND_APERTURE = {"output": None, "search_output": None, "boundary": None, "mode": "many-particle", "xmin": -0.1,
                 "xmax": 0.1, "xpmin": 0.0, "xpmax": 0.0, "ymin": 0.0, "ymax": 0.1, "ypmin": 0.0, "ypmax": 0.0,
                 "nx": 21, "n_splits": 0, "split_fraction": 0.5, "desired_resolution": 0.01, "ny": 11,
                 "verbosity": 0, "assume_nonincreasing": 0, "offset_by_orbit": 0, "n_lines": 11, "full_plane": 0,
                 "optimization_mode": 0}
MOMENTUM_APERTURE = {"output": None, "x_initial": 1e-5, "y_initial": 1e-5, "delta_negative_limit": -0.10,
                     "delta_positive_limit": 0.10, "delta_negative_start": 0.0, "delta_positive_start": 0.0,
                     "delta_step_size": 0.0025, "splits": 1, "steps_back": 1, "split_step_divisor": 10,
                     "skip_elements": 0, "process_elements": 2147483647, "s_start": 0.0, "s_end": 1.7976931348623157e308,
                     "include_name_pattern": None, "include_type_pattern": None, "fiducialize": 0, "verbosity": 1,
                     "soft_failure": 0, "output_mode": 0, "forbid_resonance_crossing": 0,
                     "allow_watch_file_output": 0}
# device memory the runner lets WATCH recording take per step
WATCH_BUDGET_BYTES = 8 << 30
# commands that change nothing the tracking path computes
INERT = {"global_settings", "print_dictionary", "semaphores", "stop", "subprocess", "run_rpnexpr"}
LINE_MODE_LINES = {"one-line": 1, "two-line": 2, "three-line": 3, "five-line": 5, "seven-line": 7, "nine-line": 9,
                   "eleven-line": 11}


def _check_find_aperture(fa: dict) -> tuple[str, bool, int]:
    """setup_aperture_search's checks (aperture_search.c:118-170).  Returns
    (mode, slope mode, lines)."""
    if not fa["output"] and not fa["optimization_mode"]:
        raise EleError("&find_aperture: no output filename specified (required if optimization_mode=0)")
    slope = fa["xmin"] == fa["xmax"]
    if slope:
        if fa["xpmin"] == fa["xpmax"] or fa["ypmin"] == fa["ypmax"]:
            raise EleError("&find_aperture: if xmin==xmax, must not have xpmin==xpmax or ypmin==ypmax")
        if fa["ymin"] != fa["ymax"]:
            raise EleError("&find_aperture: if xmin==xmax, must also have ymin==ymax")
    else:
        if fa["xmin"] >= fa["xmax"]:
            raise EleError("&find_aperture: xmin >= xmax")
        if fa["ymin"] >= fa["ymax"]:
            raise EleError("&find_aperture: ymin >= ymax")
        if fa["xpmin"] != fa["xpmax"] or fa["ypmin"] != fa["ypmax"]:
            raise EleError("&find_aperture: if xmin!=xmax, must have xpmin==xpmax and ypmin==ypmax")
    if fa["nx"] < 3:
        raise EleError("&find_aperture: nx < 3")
    if fa["ny"] < 2:
        raise EleError("&find_aperture: ny < 2")
    if fa["n_splits"]:
        if not 0 < fa["split_fraction"] < 1:
            raise EleError("&find_aperture: split_fraction must be greater than 0 and less than 1")
        if not 0 < fa["desired_resolution"] < 1:
            raise EleError("&find_aperture: desired_resolution must be greater than 0 and less than 1")
        if fa["desired_resolution"] * (fa["xmax"] - fa["xmin"]) > (fa["xmax"] - fa["xmin"]) / (fa["nx"] - 1):
            raise EleError("&find_aperture: desired_resolution is larger than coarse mesh")
    mode = fa["mode"]
    if mode == "n-line":
        lines = fa["n_lines"]
    elif mode in LINE_MODE_LINES:
        lines = LINE_MODE_LINES[mode]
    elif mode == "many-particle":
        lines = 0
    else:
        raise EleError(f"&find_aperture: mode {mode!r} is not supported by the engine's runner")
    if slope and mode != "n-line":
        raise EleError('&find_aperture: slope-based aperture search only supported for mode="n-line"')
    if fa["full_plane"] and mode == "many-particle":
        raise EleError("&find_aperture: full_plane=1 is only supported for line-based modes at present")
    if fa["optimization_mode"] and (mode in ("many-particle", "one-line", "two-line") or
                                    (mode == "n-line" and lines < 3)):
        raise EleError("&find_aperture: dynamic aperture optimization requires use of n-line mode with at "
                       "least 3 lines")
    return mode, slope, lines


def _convert(default, value):
    if isinstance(default, list):
        vals = value if isinstance(value, list) else [value]
        out = list(default)
        for i, v in enumerate(vals):
            if v is not None:
                out[i] = _convert(default[i] if i < len(default) else default[-1], v)
        return out
    if isinstance(default, float):
        return float(value)
    if isinstance(default, int) and not isinstance(default, bool):
        return int(float(value))
    return value


def _command(fields: dict, defaults: dict, name: str, allowed: set) -> dict:
    out = dict(defaults)
    for k, v in fields.items():
        if k not in defaults:
            raise EleError(f"&{name}: {k} is not a parameter the engine's runner knows")
        out[k] = _convert(defaults[k], v)
        if k not in allowed and out[k] != defaults[k]:
            raise EleError(f"&{name}: {k} = {v!r} is not supported by the engine's runner")
    return out


# ------------------------------------------------------------------ beam ----
def _truncated_normal(rng, shape, cutoff):
    g = rng.standard_normal(shape)
    if cutoff and cutoff > 0:
        bad = np.abs(g) > cutoff
        while bad.any():
            g[bad] = rng.standard_normal(int(bad.sum()))
            bad = np.abs(g) > cutoff
    return g


def _plane(u, eps, beta, alpha):
    """transform_from_normalized_coordinates: (u, u') of unit emittance to
    the plane's (x, x') at (beta, alpha, eps)."""
    x = math.sqrt(eps * beta) * u[:, 0]
    xp = math.sqrt(eps / beta) * (u[:, 1] - alpha * u[:, 0])
    return np.stack([x, xp], axis=1)


def _enforce_twiss(c, beta1, alpha1, emit1, enforce_rms):
    """elegant's enforceTwissValues (generate_bunch.c:1307-1335): the linear
    map that takes the sample's own Twiss ellipse to (beta1, alpha1), scaled
    to emittance emit1 when enforce_rms is set."""
    d = c - c.mean(axis=0)
    s11, s12, s22 = (d[:, 0] ** 2).mean(), (d[:, 0] * d[:, 1]).mean(), (d[:, 1] ** 2).mean()
    emit = math.sqrt(max(s11 * s22 - s12 * s12, 0.0))
    if not emit or not beta1:
        return c
    beta, alpha = s11 / emit, -s12 / emit
    bm = math.sqrt(beta1 * beta)
    r11, r21, r22 = beta1 / bm, (alpha - alpha1) / bm, beta / bm
    if enforce_rms:
        ratio = math.sqrt(emit1 / emit)
        r11, r21, r22 = r11 * ratio, r21 * ratio, r22 * ratio
    out = np.empty_like(c)
    out[:, 1] = c[:, 0] * r21 + c[:, 1] * r22
    out[:, 0] = c[:, 0] * r11
    return out


def bunched_beam(bb: dict, p_central: float, seed: int, twiss=None) -> Beam:
    """A Gaussian bunch from &bunched_beam values, generated the way
    generate_bunch (generate_bunch.c:57-480) builds one: per plane a
    truncated unit Gaussian (values beyond distribution_cutoff redrawn),
    mirrored into four quadrants with symmetrize, centred, transformed to the
    plane's (beta, alpha, emittance) -- the longitudinal plane's from
    sigma_s, sigma_dp and dp_s_coupling (:318-349) -- and then mapped so that
    the sample's own Twiss parameters are exactly the requested ones, its
    emittance too with enforce_rms_values (enforceTwissValues, :1307-1335);
    then the chirp, dispersion and centroid."""
    n = int(bb["n_particles_per_bunch"])
    sym = int(bb["symmetrize"])
    if sym and n % 4:
        raise EleError("&bunched_beam: symmetrize needs n_particles_per_bunch divisible by 4")
    for t in bb["distribution_type"]:
        if t.lower() != "gaussian":
            raise EleError(f"&bunched_beam: distribution_type {t!r} is not supported by the engine's runner")
    rng = np.random.Generator(np.random.PCG64(seed))
    m = n // 4 if sym else n
    cut = bb["distribution_cutoff"]
    enforce = bb["enforce_rms_values"]
    # mirror signs of the four copies per plane: every odd moment of a plane
    # and every product of two planes' coordinates cancels
    mirror = ((1, -1, 1, -1), (1, 1, -1, -1), (1, -1, -1, 1))
    c = np.empty((n, 6))
    specs = []
    for k, (emit, emit_n, beta, alpha) in enumerate(
            ((bb["emit_x"], bb["emit_nx"], bb["beta_x"], bb["alpha_x"]),
             (bb["emit_y"], bb["emit_ny"], bb["beta_y"], bb["alpha_y"]))):
        if twiss is not None:
            beta, alpha = (twiss.beta_x, twiss.alpha_x) if k == 0 else (twiss.beta_y, twiss.alpha_y)
        specs.append((emit if emit else emit_n / p_central, beta, alpha))
    sig_s, sig_dp, coupling = bb["sigma_s"], bb["sigma_dp"], bb["dp_s_coupling"]
    s56 = sig_dp * sig_s * coupling
    emit_z = math.sqrt(max((sig_dp * sig_s) ** 2 - s56 * s56, 0.0))
    specs.append((emit_z, sig_s * sig_s / emit_z, -s56 / emit_z) if emit_z else (0.0, 0.0, 0.0))
    for k, (eps, beta, alpha) in enumerate(specs):
        u = _truncated_normal(rng, (m, 2), cut[k])
        if sym:
            u = np.concatenate([u * sgn for sgn in mirror[k]])
        u -= u.mean(axis=0)
        if beta:
            pl = _plane(u, eps, beta, alpha)
            pl = _enforce_twiss(pl, beta, alpha, eps, int(enforce[k]))
        else:  # no longitudinal emittance: independent s and delta
            pl = u * np.array([sig_s, sig_dp])
        c[:, 2 * k:2 * k + 2] = pl
    c[:, 5] += bb["momentum_chirp"] * c[:, 4]
    eta = (bb["eta_x"], bb["etap_x"], bb["eta_y"], bb["etap_y"])
    if twiss is not None:
        eta = (twiss.eta_x, twiss.etap_x, 0.0, 0.0)
    for k in range(4):
        c[:, k] += eta[k] * c[:, 5]
    c += np.asarray(bb["centroid"], dtype=np.float64)[None, :]
    return Beam(c, np.arange(1, n + 1, dtype=np.int64))


# ------------------------------------------------------------------- run ----
def _lattice_with_outputs(text: str, use: str | None):
    """parse_lte, with CSRCSBEND OUTPUT_FILE names collected (the runner writes them)."""
    outputs = {}
    return parse_lte(text, use, outputs=outputs), outputs


def run_ele(path: str, device: int = 0, mode: str = "binary") -> dict:
    """Run a .ele file's tracking job on the engine; returns a summary per
    step (survivors, effort) and the files written."""
    from .aperture import find_aperture_lines, find_aperture_mp
    from .momentum_aperture import local_momentum_acceptance, momentum_aperture
    from .optics import periodic_twiss
    from .sdds import (beam_from_sdds, write_aperture, write_aperture_mp, write_csr_wake, write_losses,
                       write_momentum_aperture, write_phase_space, write_watch)
    from .track import Tracker
    mode_io = mode
    base = os.path.dirname(os.path.abspath(path))
    rootname = os.path.splitext(os.path.basename(path))[0]
    with open(path) as fh:
        cmds = parse_namelists(fh.read())
    rs = rc = bb = tw = sb = None
    summary = {"steps": [], "files": []}
    lattice = None
    csr_outputs = {}

    def name(f):
        if not f:
            return None
        return os.path.join(base, f.replace("%s", rootname))

    for cmd, fields in cmds:
        if cmd == "run_setup":
            rs = _command(fields, {**RUN_SETUP, **{k: None for k in RUN_SETUP_UNSUPPORTED_FILES}}, cmd,
                          {"lattice", "use_beamline", "rootname", "output", "final", "losses", "default_order",
                           "random_number_seed", "p_central", "p_central_mev", "print_statistics"})
            if rs["rootname"]:
                rootname = rs["rootname"]
            with open(os.path.join(base, rs["lattice"])) as fh:
                lattice, csr_outputs = _lattice_with_outputs(fh.read(), rs["use_beamline"])
        elif cmd == "run_control":
            rc = _command(fields, RUN_CONTROL, cmd, {"n_steps", "n_passes", "reset_rf_for_each_step"})
        elif cmd == "twiss_output":
            tw = _command(fields, TWISS_OUTPUT, cmd, {"matched", "filename"})
            if tw["filename"]:
                raise EleError("&twiss_output: filename (a Twiss output file) is not supported by the engine's runner")
        elif cmd == "bunched_beam":
            sb = None
            bb = _command(fields, BUNCHED_BEAM, cmd,
                          {"n_particles_per_bunch", "emit_x", "emit_nx", "beta_x", "alpha_x", "eta_x", "etap_x",
                           "emit_y", "emit_ny", "beta_y", "alpha_y", "eta_y", "etap_y", "sigma_dp", "sigma_s",
                           "dp_s_coupling", "momentum_chirp", "one_random_bunch", "symmetrize",
                           "enforce_rms_values", "distribution_cutoff", "distribution_type", "centroid",
                           "use_twiss_command_values", "save_initial_coordinates"})
        elif cmd == "sdds_beam":
            sb = _command(fields, SDDS_BEAM, cmd, {"input", "input_type", "n_tables_to_skip", "sample_interval",
                                                   "p_lower", "p_upper", "reuse_bunch", "save_initial_coordinates"})
            if not sb["input"]:
                raise EleError("&sdds_beam: no input file given")
            if sb["input_type"] != "elegant":
                raise EleError(f"&sdds_beam: input_type {sb['input_type']!r} is not supported by the engine's runner")
            bb = None
        elif cmd == "track":
            _command(fields, TRACK, cmd, {"soft_failure", "interrupt_file"})
            if rs is None or (bb is None and sb is None):
                raise EleError("&track needs &run_setup and &bunched_beam or &sdds_beam before it")
            rc = rc or dict(RUN_CONTROL)
            p0 = rs["p_central"] or rs["p_central_mev"] / ME_MEV
            twiss = None
            if bb is not None and bb["use_twiss_command_values"]:
                if not tw or not tw["matched"]:
                    raise EleError("use_twiss_command_values needs &twiss_output with matched = 1")
                twiss = periodic_twiss(lattice)
            outs = [f for f in (name(rs["final"]), name(rs["output"])) if f]
            losses = name(rs["losses"])
            watches = [(i, e) for i, e in enumerate(lattice.elements) if e.type == "WATCH" and not e.get("DISABLE")]
            for _, e in watches:
                if not e.strings.get("FILENAME"):
                    raise EleError(f"WATCH {e.name}: no FILENAME")
                if e.get("AUTO_REFERENCE") or e.get("INDEX_OFFSET"):
                    raise EleError(f"WATCH {e.name}: AUTO_REFERENCE and INDEX_OFFSET are not supported by the "
                                   "engine's runner")
            z_end = np.cumsum([e.length for e in lattice.elements])
            for step in range(rc["n_steps"]):
                if bb is None:
                    # one page per step, after n_tables_to_skip; reuse_bunch keeps the first
                    # (sdds_beam.c: new_sdds_beam)
                    page = sb["n_tables_to_skip"] + (0 if sb["reuse_bunch"] else step)
                    try:
                        beam = beam_from_sdds(name(sb["input"]), p0, page=page,
                                              sample_interval=sb["sample_interval"], p_lower=sb["p_lower"],
                                              p_upper=sb["p_upper"])
                    except ValueError as e:
                        raise EleError(f"&sdds_beam: {e}") from e
                elif step == 0 or not bb["one_random_bunch"]:
                    beam = bunched_beam(bb, p0, rs["random_number_seed"] + step, twiss)
                # WATCH records take device memory per recorded pass: the passes
                # run in calls of `chunk` passes that each fit the budget
                n_passes = rc["n_passes"]
                chunk = n_passes
                if watches:
                    per_pass = len(watches) * 7 * 8 * max(beam.n, 1)
                    limit = max(1, WATCH_BUDGET_BYTES // per_pass)
                    chunk = max(d for d in range(1, n_passes + 1) if n_passes % d == 0 and d <= limit)
                with Tracker(lattice, p0, chunk, device=device, default_order=rs["default_order"]) as t:
                    if csr_outputs:
                        t.set_csr_pages(True)
                    records = []
                    if watches:
                        t.set_watch(WATCH_BUDGET_BYTES)
                    if chunk == n_passes:
                        res = t.track(beam)
                        records = t.watch() if watches else []
                    else:
                        t.upload(beam)
                        effort = 0.0
                        for _ in range(n_passes // chunk):
                            effort += t.continue_tracking()
                            records += t.watch()
                        res = t.download()
                        res.effort = effort
                    pages = t.csr_pages() if csr_outputs else []
                summary["steps"].append({"step": step + 1, "survivors": res.n_left, "effort": res.effort})
                charge = next((e.get("TOTAL") for e in lattice.elements if e.type == "CHARGE"), 0.0)
                for f in outs:
                    write_phase_space(f, res, p0, step=step + 1, charge=charge, mode=mode, append=step > 0)
                if losses:
                    write_losses(losses, res, lattice, p0, step=step + 1, mode=mode, append=step > 0)
                macro = charge / beam.n if beam.n else 0.0
                for i, e in watches:
                    write_watch(name(e.strings["FILENAME"]), [r for r in records if r["element"] == i], p0,
                                float(z_end[i]), lattice.total_length, step=step + 1, charge=macro, watch=e.params,
                                mode=mode, append=step > 0, original_particles=beam.n,
                                previous_element=lattice.elements[i - 1].name if i > 0 else None)
                    if step == 0:
                        summary["files"].append(name(e.strings["FILENAME"]))
                for el_name, fname in csr_outputs.items():
                    idx = set(lattice.index(el_name))
                    mine = [p for p in pages if p["element"] in idx]
                    if mine:
                        write_csr_wake(name(fname), mine, mode=mode, append=step > 0)
                        summary["files"].append(name(fname))
            summary["files"] += outs + ([losses] if losses else [])
            summary["result"] = res
        elif cmd == "find_aperture":
            fa = _command(fields, FIND_APERTURE, cmd,
                          {"output", "mode", "xmin", "xmax", "xpmin", "xpmax", "ymin", "ymax", "ypmin", "ypmax", "nx",
                           "ny", "n_splits", "split_fraction", "desired_resolution", "verbosity", "n_lines",
                           "full_plane", "optimization_mode"})
            if rs is None:
                raise EleError("&find_aperture needs &run_setup before it")
            mode, slope, lines = _check_find_aperture(fa)
            rc = rc or dict(RUN_CONTROL)
            p0 = rs["p_central"] or rs["p_central_mev"] / ME_MEV
            out = name(fa["output"]) if not fa["optimization_mode"] else None
            for step in range(rc["n_steps"]):
                if mode == "many-particle":
                    res, effort = find_aperture_mp(lattice, p0, rc["n_passes"], fa["xmin"], fa["xmax"], fa["ymin"],
                                                   fa["ymax"], fa["nx"], fa["ny"], device=device)
                    if out:
                        write_aperture_mp(out, res[0], step=step + 1, mode=mode_io, append=step > 0)
                    summary["steps"].append({"step": step + 1, "boundary": res[0]["boundary"], "effort": effort})
                else:
                    res = find_aperture_lines(lattice, p0, rc["n_passes"], lines=lines, xmax=fa["xmax"],
                                              ymax=fa["ymax"], nx=fa["nx"], n_splits=fa["n_splits"],
                                              split_fraction=fa["split_fraction"], full_plane=bool(fa["full_plane"]),
                                              device=device, slope=slope, xpmax=fa["xpmax"], ypmax=fa["ypmax"])
                    if out:
                        write_aperture(out, res, step=step + 1, mode=mode_io, append=step > 0)
                    summary["steps"].append({"step": step + 1, "area": res["area"], "lines": res["lines"]})
                summary["result"] = res
            if out:
                summary["files"].append(out)
        elif cmd == "momentum_aperture":
            ma = _command(fields, MOMENTUM_APERTURE, cmd, set(MOMENTUM_APERTURE))
            if rs is None:
                raise EleError("&momentum_aperture needs &run_setup before it")
            if ma["output_mode"] not in (0, 1, 2):
                raise EleError("&momentum_aperture: output_mode must be 0, 1 or 2")
            if not ma["output"]:
                raise EleError("&momentum_aperture: no output filename specified")
            rc = rc or dict(RUN_CONTROL)
            p0 = rs["p_central"] or rs["p_central_mev"] / ME_MEV
            out = name(ma["output"])
            kw = {k: ma[k] for k in ("x_initial", "y_initial", "delta_negative_limit", "delta_positive_limit",
                                     "delta_negative_start", "delta_positive_start", "delta_step_size", "splits",
                                     "steps_back", "split_step_divisor", "skip_elements", "process_elements",
                                     "s_start", "s_end", "include_name_pattern", "include_type_pattern")}
            for step in range(rc["n_steps"]):
                try:
                    if ma["output_mode"] == 2:
                        # the grid search of multiparticleLocalMomentumAcceptance (Pelegant's mode):
                        # splits, steps_back, split_step_divisor, fiducialize and soft_failure unused
                        rows, effort = local_momentum_acceptance(
                            lattice, p0, rc["n_passes"], device=device,
                            **{k: v for k, v in kw.items()
                               if k not in ("splits", "steps_back", "split_step_divisor")})
                    else:
                        rows, effort = momentum_aperture(
                            lattice, p0, rc["n_passes"], soft_failure=bool(ma["soft_failure"]),
                            fiducialize=bool(ma["fiducialize"]),
                            forbid_resonance_crossing=bool(ma["forbid_resonance_crossing"]), device=device, **kw)
                except ValueError as e:
                    raise EleError(f"&momentum_aperture: {e}") from e
                write_momentum_aperture(out, rows, step=step + 1, mode=mode_io, output_mode=ma["output_mode"],
                                        append=step > 0)
                summary["steps"].append({"step": step + 1, "rows": rows, "effort": effort})
            summary["files"].append(out)
        elif cmd in INERT:
            continue
        else:
            raise EleError(f"&{cmd} is not a command the engine's runner implements")
    return summary
