"""CSR lattices shared by the CPU oracle pins and the GPU parity tests."""
from elegant_b200 import Element, Lattice, workloads as w


def with_gap(lat: Lattice, gap: float = 0.4) -> Lattice:
    """A plain DRIF between the first dipole and its CSRDRIFT: the CSRDRIFT
    starts behind the point where the dipole's wake was left (the reference
    then re-tracks the gap, csbend.c:3835-3848 in Stupakov mode)."""
    els = []
    for e in lat.elements:
        if e.name == "D1":
            els.append(Element("G1", "DRIF", {"L": gap}))
            e = Element(e.name, e.type, dict(e.params, L=e.params["L"] - gap))
        els.append(e)
    return Lattice(els)


def leading_drift(lat: Lattice) -> Lattice:
    """A CSRDRIFT ahead of the first dipole: on the second pass it follows the
    last dipole of the first, one revolution length back (csbend.c:3251)."""
    d = next(e for e in lat.elements if e.type == "CSRDRIFT")
    els = list(lat.elements)
    els.insert(1, Element("D0", "CSRDRIFT", dict(d.params, L=0.8)))
    return Lattice(els)


def stupakov_cases():
    """name -> lattice, each tracked one pass unless the name ends in '2p'."""
    return {
        "default": w.chicane(bins=200, n_kicks=6, stupakov=True),
        "fine_bins_3kicks": w.chicane(bins=600, n_kicks=8, stupakov=True, drift={"N_KICKS": 3}),
        "dz": w.chicane(bins=300, n_kicks=5, stupakov=True, drift={"DZ": 0.7}),
        "no_sg": w.chicane(bins=120, n_kicks=4, sg_halfwidth=0, stupakov=True, drift={"N_KICKS": 2}),
        "steady_plain": Lattice([Element(e.name, e.type, dict(e.params, **({"STEADY_STATE": 1} if i % 2 else
                                                                         {"TRAPAZOID_INTEGRATION": 0})))
                                 if e.type == "CSRCSBEND" else e
                                 for i, e in enumerate(w.chicane(bins=250, n_kicks=4, stupakov=True).elements)]),
        "gap": with_gap(w.chicane(bins=200, n_kicks=4, stupakov=True, drift={"N_KICKS": 2})),
        "gap_mode0": with_gap(w.chicane(bins=200, n_kicks=4, drift={"N_KICKS": 2})),
        "ring_2p": leading_drift(w.chicane(bins=200, n_kicks=4, stupakov=True, drift={"N_KICKS": 2})),
        "ring_mode0_2p": leading_drift(w.chicane(bins=200, n_kicks=4, drift={"N_KICKS": 2})),
    }


def _filtered(lat: Lattice, **kw) -> Lattice:
    return Lattice([Element(e.name, e.type, dict(e.params, **kw)) if e.type == "CSRCSBEND" else e
                    for e in lat.elements])


def filter_cases():
    """CSRCSBEND histogram filters (LOW/HIGH_FREQUENCY_CUTOFF0/1,
    CLIP_NEGATIVE_BINS): name -> lattice."""
    return {
        "low_pass": _filtered(w.chicane(bins=200, n_kicks=4), HIGH_FREQUENCY_CUTOFF0=0.2, HIGH_FREQUENCY_CUTOFF1=0.4),
        "high_pass": _filtered(w.chicane(bins=200, n_kicks=4), LOW_FREQUENCY_CUTOFF0=0.01, LOW_FREQUENCY_CUTOFF1=0.03),
        "both_odd_bins": _filtered(w.chicane(bins=151, n_kicks=4), LOW_FREQUENCY_CUTOFF0=0.02,
                                   HIGH_FREQUENCY_CUTOFF0=0.3, HIGH_FREQUENCY_CUTOFF1=0.5),
        "round_trip_only": _filtered(w.chicane(bins=120, n_kicks=3), LOW_FREQUENCY_CUTOFF0=0.0),
        "no_clip_stupakov": _filtered(w.chicane(bins=200, n_kicks=4, stupakov=True), HIGH_FREQUENCY_CUTOFF0=0.1,
                                      CLIP_NEGATIVE_BINS=0),
    }
