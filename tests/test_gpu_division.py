"""Division by a stored reciprocal (Markstein's correction step), used for
the CSBEND kick's X/rho0 and /rho_actual: bit-identical to IEEE division for
the lattices' divisors, random ones, ones near 1 and binade-edge ones, on
random numerators over 80 binades."""
import ctypes

import numpy as np
import pytest

from elegant_b200 import _native as nat
from elegant_b200 import workloads as w

pytestmark = pytest.mark.gpu


def test_division_by_reciprocal_is_correctly_rounded():
    lib = nat.load_library()
    f = lib.b2e_selftest_division
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64)]
    divisors = []
    for lat in (w.fodo_ring(), w.chicane()):
        for e in lat.elements:
            if e.type in ("CSBEND", "CSRCSBEND"):
                rho0 = e.params["L"] / abs(e.params["ANGLE"])
                divisors += [rho0, rho0 / (1 + e.params.get("FSE", 0.0))]
    rng = np.random.default_rng(5)
    divisors += list(10 ** rng.uniform(-1, 3, 2000)) + list(rng.uniform(1, 2, 500)) + [3.0, 7.0, 10.0]
    # divisors near 1 and significands at the ends of the binade (all ones,
    # one ulp above a power of two)
    divisors += list(1 + rng.uniform(-0.1, 0.1, 1000)) + [1 + 2.0 ** -52, 1 - 2.0 ** -53, 2 - 2.0 ** -52,
                                                         -(2 - 2.0 ** -52), 0.75 - 2.0 ** -54, 1.5 + 2.0 ** -52]
    b = np.ascontiguousarray(divisors, dtype=np.float64)
    bad = ctypes.c_int64(-1)
    assert f(b.ctypes.data, len(b), 200_000, 12345, ctypes.byref(bad)) == 0
    assert bad.value == 0
