"""The NAFF method of elegant_b200/csrc/b2e_naff.cu in numpy (test
infrastructure): Hann window on the mean-removed signal, the largest grid
line k/N, then 60 bisections on the sign of d|F|^2/dnu on [(k-1)/N,
(k+1)/N] within [0, 1/2]; amplitude 2|F|/N, phase arg F."""
import math

import numpy as np


def naff(x):
    x = np.asarray(x, dtype=np.float64)
    n = x.size
    t = np.arange(n)
    y = (x - x.mean()) * (1 - np.cos(2 * np.pi * t / n))
    spec = np.abs(np.fft.fft(y)[1:n // 2 + 1]) ** 2
    k = int(np.argmax(spec)) + 1

    def sums(nu):
        e = np.exp(-2j * np.pi * nu * t)
        f = np.sum(y * e)
        df = np.sum(y * (-2j * np.pi * t) * e)
        return f, 2 * (f.real * df.real + f.imag * df.imag)
    a, b = max((k - 1) / n, 0.0), min((k + 1) / n, 0.5)
    for _ in range(60):
        m = 0.5 * (a + b)
        if sums(m)[1] > 0:
            a = m
        else:
            b = m
    nu = 0.5 * (a + b)
    f = sums(nu)[0]
    return nu, 2 * abs(f) / n, math.atan2(f.imag, f.real)


def adjust_tune_half_plane(frequency, phase0, phase1):
    """adjustTuneHalfPlane (twiss.cc:4036-4046)."""
    if abs(phase0 - phase1) > math.pi:
        if phase0 < phase1:
            phase0 += 2 * math.pi
        else:
            phase1 += 2 * math.pi
    return frequency if phase0 < phase1 else 1 - frequency
