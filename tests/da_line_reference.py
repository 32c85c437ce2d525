"""elegant's line-mode aperture search (aperture_search.c:910-1240) restated
one particle per run on a CPU oracle (test infrastructure): the check for
elegant_b200.aperture.find_aperture_lines.  Use a lattice without RF: the
reference keeps the phase reference of its first tracked particle for the
whole search, which per-particle oracle runs cannot reproduce."""
import numpy as np

from elegant_b200.aperture import line_factors


def serial_line_search(oracle, lattice, p_central, n_passes, lines=11, xmax=0.1, ymax=0.1, nx=21, n_splits=0,
                       split_fraction=0.5, full_plane=False, slope=False, xpmax=0.0, ypmax=0.0):
    """slope=True: the lines in (x', y') up to (xpmax, ypmax) (aperture_search.c:1029-1035, :1070-1076)."""
    fx, fy = line_factors(lines, full_plane)
    if slope:
        xmax, ymax = xpmax, ypmax
    cx, cy = (1, 3) if slope else (0, 2)
    origin_stable = False
    out = []
    for line in range(lines):
        xs, ys = (-1.0, -1.0) if fx[line] > 0 else (1.0, -1.0)
        lost_pass = -1
        dx = dy = 0.0
        for split in range(n_splits + 1):
            if split == 0:
                dx = xmax / (nx - 1) * fx[line]
                dy = ymax / (nx - 1) * fy[line]
                x0 = y0 = 0.0
                steps = nx
            else:
                x0, y0 = xs, ys
                dx *= split_fraction
                dy *= split_fraction
                x0 += dx
                y0 += dy
                steps = max(int(1 / split_fraction - 0.5), 1)
            for index in range(steps):
                if index != 0 or split != 0 or not origin_stable:
                    c = np.zeros((1, 6))
                    c[0, cx] = index * dx + x0
                    c[0, cy] = index * dy + y0
                    rows, n_left, _ = oracle.track(lattice, c, np.array([1]), p_central, n_passes)[:3]
                    if n_left == 0:
                        lost_pass = int(rows[0, 7])
                        break
                if index == 0 and split == 0:
                    origin_stable = True
                xv, yv = x0 + index * dx, y0 + index * dy
                if fx[line]:
                    if (fx[line] > 0 and xs < xv) or (fx[line] < 0 and xs > xv):
                        xs, ys = xv, yv
                elif ys < yv:
                    xs, ys = xv, yv
        out.append((xs, ys, lost_pass))
    return out, origin_stable
