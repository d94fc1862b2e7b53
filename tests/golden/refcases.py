"""Inputs shared by the reference-kernel parity test (GPU) and the golden
fixtures it records.  Positions come from the oracle's drand48 generator and
are kept inside the box the reference kernels can index (they do not clamp:
cudaLJ.cu:130-132 asserts, and release builds compile the asserts out)."""
import math

import numpy as np

import ljoracle as O


def _below(v, box):
    return np.minimum(v, np.nextafter(np.float32(box), np.float32(0))).astype(np.float32)


def uniform_case(seed, box_div, per_cell):
    """The reference's uniform sweep point (cudaLJ.cu:748-762): box 1,
    cell width 1 / box_div, N = box_div^3 * per_cell."""
    n = box_div ** 3 * per_cell
    cutoff = float(np.float32(1.0) / np.float32(box_div))
    x, y, z = O.generate_uniform(seed, n)
    return (_below(x, 1.0), _below(y, 1.0), _below(z, 1.0)), 1.0, cutoff


def surface_case(seed, box_div, per_cell):
    """The reference's surface sweep point (cudaLJ.cu:716-739): unit sphere
    centred at (1, 1, 1), coordinates capped at 2 - 1e-6 as InitParticlesSphere
    does (cudaLJ.cu:210-214), cell width from the expected neighbour count."""
    nb_boxes = box_div ** 3
    n = nb_boxes * per_cell
    ppc = n / nb_boxes
    coef = 1.0 - (2 * 9 * ppc) / n
    radius = math.acos(min(1.0, max(-1.0, coef)))
    box = np.float32(math.ceil(2.0 / radius) * radius)
    grid_dim = int(float(box) / radius)
    cell = np.float32(box / np.float32(grid_dim))
    x, y, z = O.generate_sphere(seed, n, (1.0, 1.0, 1.0), 1.0)
    cap = np.float32(2 - 1e-6)
    return tuple(np.minimum(np.maximum(a, np.float32(0)), cap).astype(np.float32) for a in (x, y, z)), float(box), \
        float(cell)


CASES = {
    "uniform_div8_ppc8": lambda: uniform_case(1234, 8, 8),
    "uniform_div16_ppc4": lambda: uniform_case(42, 16, 4),
    "uniform_div4_ppc32": lambda: uniform_case(7, 4, 32),
    "surface_div8_ppc8": lambda: surface_case(1234, 8, 8),
}


def sorted_within_cells(index, prefix):
    """The reference's per-cell index sets in canonical (ascending) order."""
    out = index.copy()
    for c in range(len(prefix) - 1):
        a, b = prefix[c], prefix[c + 1]
        if b - a > 1:
            out[a:b] = np.sort(out[a:b])
    return out
