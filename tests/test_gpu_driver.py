"""GPU: the C++ host driver (ljcell_driver, over the C ABI) runs the
reference's sweep and writes the reference's CSV columns (cudaLJ.cu:779-788);
its NbInteractions equal the oracle's candidate counts for the same seeded
positions."""
import csv
import os
import subprocess

import numpy as np
import pytest

import ljoracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "particle-interaction-with-optix_b200", "ljcell", "ljcell_driver")
COLUMNS = ["NbParticles", "NbInteractions", "NbLoops", "boxDiv", "nbCells", "partspercell",
           "interactionsperparticle", "timeinit", "timecompute", "timetotal"]


def test_driver_uniform_sweep(tmp_path, torch_cuda):
    assert os.path.exists(DRIVER), "ljcell_driver not built"
    out = tmp_path / "results.csv"
    r = subprocess.run([DRIVER, "--max-box-div", "4", "--loops", "2", "--out", str(out)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    rows = list(csv.reader(open(out)))
    assert rows[0] == COLUMNS
    seen = {}
    for row in rows[1:]:
        n, nb, loops, div = int(row[0]), int(row[1]), int(row[2]), int(row[3])
        seen[(n, div)] = nb
        assert loops == 2 and float(row[9]) > 0
    assert len(seen) == 6 + 6   # boxDiv 2 and 4, N = boxDiv^3 .. 32 boxDiv^3
    for (n, div), nb in seen.items():
        w = float(np.float32(1.0) / np.float32(div))
        g = O.grid_from_box((0, 0, 0), (1, 1, 1), w)
        expect = 0
        for loop in range(2):
            x, y, z = O.generate_uniform(1234 + loop, n)
            expect += O.count_candidates(g, O.bin_particles(g, x, y, z, O.ORDER_INDEX).offsets)
        assert nb == expect, (n, div)


def test_driver_surface_sweep(tmp_path, torch_cuda):
    out = tmp_path / "results-surface.csv"
    r = subprocess.run([DRIVER, "-gs", "--max-box-div", "4", "--loops", "1", "--out", str(out)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    rows = list(csv.reader(open(out)))
    assert rows[0] == COLUMNS and len(rows) > 1
