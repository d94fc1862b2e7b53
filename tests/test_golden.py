"""CPU: the oracle against golden fixtures recorded from the REFERENCE's own
kernels (cudaLJ.cu built from source, run on a B200 by
tests/golden/make_golden.py).  Pins the oracle's binning (counts, offsets,
per-cell particle sets), its candidate count and its compat energies to the
reference's actual outputs."""
import glob
import os

import numpy as np
import pytest

import ljoracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_*.npz")))


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 4, "golden fixtures missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[4:-4] for p in GOLDEN])
def test_oracle_matches_reference_outputs(path):
    d = np.load(path)
    x, y, z = d["x"], d["y"], d["z"]
    box, cutoff = float(d["box"]), float(d["cutoff"])
    g = O.grid_from_box((0, 0, 0), (box,) * 3, cutoff)
    b = O.bin_particles(g, x, y, z, O.ORDER_INDEX)
    np.testing.assert_array_equal(b.counts, d["counts"])
    np.testing.assert_array_equal(b.offsets, d["prefix"])
    np.testing.assert_array_equal(b.perm, d["index_sorted"])
    assert O.count_candidates(g, b.offsets) == int(d["nbinter"])
    v = np.empty(len(x), np.float32)
    v[b.perm] = O.compat_energy(g, b)
    ref = d["v_by_index"]
    rel = np.abs(v - ref) / np.where(ref == 0, 1, np.abs(ref))
    assert rel.max() <= 1e-5, rel.max()
