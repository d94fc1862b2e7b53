"""GPU parity against the REFERENCE's own kernels (cudaLJ.cu built from source
into oracle/_ref/libljref.so) on the same injected positions: counts, offsets
and cell descriptors bit-exact, per-cell particle sets equal (the reference's
within-cell order is not deterministic), candidate count exact, compat
energies within the reference's own 1e-5 relative tolerance
(CheckEqualCpu, cudaLJ.cu:419-423)."""
import os
import sys

import numpy as np
import pytest

import ljoracle as O

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import refcases  # noqa: E402

pytestmark = pytest.mark.gpu


def np_(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def ref_available():
    if not O.ref_available():
        pytest.fail("oracle/_ref/libljref.so missing: build it with `make -C oracle ref` where the reference "
                    "sources are mounted")
    return True


@pytest.mark.parametrize("name", sorted(refcases.CASES))
def test_against_reference_kernels(torch_cuda, ctx, ref_available, name):
    import ljcell

    torch = torch_cuda
    (x, y, z), box, cutoff = refcases.CASES[name]()
    r = O.ref_run(x, y, z, box, cutoff)
    g = ljcell.grid_compat(box, cutoff)
    d = [torch.from_numpy(a).cuda() for a in (x, y, z)]
    b = ctx.bin(g, *d, order=ljcell.ORDER_INDEX, soa=True, cells=True)
    v = ctx.compute_compat(g, b)
    cand = ctx.count_candidates(g, b.offsets)
    ctx.sync()
    n = len(x)
    np.testing.assert_array_equal(np_(b.counts), r.counts)
    np.testing.assert_array_equal(np_(b.offsets), r.prefix)
    np.testing.assert_array_equal(np_(b.cells), r.cells)
    perm = np_(b.index)[:n]
    np.testing.assert_array_equal(perm, refcases.sorted_within_cells(r.index, r.prefix))
    assert int(np_(cand)[0]) == r.nbinter
    ref_v = np.empty(n, np.float32)
    ref_v[r.index] = r.v
    ours = np.empty(n, np.float32)
    ours[perm] = np_(v)[:n]
    rel = np.abs(ours - ref_v) / np.where(ref_v == 0, 1, np.abs(ref_v))
    assert rel.max() <= 1e-5, rel.max()
    # the oracle agrees with the reference too
    og = O.grid_from_box((0, 0, 0), (box,) * 3, cutoff)
    ob = O.bin_particles(og, x, y, z, O.ORDER_INDEX)
    ov = np.empty(n, np.float32)
    ov[ob.perm] = O.compat_energy(og, ob)
    assert (np.abs(ov - ref_v) / np.where(ref_v == 0, 1, np.abs(ref_v))).max() <= 1e-5


def test_reference_harness_refuses_out_of_box(ref_available):
    x = np.array([0.5, 1.0], np.float32)   # 1.0 / 0.25 = 4 = grid dim: the reference would index past its arrays
    with pytest.raises(RuntimeError):
        O.ref_run(x, x.copy(), x.copy(), 1.0, 0.25)
