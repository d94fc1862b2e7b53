"""The standalone spatial sort (lj_reorder), the reference's reorder()
(SDK/optixMultiSphereAABB/sort.cu:7-41): keys, stored .w and the sorted
order, bit-exact against the oracle's restatement on seeded inputs and the
edge cases of its arithmetic (points on cell faces, at 1.0, one crowded cell
above the per-record rank limit, keys above 2^24 that round as floats)."""
import numpy as np
import pytest

import ljoracle as O


def _points(n, seed=1234):
    x, y, z = O.generate_uniform(seed, n)
    return np.stack([x, y, z, np.zeros(n, np.float32)], axis=1)


def test_oracle_reorder_small_by_hand():
    # radius 0.5: width 2; keys x + 2y + 4z
    p = np.array([[0.9, 0.9, 0.9, 0], [0.1, 0.1, 0.1, 0], [0.6, 0.1, 0.1, 0], [0.2, 0.1, 0.2, 0]], np.float32)
    out = O.reorder(p, 0.5)
    assert out[:, 3].tolist() == [0.0, 0.0, 1.0, 7.0]
    # equal keys keep input order
    assert out[0, 0] == np.float32(0.1) and out[1, 0] == np.float32(0.2)


def test_oracle_reorder_is_a_permutation_sorted_by_key():
    p = _points(20_000)
    out = O.reorder(p, 0.05)
    assert np.all(np.diff(out[:, 3]) >= 0)
    a = np.sort(p[:, :3].view(np.void), axis=0)
    b = np.sort(out[:, :3].copy().view(np.void), axis=0)
    assert np.array_equal(a, b)


def test_oracle_reorder_float_keys_round_like_the_reference():
    # width 400: ids up to 6.4e7 > 2^24, so distinct ids can share one float .w
    r = np.float32(1.0) / np.float32(400.0)
    p = np.array([[0.999, 0.999, 0.999, 0], [0.9965, 0.999, 0.999, 0], [0.5, 0.5, 0.5, 0]], np.float32)
    out = O.reorder(p, float(r))
    ids = (np.trunc(p[:, :3] / r).astype(np.int64) * np.array([1, 400, 160000])).sum(1)
    assert sorted(out[:, 3].tolist()) == sorted(ids.astype(np.float32).tolist())


def _away_from_faces(p, radius, ulps=8):
    """Rows whose coordinates all lie further than `ulps` float steps of the quotient from a cell
    face: there the reference build's fast division and the oracle's IEEE division truncate alike."""
    q = p[:, :3].astype(np.float64) / np.float64(np.float32(radius))
    gap = np.abs(q - np.round(q))
    step = np.spacing(np.maximum(np.abs(q), 1.0).astype(np.float32)).astype(np.float64)
    return p[np.all(gap > ulps * step, axis=1)]


def _near_faces(n, radius, seed):
    """Points on and within one float step of cell faces (random cells and axes), in [0, 1)."""
    rng = np.random.default_rng(seed)
    r = np.float32(radius)
    width = int(np.float32(1.0) / r)
    b = (rng.integers(0, width, (n, 3)).astype(np.float32) * r).astype(np.float32)
    step = rng.integers(-1, 2, (n, 3))
    b = np.where(step > 0, np.nextafter(b, np.float32(2)), np.where(step < 0, np.nextafter(b, np.float32(-1)), b))
    b = np.clip(b, 0, np.nextafter(np.float32(1), np.float32(0))).astype(np.float32)
    return np.concatenate([b, np.zeros((n, 1), np.float32)], axis=1)


def _same_as_reference(got, ref):
    """Sorted keys equal bit for bit, and every key holds the same points (the reference's
    thrust::sort leaves the order within a key open)."""
    assert np.array_equal(got[:, 3].view(np.uint32), ref[:, 3].view(np.uint32))
    ka = np.lexsort((got[:, 2], got[:, 1], got[:, 0], got[:, 3]))
    kb = np.lexsort((ref[:, 2], ref[:, 1], ref[:, 0], ref[:, 3]))
    assert np.array_equal(got[ka].view(np.uint32), ref[kb].view(np.uint32))


@pytest.fixture
def sortref():
    if not O.sortref_available():
        pytest.skip("reference sort.cu not built (make -C oracle sortref, needs the reference sources)")


@pytest.mark.gpu
@pytest.mark.parametrize("n,radius", [(1, 0.1), (1000, 0.25), (100_000, 0.05), (1_000_000, 0.01),
                                      (300_000, 1.0 / 300.0), (50_000, 1.0 / 500.0), (200_000, 1.0 / 450.0),
                                      (200_000, 1.0 / 511.0)])
def test_gpu_reorder_matches_oracle(torch_cuda, ctx, n, radius):
    """Bit-exact against the oracle's restatement on points away from the cell faces."""
    torch = torch_cuda
    p = _away_from_faces(_points(n, seed=n), radius)
    d = torch.from_numpy(p.copy()).cuda()
    ctx.reorder(d, radius)
    ctx.sync()
    ref = O.reorder(p, radius)
    assert np.array_equal(d.cpu().numpy().view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("radius", [0.1, 0.05, 0.01, 1.0 / 300.0, 1.0 / 450.0, 1.0 / 500.0, 1.0 / 511.0,
                                    1.0 / 512.0])
def test_gpu_reorder_matches_reference(torch_cuda, ctx, sortref, radius):
    """Against the reference's own sort.cu, built from source with its own flags (--use_fast_math),
    on random points and on points on and next to cell faces, where the division matters."""
    torch = torch_cuda
    p = np.concatenate([_points(200_000, seed=11), _near_faces(200_000, radius, seed=12)])
    d = torch.from_numpy(p.copy()).cuda()
    ctx.reorder(d, radius)
    ctx.sync()
    got = d.cpu().numpy()
    assert np.array_equal(np.sort(O.sortref_keys(p, radius)).view(np.uint32), got[:, 3].view(np.uint32))
    _same_as_reference(got, O.sortref_reorder(p, radius))


@pytest.mark.gpu
def test_gpu_reorder_key_above_2_24_as_the_reference(torch_cuda, ctx, sortref):
    """Width 511, cell (1, 0, 65): the exact id 16,972,866 is a float, and the reference built from
    source stores it too (its compiler contracts the float key sum into fused multiply-adds, which
    round once, as the integer id stored in .w does)."""
    torch = torch_cuda
    r = np.float32(1.0 / 511.0)
    p = np.array([[1.5 * r, 0.25 * r, 65.5 * r, 0], [0.5, 0.5, 0.5, 0]], np.float32)
    assert int(O.sortref_keys(p, float(r))[0]) == 16_972_866
    d = torch.from_numpy(p.copy()).cuda()
    ctx.reorder(d, float(r))
    ctx.sync()
    assert 16_972_866.0 in d.cpu().numpy()[:, 3].tolist()


@pytest.mark.gpu
def test_gpu_reorder_edges(torch_cuda, ctx, sortref):
    """A crowded cell (above the per-record rank limit: the large-cell path), points on faces, at
    1.0 and at 0.0, against the reference's own sort.cu."""
    torch = torch_cuda
    rng = np.random.default_rng(7)
    n = 5000
    p = np.zeros((n, 4), np.float32)
    p[:3000, :3] = rng.uniform(0.30, 0.34, (3000, 3)).astype(np.float32)
    p[3000:4000, :3] = (rng.integers(0, 11, (1000, 3)) / np.float32(10.0)).astype(np.float32)
    p[4000:4500, :3] = 1.0
    p[4500:, :3] = rng.uniform(0, 1, (500, 3)).astype(np.float32)
    d = torch.from_numpy(p.copy()).cuda()
    ctx.reorder(d, 0.1)
    ctx.sync()
    got = d.cpu().numpy()
    _same_as_reference(got, O.sortref_reorder(p, 0.1))
    # points of one key keep their input order (checked on the points that occur once)
    rows = [tuple(v) for v in p[:, :3].view(np.uint32)]
    first = {}
    for i, t in enumerate(rows):
        first[t] = -1 if t in first else i
    src = np.array([first[tuple(v)] for v in got[:, :3].view(np.uint32)])
    for key in np.unique(got[:, 3]):
        idx = src[(got[:, 3] == key) & (src >= 0)]
        assert np.all(np.diff(idx) > 0), key


@pytest.mark.gpu
def test_gpu_reorder_out_of_domain_is_reported(torch_cuda, ctx):
    import ljcell

    torch = torch_cuda
    p = _points(1000)
    p[10, :3] = 50.0   # key 555,500, beyond the 1,111 keys of the [0, 1] domain at radius 0.1
    d = torch.from_numpy(p).cuda()
    with pytest.raises(ljcell.LJError):
        ctx.reorder(d, 0.1)
        ctx.sync()
    ctx.sync()  # the status word was cleared by the failing sync


def test_reorder_rejects_bad_arguments():
    import ljcell

    lib = ljcell.lib()
    assert lib.lj_reorder(None, 10, None, 0.1) == 1  # LJ_EINVAL
