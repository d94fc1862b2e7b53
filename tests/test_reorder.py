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


@pytest.mark.gpu
@pytest.mark.parametrize("n,radius", [(1, 0.1), (1000, 0.25), (100_000, 0.05), (1_000_000, 0.01),
                                      (300_000, 1.0 / 300.0), (50_000, 1.0 / 500.0)])
def test_gpu_reorder_matches_oracle(torch_cuda, ctx, n, radius):
    torch = torch_cuda
    p = _points(n, seed=n)
    d = torch.from_numpy(p.copy()).cuda()
    ctx.reorder(d, radius)
    ctx.sync()
    ref = O.reorder(p, radius)
    assert np.array_equal(d.cpu().numpy().view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_gpu_reorder_edges(torch_cuda, ctx):
    torch = torch_cuda
    rng = np.random.default_rng(7)
    n = 5000
    p = np.zeros((n, 4), np.float32)
    # crowded cell (above the per-record rank limit, sorted by the large-cell path), faces, 1.0, 0.0
    p[:3000, :3] = rng.uniform(0.30, 0.34, (3000, 3)).astype(np.float32)
    p[3000:4000, :3] = (rng.integers(0, 11, (1000, 3)) / np.float32(10.0)).astype(np.float32)
    p[4000:4500, :3] = 1.0
    p[4500:, :3] = rng.uniform(0, 1, (500, 3)).astype(np.float32)
    d = torch.from_numpy(p.copy()).cuda()
    ctx.reorder(d, 0.1)
    ctx.sync()
    ref = O.reorder(p, 0.1)
    assert np.array_equal(d.cpu().numpy().view(np.uint32), ref.view(np.uint32))


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
