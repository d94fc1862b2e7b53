"""GPU: the slab decomposition (ljcell.slab) with its ranks emulated one after another in one
process on one GPU; the halo exchange hands each emulated rank the boundary layers of its
neighbours in memory.  Each rank bins its own particles plus the two halo layers on the global
grid and evaluates only its own sorted range through lj_compute_range.  Against the single-domain
lj_compute of the same system with the same pair kernel: every particle is evaluated by exactly
one rank, its energy and force carry the same bits, the pair counts add up exactly and the summed
FP64 totals agree to 1e-12.  Sizes: 100k uniform at rc = 0.05 (20 layers) over 2, 3 and 5 ranks
with each pair kernel; a system filling only the lower half of the box (ranks with no particles
and empty halos); and the 10M uniform workload at rc = 0.01 over 2, 4 and 8 ranks."""
import numpy as np
import pytest

import ljoracle as O
from test_gpu_parity import dev

pytestmark = pytest.mark.gpu


def single_domain(ctx, g, p, xyz):
    import torch

    b = ctx.bin(g, xyz[:, 0].contiguous(), xyz[:, 1].contiguous(), xyz[:, 2].contiguous(), order=1)
    e, f, t = ctx.compute(g, p, b)
    ids = b.xyzi[:, 3].contiguous().view(torch.int32).long()
    n = xyz.shape[0]
    eo = torch.empty(n, dtype=torch.float32, device=xyz.device)
    fo = torch.empty((n, 3), dtype=torch.float32, device=xyz.device)
    eo[ids], fo[ids] = e[:n], f[:n]
    return eo, fo, t


def emulated_ranks(ctx, g, p, xyz, world):
    """Runs the W ranks of the decomposition in turn; returns per-original-index energy and force,
    how many ranks evaluated each particle, the list of per-rank totals and halo sizes."""
    import torch

    import ljcell
    from ljcell import slab

    doms = [slab.SlabDomain.of(g, r, world) for r in range(world)]
    masks = []
    for d in doms:
        zc = d.z_cells(xyz[:, 2])
        masks.append((zc >= d.z0) & (zc < d.z1))
    owns = [xyz[m].contiguous() for m in masks]
    own_ids = [torch.nonzero(m)[:, 0] for m in masks]
    halos = [d.halo_out(o) for d, o in zip(doms, owns)]
    empty = xyz[:0]
    n = xyz.shape[0]
    eo = torch.full((n,), float("nan"), dtype=torch.float32, device=xyz.device)
    fo = torch.full((n, 3), float("nan"), dtype=torch.float32, device=xyz.device)
    seen = torch.zeros(n, dtype=torch.int32, device=xyz.device)
    totals, halo_sizes = [], []
    for r, d in enumerate(doms):
        below = halos[r - 1][1] if r > 0 else empty
        above = halos[r + 1][0] if r < world - 1 else empty
        res = slab.step(ctx, g, p, d, owns[r], exchange=lambda dom, down, up, a=below, b=above: (a, b))
        local = res.binned.xyzi[res.kb:res.ke, 3].contiguous().view(torch.int32).long() - below.shape[0]
        assert res.ke - res.kb == owns[r].shape[0]
        assert (res.kb, res.ke) == d.target_range(res.binned.offsets)
        if res.ke > res.kb:
            assert int(local.min()) >= 0 and int(local.max()) < owns[r].shape[0]
        gid = own_ids[r][local]
        eo[gid] = res.energy[res.kb:res.ke]
        fo[gid] = res.force[res.kb:res.ke]
        seen[gid] += 1
        totals.append(ljcell.totals_from_tensor(res.totals))
        halo_sizes.append(res.halo)
    return eo, fo, seen, totals, halo_sizes


def check(ctx, g, p, xyz, world):
    import torch

    import ljcell

    e1, f1, t1 = single_domain(ctx, g, p, xyz)
    eo, fo, seen, totals, halo = emulated_ranks(ctx, g, p, xyz, world)
    ctx.sync()
    t1 = ljcell.totals_from_tensor(t1)
    assert bool((seen == 1).all())
    assert torch.equal(eo.view(torch.int32), e1.view(torch.int32))
    assert torch.equal(fo.view(torch.int32), f1.view(torch.int32))
    assert sum(t["pairs"] for t in totals) == t1["pairs"]
    for key in ("energy", "virial"):
        s = sum(t[key] for t in totals)
        assert abs(s - t1[key]) <= 1e-12 * abs(t1[key]) + 1e-300, (key, s, t1[key])
    return halo


@pytest.mark.parametrize("kernel", [0, 1, 6, 10, 12])
@pytest.mark.parametrize("world", [2, 3, 5])
def test_slab_ranks_match_single_domain(torch_cuda, ctx, world, kernel):
    import ljcell

    torch = torch_cuda
    x, y, z = O.generate_uniform(4321, 100_000)
    rc = 0.05
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    p = ljcell.params(rc)
    xyz = torch.stack([dev(torch, x), dev(torch, y), dev(torch, z)], 1).contiguous()
    ctx.set_tuning(kernel)
    try:
        halo = check(ctx, g, p, xyz, world)
    finally:
        ctx.set_tuning(0)
    assert all(h > 0 for h in halo)


def test_slab_ranks_with_empty_slabs(torch_cuda, ctx):
    """Particles only in z < 0.5 over 4 ranks of 20 layers: the upper ranks own nothing, and the
    top rank receives an empty halo."""
    import ljcell

    torch = torch_cuda
    x, y, z = O.generate_uniform(77, 50_000)
    z = (z * np.float32(0.5)).astype(np.float32)
    rc = 0.05
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    p = ljcell.params(rc)
    xyz = torch.stack([dev(torch, x), dev(torch, y), dev(torch, z)], 1).contiguous()
    halo = check(ctx, g, p, xyz, 4)
    assert halo[-1] == 0


@pytest.mark.parametrize("world", [2, 4, 8])
def test_slab_ranks_uniform_10M(torch_cuda, ctx, world):
    """The 10M uniform workload at rc = 0.01 (100 layers) split over 2, 4 and 8 ranks."""
    import ljcell

    torch = torch_cuda
    x, y, z = O.generate_uniform(1234, 10_000_000)
    rc = 0.01
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    p = ljcell.params(rc)
    xyz = torch.stack([dev(torch, x), dev(torch, y), dev(torch, z)], 1).contiguous()
    halo = check(ctx, g, p, xyz, world)
    # one-cell halo layers: about 2 (or 1 at the ends) of the 100 layers' particles per rank
    for r, h in enumerate(halo):
        layers = 1 if r in (0, world - 1) else 2
        assert abs(h - layers * 100_000) < 5_000, (r, h)
    del xyz
    torch.cuda.empty_cache()


@pytest.mark.parametrize("n", [0, 1, 1023, 1024, 1025, 100_000])
def test_select_layers_matches_host_selection(torch_cuda, ctx, n):
    """lj_select_layers returns the particles of two z layers in input order, as the host-side
    selection (SlabDomain.halo_out) does: same rows, same order, bit for bit; faces, points outside
    the box and a non-finite z included; a negative layer selects nothing; both layers may be one."""
    import ljcell
    from ljcell import slab

    torch = torch_cuda
    rng = np.random.default_rng(n + 7)
    xyz = rng.uniform(-0.1, 1.1, (n, 3)).astype(np.float32)
    if n >= 8:
        xyz[:4, 2] = np.float32(0.05) * np.arange(4, dtype=np.float32)   # on the layer faces
        xyz[4, 2] = np.nan
        xyz[5, 2] = np.inf
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), 0.05)
    t = torch.from_numpy(xyz).to("cuda")
    for world, rank in ((4, 1), (4, 0), (4, 3), (20, 7)):
        dom = slab.SlabDomain.of(g, rank, world)
        down, up = dom.halo_out(t)
        lo = dom.z0 if rank > 0 else -1
        hi = dom.z1 - 1 if rank < world - 1 else -1
        got_lo, got_hi = ctx.select_layers(g, t, lo, hi)
        assert torch.equal(got_lo.view(torch.int32), down.view(torch.int32))
        assert torch.equal(got_hi.view(torch.int32), up.view(torch.int32))
    zc = slab.SlabDomain.of(g, 0, 1).z_cells(t[:, 2])
    for layer in (0, 5, 19):
        a, b = ctx.select_layers(g, t, layer, layer)
        want = t[zc == layer].view(torch.int32)
        assert torch.equal(a.view(torch.int32), want) and torch.equal(b.view(torch.int32), want)
