"""CPU: the slab decomposition's host logic (ljcell.slab).  The layer split, the cell layer of a
coordinate against the oracle's binning (faces, outside the box, NaN, infinities), and a
multi-process run over gloo (world sizes 2 and 3): each rank takes the particles of its layers,
exchanges one halo layer with each neighbour through exchange_p2p, bins own + halo on the global
grid with the oracle, evaluates its own sorted range with the oracle's FP32 loop and all-reduces
the totals.  Every particle must be evaluated by exactly one rank, with the bits of the
single-domain oracle run, and the pair counts must add up to the single-domain count.  The oracle
stands in here for lj_compute_range, which the GPU tests run."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import ljoracle as O
from ljcell.slab import SlabDomain

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RC = 0.05


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _system(seed=99, n=30_000):
    x, y, z = O.generate_uniform(seed, n)
    # a few particles on the faces of z layers and outside the box, as the binning clamps them
    z[:64] = np.float32(RC) * np.arange(64, dtype=np.float32) % np.float32(1.0)
    z[64:70] = np.array([-0.5, 1.0, 1.5, -0.0, 0.999999, 1e-30], np.float32)
    return x, y, z


def test_layer_split_is_a_partition():
    g = O.grid_from_box((0, 0, 0), (1, 1, 1), RC)
    for world in (1, 2, 3, 7, g.dim[2]):
        doms = [SlabDomain.of(g, r, world) for r in range(world)]
        assert doms[0].z0 == 0 and doms[-1].z1 == g.dim[2]
        for a, b in zip(doms, doms[1:]):
            assert a.z1 == b.z0 and a.z1 > a.z0
    with pytest.raises(ValueError):
        SlabDomain.of(g, 0, g.dim[2] + 1)
    with pytest.raises(ValueError):
        SlabDomain.of(g, 2, 2)


def test_pair_kernel_rule_follows_the_own_layers():
    """With the default tuning a rank picks the pair kernel the library's default would pick for its
    own layers alone: two consecutive targets per lane with x-windows (10) from 2 particles per cell,
    else targets paired inside their cell (12)."""
    from ljcell.slab import PAIR_CELL, pair_kernel_for

    g = O.grid_from_box((0, 0, 0), (1, 1, 1), 0.05)   # 20 x 20 x 20 cells
    d = SlabDomain.of(g, 1, 4)                         # layers [5, 10): 2000 cells
    cells = (d.z1 - d.z0) * d.gx * d.gy
    assert cells == 2000
    assert pair_kernel_for(d, int(PAIR_CELL * cells)) == 10
    assert pair_kernel_for(d, int(PAIR_CELL * cells) - 1) == 12
    assert pair_kernel_for(d, 0) == 12


def test_z_cells_match_the_binning():
    g = O.grid_from_box((-0.25, 0, 0.125), (1, 1, 1.3), 0.07)
    rng = np.random.default_rng(3)
    z = rng.uniform(-0.5, 2.0, 200_000).astype(np.float32)
    faces = (np.float32(0.125) + np.float32(g.width) * np.arange(-2, g.dim[2] + 3, dtype=np.float32))
    z = np.concatenate([z, faces, np.nextafter(faces, np.float32(-np.inf)), np.nextafter(faces, np.float32(np.inf)),
                        np.array([np.nan, np.inf, -np.inf, 0.0, -0.0, 3e38, -3e38], np.float32)])
    x = np.full_like(z, 0.5)
    cz = O.cells_of(g, x, x, z) // (g.dim[0] * g.dim[1])
    dom = SlabDomain.of(g, 0, 1)
    assert np.array_equal(dom.z_cells(torch.from_numpy(z)).numpy(), cz)


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "particle-interaction-with-optix_b200")):
        sys.path.insert(0, p)
    from datetime import timedelta

    import torch.distributed as dist

    import ljoracle as O
    from ljcell.slab import SlabDomain, allreduce_totals, exchange_p2p

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    x, y, z = _system()
    g = O.grid_from_box((0, 0, 0), (1, 1, 1), RC)
    dom = SlabDomain.of(g, rank, world)
    xyz = torch.from_numpy(np.stack([x, y, z], 1))
    zc = dom.z_cells(xyz[:, 2])
    mask = (zc >= dom.z0) & (zc < dom.z1)
    own, own_ids = xyz[mask].contiguous(), torch.nonzero(mask)[:, 0]
    assert torch.equal(own, dom.own(xyz))
    down, up = dom.halo_out(own)
    below, above = exchange_p2p(dom, down, up)
    local = torch.cat([below, own, above]).numpy()
    b = O.bin_particles(g, *(np.ascontiguousarray(local[:, k]) for k in range(3)), O.ORDER_X)
    kb, ke = dom.target_range(torch.from_numpy(b.offsets))
    n = len(local)
    e32, f32 = np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
    sigma = float(np.float32(RC) / np.float32(2.5))
    pairs = O.config_forces_f32_range(g, b, kb, ke, RC, 1.0, sigma, e32, f32, 1)
    local_idx = b.perm[kb:ke] - len(below)
    assert local_idx.min() >= 0 and local_idx.max() < len(own)      # the range holds own particles only
    assert ke - kb == len(own)
    tot = torch.zeros(4, dtype=torch.float64)
    tot[:2] = torch.tensor([0.5 * e32[kb:ke].astype(np.float64).sum(), 0.0])
    tot[2:3].view(torch.int64)[0] = pairs
    red = allreduce_totals(tot)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), ids=own_ids.numpy()[local_idx], e=e32[kb:ke],
             f=f32[kb:ke], pairs=pairs, total_pairs=red["pairs"], energy=red["energy"],
             halo=len(below) + len(above))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_ranks_gloo_match_single_domain(tmp_path, world):
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [dict(np.load(tmp_path / f"rank{r}.npz")) for r in range(world)]
    x, y, z = _system()
    n = len(x)
    g = O.grid_from_box((0, 0, 0), (1, 1, 1), RC)
    b = O.bin_particles(g, x, y, z, O.ORDER_X)
    e32, f32 = np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
    sigma = float(np.float32(RC) / np.float32(2.5))
    pairs = O.config_forces_f32_range(g, b, 0, n, RC, 1.0, sigma, e32, f32, 1)
    e_orig, f_orig = np.empty_like(e32), np.empty_like(f32)
    e_orig[b.perm], f_orig[b.perm] = e32, f32

    ids = np.concatenate([r["ids"] for r in res])
    assert np.array_equal(np.sort(ids), np.arange(n))                  # each particle on exactly one rank
    for r in res:
        assert np.array_equal(r["e"].view(np.uint32), e_orig[r["ids"]].view(np.uint32))
        assert np.array_equal(r["f"].view(np.uint32), f_orig[r["ids"]].view(np.uint32))
        assert int(r["total_pairs"]) == pairs
        assert float(r["energy"]) == pytest.approx(0.5 * e32.astype(np.float64).sum(), rel=1e-12)
    assert sum(int(r["pairs"]) for r in res) == pairs
    assert all(int(r["halo"]) > 0 for r in res)
