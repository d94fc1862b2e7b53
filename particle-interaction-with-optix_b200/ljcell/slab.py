"""Spatial decomposition of one system over several GPUs: slabs of z layers with a one-cell halo.

The reference runs one system on one GPU (cudaLJ.cu has no exchange step).  Here rank r of W owns
the z layers [z0, z1) of the global cell grid, a balanced split, and the particles whose cell lies
in them.  One step on a rank:

  1. the particles of its first own layer go to rank r - 1 and those of its last own layer to
     rank r + 1 (point-to-point, counts then coordinates);
  2. it bins its own particles together with the two received halo layers on the GLOBAL grid
     (same origin, width and dims on every rank, so every particle lands in the cell the
     single-GPU binning gives it and the 27-cell stencils are the same);
  3. its own particles are one contiguous range of the sorted order (the layers z0 .. z1 - 1 sit
     between the halo layers): lj_compute_range evaluates exactly those targets, with the halo
     particles as candidates;
  4. the totals (energy, virial, pair count) are summed over the ranks (an FP64 all-reduce).

A particle's candidates, their cells and their order within the x-sorted rows are then those of
the single-domain run, so its energy and force come out the same.  Particles that move across a
slab boundary between steps would have to be handed to the neighbour before the next step; this
module evaluates one configuration (the benchmark step), it does not move particles.

The exchange is a parameter of `step`: `exchange_p2p` uses torch.distributed point-to-point
operations (NCCL between GPUs over NVLink, gloo between CPU processes); tests may pass an
in-process exchange between emulated ranks.
"""
from __future__ import annotations

from dataclasses import dataclass


def _torch():
    import torch

    return torch


@dataclass
class SlabDomain:
    """The z layers [z0, z1) of a grid with `gz` layers owned by `rank` of `world`."""
    rank: int
    world: int
    gx: int
    gy: int
    gz: int
    oz: float
    width: float

    @classmethod
    def of(cls, g, rank: int, world: int) -> "SlabDomain":
        if world < 1 or not 0 <= rank < world:
            raise ValueError(f"rank {rank} of {world}")
        if g.dim[2] < world:
            raise ValueError(f"{g.dim[2]} z layers cannot be split over {world} ranks")
        return cls(rank, world, int(g.dim[0]), int(g.dim[1]), int(g.dim[2]), float(g.origin[2]), float(g.width))

    @property
    def z0(self) -> int:
        return self.gz * self.rank // self.world

    @property
    def z1(self) -> int:
        return self.gz * (self.rank + 1) // self.world

    def z_cells(self, z):
        """Cell layer of each z coordinate as the library bins it (IEEE float32 subtraction and
        division, truncation, clamped to [0, gz - 1]; NaN lands in layer 0)."""
        torch = _torch()
        q = (z - torch.tensor(self.oz, dtype=torch.float32, device=z.device)) / \
            torch.tensor(self.width, dtype=torch.float32, device=z.device)
        q = torch.nan_to_num(q, nan=0.0)
        c = torch.where(q > 0, q.trunc(), torch.zeros_like(q))
        return c.clamp(max=self.gz - 1).to(torch.int64)

    def own(self, xyz):
        """The rows of an (n, 3) coordinate tensor whose cell layer this rank owns."""
        zc = self.z_cells(xyz[:, 2])
        return xyz[(zc >= self.z0) & (zc < self.z1)].contiguous()

    def halo_out(self, own_xyz):
        """(to the rank below, to the rank above): own particles of the first and last own layer
        (empty at the ends of the grid)."""
        torch = _torch()
        zc = self.z_cells(own_xyz[:, 2])
        empty = own_xyz[:0]
        down = own_xyz[zc == self.z0].contiguous() if self.rank > 0 else empty
        up = own_xyz[zc == self.z1 - 1].contiguous() if self.rank < self.world - 1 else empty
        return down, up

    def target_range(self, offsets):
        """[kb, ke): the sorted positions of the own layers in offsets of the global grid."""
        layer = self.gx * self.gy
        torch = _torch()
        idx = torch.tensor([self.z0 * layer, self.z1 * layer], dtype=torch.int64, device=offsets.device)
        kb, ke = offsets.index_select(0, idx).tolist()
        return int(kb), int(ke)


def exchange_p2p(dom: SlabDomain, down, up, group=None):
    """Halo exchange with the neighbours through torch.distributed: counts first, then the (k, 3)
    float32 coordinates.  Returns (from the rank below, from the rank above)."""
    torch = _torch()
    import torch.distributed as dist

    dev = down.device
    r, w = dom.rank, dom.world
    has_below, has_above = r > 0, r < w - 1
    n_out = [torch.tensor([down.shape[0]], dtype=torch.int64, device=dev),
             torch.tensor([up.shape[0]], dtype=torch.int64, device=dev)]
    n_in = [torch.zeros(1, dtype=torch.int64, device=dev), torch.zeros(1, dtype=torch.int64, device=dev)]
    ops = []
    if has_below:
        ops += [dist.P2POp(dist.isend, n_out[0], r - 1, group), dist.P2POp(dist.irecv, n_in[0], r - 1, group)]
    if has_above:
        ops += [dist.P2POp(dist.isend, n_out[1], r + 1, group), dist.P2POp(dist.irecv, n_in[1], r + 1, group)]
    if ops:
        for q in dist.batch_isend_irecv(ops):
            q.wait()
    below = torch.empty((int(n_in[0].item()), 3), dtype=torch.float32, device=dev)
    above = torch.empty((int(n_in[1].item()), 3), dtype=torch.float32, device=dev)
    ops = []
    if has_below:
        if down.shape[0]:
            ops.append(dist.P2POp(dist.isend, down, r - 1, group))
        if below.shape[0]:
            ops.append(dist.P2POp(dist.irecv, below, r - 1, group))
    if has_above:
        if up.shape[0]:
            ops.append(dist.P2POp(dist.isend, up, r + 1, group))
        if above.shape[0]:
            ops.append(dist.P2POp(dist.irecv, above, r + 1, group))
    if ops:
        for q in dist.batch_isend_irecv(ops):
            q.wait()
    return below, above


@dataclass
class SlabResult:
    binned: object       # the rank's Binned (own + halo particles, global grid)
    kb: int              # own targets: sorted positions [kb, ke)
    ke: int
    energy: object       # per sorted particle; valid on [kb, ke)
    force: object
    totals: object       # lj_totals of the own targets (device)
    halo: int            # halo particles received


# Particles per cell from which the library's default pair kernel takes two consecutive targets
# per lane with x-windows (kernel 10) instead of targets paired inside their cell over whole rows
# (kernel 12).  The library applies it to n / ncells of the whole grid; a slab fills only its own
# layers, so `step` applies it to the occupancy of those.
PAIR_CELL = 2.0


def pair_kernel_for(dom: SlabDomain, targets: int) -> int:
    cells = (dom.z1 - dom.z0) * dom.gx * dom.gy
    return 10 if targets >= PAIR_CELL * cells else 12


def step(ctx, g, p, dom: SlabDomain, own_xyz, exchange=None, order=1) -> SlabResult:
    """One decomposed evaluation on this rank (see the module docstring).  own_xyz: (m, 3) float32
    device coordinates of the rank's own particles, all in its layers [z0, z1) (as
    SlabDomain.own selects them).  exchange(dom, down, up) -> (below, above);
    default: exchange_p2p.  With the context's pair kernel left at 0 (default), the kernel is
    chosen from the occupancy of the own layers; a kernel set with set_tuning is kept.

    The boundary layers are picked on the device (lj_select_layers, input order kept); the local
    particles [below, own, above] are binned as one AoS array.  Their sorted order puts the layer
    below first and the layer above last (cells are ordered by z first), so the own particles are
    the sorted positions [len(below), len(below) + m) without reading the offsets back."""
    torch = _torch()
    down, up = ctx.select_layers(g, own_xyz, dom.z0 if dom.rank > 0 else -1,
                                 dom.z1 - 1 if dom.rank < dom.world - 1 else -1)
    below, above = (exchange or exchange_p2p)(dom, down, up)
    local = torch.cat([below, own_xyz, above]).contiguous()
    flat = local.view(-1)
    b = ctx.bin(g, flat, flat[1:], flat[2:], stride=3, order=order)
    kb = int(below.shape[0])
    ke = kb + int(own_xyz.shape[0])
    tuning = ctx.get_tuning()
    if tuning["pair_kernel"] == 0:
        ctx.set_tuning(pair_kernel_for(dom, ke - kb), tuning["scatter_passes"])
    try:
        e, f, tot = ctx.compute_range(g, p, b, kb, ke)
    finally:
        if tuning["pair_kernel"] == 0:
            ctx.set_tuning(0, tuning["scatter_passes"])
    return SlabResult(b, kb, ke, e, f, tot, int(below.shape[0] + above.shape[0]))


def allreduce_totals(totals, group=None) -> dict:
    """Sum of the ranks' lj_totals (FP64 energy and virial, pair count) through torch.distributed."""
    torch = _torch()
    import torch.distributed as dist

    t = totals.reshape(-1)[:4]
    ew = t[:2].clone()
    pairs = t[2:3].view(torch.int64).clone()     # the uint64 pair count (below 2^63)
    dist.all_reduce(ew, group=group)
    dist.all_reduce(pairs, group=group)
    return {"energy": float(ew[0]), "virial": float(ew[1]), "pairs": int(pairs[0])}
