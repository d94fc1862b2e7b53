"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU
oracle on the same seeded inputs.  Integer and index outputs (generation of
the uniform box, counts, offsets, permutation, cell ids, descriptors,
candidate and interacting-pair counts) must be bit-exact; floating-point
outputs are held to the tolerances stated in each test."""
import numpy as np
import pytest

import ljoracle as O

pytestmark = pytest.mark.gpu

# FP32 pair math against the FP64 oracle: error relative to each particle's
# conditioning scale (sum of the pair terms' magnitudes before cancellation),
# at most max(1e-5, 16 u sqrt(m)) for a particle with m interacting neighbours
# (u = 2^-24: float summation error grows like u sqrt(m)).  Particles whose
# FP64 energy or force exceeds the float range are not compared.
FORCE_SCALED_TOL = 1e-5
ENERGY_SCALED_TOL = 1e-5
FORCE_NORMWISE_TOL = 1e-5     # ||F - F64|| / ||F64|| over all particles
TOTAL_ENERGY_TOL = 1e-6       # |E - E64| / |E64|
COMPAT_REL_TOL = 1e-5         # reference tolerance, cudaLJ.cu:246-250


def np_(t):
    return t.detach().cpu().numpy()


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


# ------------------------------------------------------------------ inputs
def case_positions(name):
    if name == "uniform_c1":
        x, y, z = O.generate_uniform(1234, 100_000)
        return (x, y, z), ((0, 0, 0), (1, 1, 1)), 0.05
    if name == "uniform_dense":
        x, y, z = O.generate_uniform(77, 60_000)
        return (x, y, z), ((0, 0, 0), (1, 1, 1)), 0.1
    if name == "shell":
        x, y, z = O.generate_sphere(1234, 150_000, (0.5, 0.5, 0.5), 1.0)
        return (x, y, z), ((-0.5,) * 3, (1.5,) * 3), 0.01
    if name == "clustered":
        # one cell holds 5000 particles (beyond the warp sort), plus background
        rng = np.random.default_rng(5)
        a = rng.random((5000, 3), dtype=np.float32) * np.float32(0.01) + np.float32(0.4)
        b = rng.random((20000, 3), dtype=np.float32)
        p = np.concatenate([a, b]).astype(np.float32)
        return (p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy()), ((0, 0, 0), (1, 1, 1)), 0.05
    if name == "outside_and_faces":
        rng = np.random.default_rng(9)
        w = np.float32(0.0625)
        faces = np.unique((rng.integers(0, 17, (3000, 3)) * w).astype(np.float32), axis=0)  # no coincident pairs
        out = (rng.random((500, 3)) * 1.6 - 0.3).astype(np.float32)
        inner = rng.random((8000, 3), dtype=np.float32)
        p = np.concatenate([faces, out, inner]).astype(np.float32)
        return (p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy()), ((0, 0, 0), (1, 1, 1)), float(w)
    if name.startswith("tiny"):
        n = int(name[4:])
        x, y, z = O.generate_uniform(3, n)
        return (x, y, z), ((0, 0, 0), (1, 1, 1)), 0.25
    raise KeyError(name)


BIN_CASES = ["uniform_c1", "uniform_dense", "shell", "clustered", "outside_and_faces", "tiny1", "tiny2", "tiny33"]


def bin_both(torch, ctx, name, order, stride=1):
    import ljcell

    (x, y, z), (lo, hi), rc = case_positions(name)
    g = ljcell.grid_from_box(lo, hi, rc)
    og = O.grid_from_box(lo, hi, rc)
    if stride == 3:
        aos = dev(torch, np.stack([x, y, z], axis=1).reshape(-1))
        b = ctx.bin(g, aos, aos[1:], aos[2:], stride=3, order=order, out=ctx.alloc_binned(g, len(x), order, True,
                                                                                             True))
    else:
        b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=order, soa=True, cells=True)
    ctx.sync()
    ob = O.bin_particles(og, x, y, z, order)
    return (x, y, z), g, og, b, ob, rc


# ------------------------------------------------------------------ generation
def test_generate_uniform_bit_exact(ctx):
    n = 100_003
    soa, aos = ctx.generate_uniform(1234, n, aos=True)
    ctx.sync()
    x, y, z = O.generate_uniform(1234, n)
    np.testing.assert_array_equal(np_(soa["x"]), x)
    np.testing.assert_array_equal(np_(soa["y"]), y)
    np.testing.assert_array_equal(np_(soa["z"]), z)
    np.testing.assert_array_equal(np_(aos), np.stack([x, y, z], 1))
    np.testing.assert_array_equal(np_(soa["index"]), np.arange(n, dtype=np.int32))
    assert np.all(np_(soa["v"]) == -1.0)


def test_generate_uniform_box_bit_exact(ctx):
    soa, _ = ctx.generate_uniform(99, 5000, lo=(-0.5, 0.25, 2.0), hi=(1.5, 0.75, 3.0))
    ctx.sync()
    x, y, z = O.generate_uniform(99, 5000, (-0.5, 0.25, 2.0), (1.5, 0.75, 3.0))
    np.testing.assert_array_equal(np_(soa["x"]), x)
    np.testing.assert_array_equal(np_(soa["z"]), z)


def test_generate_sphere_within_one_ulp(ctx):
    n = 50_000
    soa, _ = ctx.generate_sphere(1234, n, (0.5, 0.5, 0.5), 1.0)
    ctx.sync()
    ref = O.generate_sphere(1234, n, (0.5, 0.5, 0.5), 1.0)
    for k, r in zip("xyz", ref):
        d = np.abs(np_(soa[k]).astype(np.float64) - r.astype(np.float64))
        assert np.all(d <= np.spacing(np.abs(r)).astype(np.float64)), k


# ------------------------------------------------------------------ scan
@pytest.mark.parametrize("ncells", [1, 5, 4095, 4096, 4097, 123_457, 1_000_000, 64_000_000])
def test_exclusive_scan(torch_cuda, ctx, ncells):
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(ncells)
    counts = torch.randint(0, 4, (ncells,), dtype=torch.int32, device="cuda", generator=g)
    off = ctx.exclusive_scan(counts)
    ctx.sync()
    c = np_(counts).astype(np.int64)
    ref = np.concatenate([[0], np.cumsum(c)])
    np.testing.assert_array_equal(np_(off).astype(np.int64), ref)


def test_exclusive_scan_unaligned(torch_cuda, ctx):
    torch = torch_cuda
    base = torch.randint(0, 9, (100_001,), dtype=torch.int32, device="cuda")
    out = torch.empty(100_002, dtype=torch.int32, device="cuda")
    off = ctx.exclusive_scan(base[1:], out[1:])
    ctx.sync()
    ref = np.concatenate([[0], np.cumsum(np_(base[1:]).astype(np.int64))])
    np.testing.assert_array_equal(np_(off), ref)


def test_scan_matches_reference_semantics(torch_cuda, ctx):
    # reference: memset prefix, PrefixFullV2(counts, prefix + 1) -> prefix[0] = 0, prefix[i+1] = sum counts[0..i]
    torch = torch_cuda
    counts = torch.randint(0, 30, (20 ** 3,), dtype=torch.int32, device="cuda")
    off = ctx.exclusive_scan(counts)
    ctx.sync()
    o = np_(off)
    assert o[0] == 0 and np.array_equal(np.diff(o), np_(counts))


# ------------------------------------------------------------------ binning
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("name", BIN_CASES)
def test_bin_bit_exact(torch_cuda, ctx, name, order):
    (x, y, z), g, og, b, ob, _ = bin_both(torch_cuda, ctx, name, order)
    np.testing.assert_array_equal(np_(b.counts), ob.counts)
    np.testing.assert_array_equal(np_(b.offsets), ob.offsets)
    n = len(x)
    xyzi = np_(b.xyzi)[:n]
    np.testing.assert_array_equal(xyzi[:, 3].view(np.int32), ob.perm)
    np.testing.assert_array_equal(xyzi[:, 0], ob.sx)
    np.testing.assert_array_equal(xyzi[:, 1], ob.sy)
    np.testing.assert_array_equal(xyzi[:, 2], ob.sz)
    np.testing.assert_array_equal(np_(b.cell)[:n], ob.cell_sorted)
    np.testing.assert_array_equal(np_(b.sx)[:n], ob.sx)
    np.testing.assert_array_equal(np_(b.index)[:n], ob.perm)
    cells = np_(b.cells)
    np.testing.assert_array_equal(cells[:, 0], ob.counts)
    np.testing.assert_array_equal(cells[:, 1], ob.offsets[:-1])


@pytest.mark.parametrize("name", ["uniform_c1", "outside_and_faces"])
def test_bin_aos_point3d_input(torch_cuda, ctx, name):
    (x, y, z), g, og, b, ob, _ = bin_both(torch_cuda, ctx, name, 1, stride=3)
    np.testing.assert_array_equal(np_(b.offsets), ob.offsets)
    np.testing.assert_array_equal(np_(b.xyzi)[:len(x), 3].view(np.int32), ob.perm)


def test_count_cells_and_descriptors(torch_cuda, ctx):
    torch = torch_cuda
    import ljcell

    x, y, z = O.generate_uniform(8, 70_000)
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), 0.04)
    og = O.grid_from_box((0, 0, 0), (1, 1, 1), 0.04)
    counts = ctx.count_cells(g, dev(torch, x), dev(torch, y), dev(torch, z))
    off = ctx.exclusive_scan(counts)
    cells = ctx.cell_descriptors(off)
    ctx.sync()
    ob = O.bin_particles(og, x, y, z)
    np.testing.assert_array_equal(np_(counts), ob.counts)
    np.testing.assert_array_equal(np_(cells)[:, 1], ob.offsets[:-1])


def test_bin_empty(torch_cuda, ctx):
    torch = torch_cuda
    import ljcell

    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), 0.25)
    e = torch.empty(0, dtype=torch.float32, device="cuda")
    b = ctx.bin(g, e, e, e)
    ctx.sync()
    assert np.all(np_(b.counts) == 0) and np.all(np_(b.offsets) == 0)
    energy, force, tot = ctx.compute(g, ljcell.params(0.25), b)
    ctx.sync()
    assert ljcell.totals_from_tensor(tot)["pairs"] == 0


def test_non_finite_position_reported(torch_cuda, ctx):
    torch = torch_cuda
    import ljcell

    x, y, z = O.generate_uniform(1, 1000)
    x[10] = np.nan
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), 0.1)
    ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z))
    with pytest.raises(ljcell.LJError) as ei:
        ctx.sync()
    assert ei.value.status == ljcell.LJ_ERANGE
    ctx.sync()  # status word cleared


# ------------------------------------------------------------------ candidates / compat law
@pytest.mark.parametrize("name", ["uniform_c1", "shell", "clustered", "outside_and_faces", "tiny2"])
def test_candidate_count_exact(torch_cuda, ctx, name):
    (x, y, z), g, og, b, ob, _ = bin_both(torch_cuda, ctx, name, 1)
    cnt = ctx.count_candidates(g, b.offsets)
    ctx.sync()
    assert int(np_(cnt)[0]) == O.count_candidates(og, ob.offsets)


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("name", ["uniform_c1", "shell", "outside_and_faces", "tiny33"])
def test_compat_energy(torch_cuda, ctx, name, order):
    (x, y, z), g, og, b, ob, _ = bin_both(torch_cuda, ctx, name, order)
    v = np_(ctx.compute_compat(g, b))[:len(x)]
    ctx.sync()
    ref = O.compat_energy(og, ob)
    rel = np.where(ref == 0, np.abs(v), np.abs((ref - v) / np.where(ref == 0, 1, ref)))
    assert rel.max() <= COMPAT_REL_TOL


# ------------------------------------------------------------------ config law
# (order, pair kernel): LJ_ORDER_INDEX has one kernel; LJ_ORDER_X has kernels 1, 6, 10, 11 and 12 (see lj_tuning)
VARIANTS = [(0, 0), (1, 1), (1, 6), (1, 10), (1, 11), (1, 12)]


@pytest.mark.parametrize("order,kernel", VARIANTS, ids=[f"order{o}-k{k}" for o, k in VARIANTS])
@pytest.mark.parametrize("name", ["uniform_c1", "uniform_dense", "shell", "clustered", "outside_and_faces",
                                  "tiny2", "tiny33"])
def test_config_forces(torch_cuda, ctx, name, order, kernel):
    import ljcell

    ctx.set_tuning(kernel)
    (x, y, z), g, og, b, ob, rc = bin_both(torch_cuda, ctx, name, order)
    # the cluster packs 5000 particles into 1e-6 volume: a small sigma keeps s^12 inside float range
    p = ljcell.params(rc, sigma=rc / 500 if name == "clustered" else None)
    energy, force, tot = ctx.compute(g, p, b)
    ctx.sync()
    n = len(x)
    t = ljcell.totals_from_tensor(tot)
    ref = O.config_forces(og, ob, rc, 1.0, p.sigma)
    assert t["pairs"] == ref.pairs
    e = np_(energy)[:n]
    f = np_(force)[:n]
    fe = ref.force_errors(f, FORCE_SCALED_TOL)
    ee = ref.energy_errors(e, ENERGY_SCALED_TOL)
    assert fe["max_scaled_over_tol"] <= 1.0, fe
    assert fe["normwise"] <= FORCE_NORMWISE_TOL, fe
    assert ee["max_scaled_over_tol"] <= 1.0, ee
    ctx.set_tuning(0)
    if ref.pairs and fe["excluded"] == 0:
        assert abs(t["energy"] - ref.etot) <= TOTAL_ENERGY_TOL * abs(ref.etot), (t["energy"], ref.etot)
        assert abs(t["virial"] - ref.virial) <= TOTAL_ENERGY_TOL * abs(ref.virial) + 1e-300
        assert abs(t["energy"] - 0.5 * e.astype(np.float64).sum()) <= 1e-12 * abs(ref.etot) + 1e-300


@pytest.mark.parametrize("alias,kernel", [(2, 1), (3, 1), (4, 1), (5, 6), (7, 6), (8, 10), (9, 10)])
def test_retired_kernel_numbers_run_their_family(torch_cuda, ctx, alias, kernel):
    """Tuning values of retired variants select the surviving kernel of their family: same bits."""
    import ljcell

    torch = torch_cuda
    (x, y, z), (lo, hi), rc = case_positions("uniform_dense")
    g = ljcell.grid_from_box(lo, hi, rc)
    b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
    outs = []
    for k in (alias, kernel):
        ctx.set_tuning(k)
        e, f, tot = ctx.compute(g, ljcell.params(rc), b)
        ctx.sync()
        outs.append((np_(e), np_(f), np_(tot)))
    ctx.set_tuning(0)
    for a, c in zip(*outs):
        assert np.array_equal(a.view(np.uint8), c.view(np.uint8))


def test_config_tiny_cutoff_pair_count(torch_cuda, ctx):
    # small cutoff relative to coordinates: the window slack must still keep every partner
    import ljcell

    torch = torch_cuda
    rng = np.random.default_rng(12)
    base = rng.random((20000, 3)).astype(np.float32) * np.float32(0.02) + np.float32(100.0)
    x, y, z = (base[:, i].copy() for i in range(3))
    lo, hi, rc = (100.0, 100.0, 100.0), (100.02, 100.02, 100.02), 0.0008
    g = ljcell.grid_from_box(lo, hi, rc)
    og = O.grid_from_box(lo, hi, rc)
    b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
    _, _, tot = ctx.compute(g, ljcell.params(rc), b)
    ctx.sync()
    ob = O.bin_particles(og, x, y, z, 1)
    ref = O.config_forces(og, ob, rc)
    assert ljcell.totals_from_tensor(tot)["pairs"] == ref.pairs


@pytest.mark.parametrize("kernel", [1, 6, 10, 11, 12])
def test_deterministic(torch_cuda, ctx, kernel):
    import ljcell

    torch = torch_cuda
    ctx.set_tuning(kernel)
    (x, y, z), (lo, hi), rc = case_positions("uniform_c1")
    g = ljcell.grid_from_box(lo, hi, rc)
    outs = []
    for _ in range(2):
        b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
        e, f, tot = ctx.compute(g, ljcell.params(rc), b)
        ctx.sync()
        outs.append((np_(b.xyzi), np_(e), np_(f), np_(tot)))
    ctx.set_tuning(0)
    for a, c in zip(*outs):
        assert np.array_equal(a.view(np.uint8), c.view(np.uint8))


@pytest.mark.parametrize("name,kernel", [("uniform_c1", 0), ("uniform_c1", 1), ("uniform_c1", 6),
                                         ("uniform_c1", 10), ("uniform_c1", 11), ("uniform_c1", 12),
                                         ("tiny33", 0), ("tiny33", 12)])
def test_simulate_host_matches_device_path(torch_cuda, ctx, name, kernel):
    """The host entry runs the pair stage in target chunks (one chunk for small
    n); per-particle outputs equal one full-range
    device call bit for bit, totals to FP64 rounding of the chunk sum."""
    import ljcell

    torch = torch_cuda
    (x, y, z), (lo, hi), rc = case_positions(name)
    n = len(x)
    g = ljcell.grid_from_box(lo, hi, rc)
    p = ljcell.params(rc)
    he = np.empty(n, np.float32)
    hf = np.empty((n, 3), np.float32)
    hi_ = np.empty(n, np.int32)
    ctx.set_tuning(kernel)
    try:
        tot = ctx.simulate_host(g, p, x, y, z, he, hf, hi_)
        b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
        e, f, t2 = ctx.compute(g, p, b)
        ctx.sync()
    finally:
        ctx.set_tuning(0)
    np.testing.assert_array_equal(he, np_(e)[:n])
    np.testing.assert_array_equal(hf, np_(f)[:n])
    np.testing.assert_array_equal(hi_, np_(b.xyzi)[:n, 3].view(np.int32))
    t2 = ljcell.totals_from_tensor(t2)
    assert tot.pairs == t2["pairs"]
    assert abs(tot.energy - t2["energy"]) <= 1e-12 * max(abs(t2["energy"]), 1e-300)


def test_autotune_compute_picks_a_kernel_and_keeps_results(torch_cuda, ctx):
    import ljcell

    (x, y, z), g, og, b, ob, rc = bin_both(torch_cuda, ctx, "uniform_dense", 1)
    p = ljcell.params(rc)
    kern, ms = ctx.autotune_compute(g, p, b)
    assert kern in (1, 6, 10, 11, 12) and ms > 0 and ctx.get_tuning()["pair_kernel"] == kern
    _, _, tot = ctx.compute(g, p, b)
    ctx.sync()
    ctx.set_tuning(0)
    assert ljcell.totals_from_tensor(tot)["pairs"] == O.config_forces(og, ob, rc).pairs


@pytest.mark.parametrize("passes", [1, 2, 3, 8])
@pytest.mark.parametrize("name", ["uniform_c1", "shell", "clustered"])
def test_bin_scatter_passes_bit_exact(torch_cuda, ctx, name, passes):
    """The binning scatter split into passes over cell ranges gives the oracle's binning bit for bit."""
    ctx.set_tuning(0, passes)
    try:
        (x, y, z), g, og, b, ob, _ = bin_both(torch_cuda, ctx, name, 1)
    finally:
        ctx.set_tuning(0)
    np.testing.assert_array_equal(np_(b.offsets), ob.offsets)
    np.testing.assert_array_equal(np_(b.xyzi)[:len(x), 3].view(np.int32), ob.perm)
    np.testing.assert_array_equal(np_(b.cell)[:len(x)], ob.cell_sorted)


def test_simulate_host_async_matches_one_call(torch_cuda, ctx):
    """Back-to-back lj_simulate_host_async calls (two device buffer sets used in turn, uploads on their
    own stream) give, per call, the outputs of lj_simulate_host on the same inputs, bit for bit."""
    import ljcell

    torch = torch_cuda
    (x, y, z), (lo, hi), rc = case_positions("uniform_c1")
    n = len(x)
    g = ljcell.grid_from_box(lo, hi, rc)
    p = ljcell.params(rc)
    inputs = [(x, y, z), (y.copy(), z.copy(), x.copy()), (z.copy(), x.copy(), y.copy())]

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    outs = []
    for (a, b, c) in inputs:
        hp = [pinned(n, torch.float32) for _ in range(3)]
        for h, v in zip(hp, (a, b, c)):
            h[:] = v
        outs.append((hp, pinned(n, torch.float32), pinned((n, 3), torch.float32), pinned(n, torch.int32)))
    tots = [ctx.simulate_host_async(g, p, *hp, he, hf, hi_) for hp, he, hf, hi_ in outs]
    ctx.simulate_host_wait()
    for (hp, he, hf, hi_), t in zip(outs, tots):
        re, rf, ri = np.empty(n, np.float32), np.empty((n, 3), np.float32), np.empty(n, np.int32)
        rt = ctx.simulate_host(g, p, *hp, re, rf, ri)
        np.testing.assert_array_equal(he, re)
        np.testing.assert_array_equal(hf, rf)
        np.testing.assert_array_equal(hi_, ri)
        assert t.pairs == rt.pairs and t.energy == rt.energy


@pytest.mark.parametrize("name", ["uniform_c1", "tiny33", "outside_and_faces"])
def test_simulate_host_inorder_matches_sorted_entry(torch_cuda, ctx, name):
    """lj_simulate_host_inorder(_async) returns energy and force in the caller's order: the sorted-order
    results of lj_simulate_host put back through its index, bit for bit; queued input-order and
    sorted-order calls may share one queue."""
    torch = torch_cuda
    import ljcell

    (x, y, z), (lo, hi), rc = case_positions(name)
    n = len(x)
    g = ljcell.grid_from_box(lo, hi, rc)
    p = ljcell.params(rc)
    se, sf, si = np.empty(n, np.float32), np.empty((n, 3), np.float32), np.empty(n, np.int32)
    st = ctx.simulate_host(g, p, x, y, z, se, sf, si)
    want_e, want_f = np.empty_like(se), np.empty_like(sf)
    want_e[si], want_f[si] = se, sf
    ie, if_ = np.empty(n, np.float32), np.empty((n, 3), np.float32)
    it = ctx.simulate_host_inorder(g, p, x, y, z, ie, if_)
    assert np.array_equal(ie.view(np.uint32), want_e.view(np.uint32))
    assert np.array_equal(if_.view(np.uint32), want_f.view(np.uint32))
    assert it.pairs == st.pairs and abs(it.energy - st.energy) <= 1e-12 * abs(st.energy) + 1e-300

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    hp = [pinned(n, torch.float32) for _ in range(3)]
    for h, v in zip(hp, (x, y, z)):
        h[:] = v
    outs = [(pinned(n, torch.float32), pinned((n, 3), torch.float32)) for _ in range(3)]
    ae, af, ai = pinned(n, torch.float32), pinned((n, 3), torch.float32), pinned(n, torch.int32)
    tots = [ctx.simulate_host_inorder_async(g, p, *hp, *outs[0]),
            ctx.simulate_host_async(g, p, *hp, ae, af, ai),
            ctx.simulate_host_inorder_async(g, p, *hp, *outs[1]),
            ctx.simulate_host_inorder_async(g, p, *hp, *outs[2])]
    ctx.simulate_host_wait()
    for e, f in outs:
        assert np.array_equal(e.view(np.uint32), want_e.view(np.uint32))
        assert np.array_equal(f.view(np.uint32), want_f.view(np.uint32))
    assert np.array_equal(ae, se) and np.array_equal(af, sf) and np.array_equal(ai, si)
    assert all(t.pairs == st.pairs for t in tots)


@pytest.mark.parametrize("kernel", [1, 6, 10, 11, 12])
def test_simulate_host_inorder_every_kernel(torch_cuda, ctx, kernel):
    """Each pair kernel writes a target's results at its input index in the input-order entry: the
    sorted entry's results put back through its index, bit for bit, with the same kernel."""
    import ljcell

    (x, y, z), (lo, hi), rc = case_positions("uniform_c1")
    n = len(x)
    g = ljcell.grid_from_box(lo, hi, rc)
    p = ljcell.params(rc)
    ctx.set_tuning(kernel)
    try:
        se, sf, si = np.empty(n, np.float32), np.empty((n, 3), np.float32), np.empty(n, np.int32)
        st = ctx.simulate_host(g, p, x, y, z, se, sf, si)
        ie, if_ = np.empty(n, np.float32), np.empty((n, 3), np.float32)
        it = ctx.simulate_host_inorder(g, p, x, y, z, ie, if_)
    finally:
        ctx.set_tuning(0)
    want_e, want_f = np.empty_like(se), np.empty_like(sf)
    want_e[si], want_f[si] = se, sf
    assert np.array_equal(ie.view(np.uint32), want_e.view(np.uint32))
    assert np.array_equal(if_.view(np.uint32), want_f.view(np.uint32))
    assert it.pairs == st.pairs


# Grids other than the unit cube: an anisotropic box far from the origin, a single row of cells
# (no neighbour rows in y or z), and cells twice as wide as the cutoff (a grid built for a larger
# cutoff and reused).  box lo, hi, grid cell width, law cutoff, particles.
GEOMETRIES = {
    "anisotropic_offset": ((-0.3, 0.1, 2.0), (0.9, 0.35, 2.2), 0.02, 0.02, 40_000),
    "one_row": ((0.0, 0.0, 0.0), (1.0, 0.03, 0.03), 0.03, 0.03, 3_000),
    "wide_cells": ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 0.1, 0.045, 60_000),
}


@pytest.mark.parametrize("kernel", [0, 1, 6, 10, 11, 12])
@pytest.mark.parametrize("geom", list(GEOMETRIES))
def test_config_forces_geometries(torch_cuda, ctx, geom, kernel):
    import ljcell

    torch = torch_cuda
    lo, hi, width, rc, n = GEOMETRIES[geom]
    rng = np.random.default_rng(len(geom) * 31 + n)
    lo32, hi32 = np.array(lo, np.float32), np.array(hi, np.float32)
    pts = (lo32 + (hi32 - lo32) * rng.random((n, 3), dtype=np.float32)).astype(np.float32)
    x, y, z = (np.ascontiguousarray(pts[:, k]) for k in range(3))
    g = ljcell.grid_from_box(lo, hi, width)
    og = O.grid_from_box(lo, hi, width)
    assert tuple(og.dim) == tuple(g.dim)
    p = ljcell.params(rc)
    ctx.set_tuning(kernel)
    try:
        b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
        energy, force, tot = ctx.compute(g, p, b)
        ctx.sync()
    finally:
        ctx.set_tuning(0)
    ob = O.bin_particles(og, x, y, z, O.ORDER_X)
    assert np.array_equal(np_(b.offsets), ob.offsets)
    ref = O.config_forces(og, ob, rc, 1.0, p.sigma)
    t = ljcell.totals_from_tensor(tot)
    assert t["pairs"] == ref.pairs and ref.pairs > 0
    fe = ref.force_errors(np_(force)[:n], FORCE_SCALED_TOL)
    ee = ref.energy_errors(np_(energy)[:n], ENERGY_SCALED_TOL)
    assert fe["max_scaled_over_tol"] <= 1.0 and fe["normwise"] <= FORCE_NORMWISE_TOL, fe
    assert ee["max_scaled_over_tol"] <= 1.0, ee
