"""GPU parity at the full sizes of the benchmark workloads, against the CPU oracle on the same
positions (the oracle's own seeded drand48 positions, fed to both sides):

  uniform 10M, rc = 0.01   (100^3 cells, about 42 partners per particle: the headline workload)
  shell    4M, rc = 0.005  (unit sphere about (0.5, 0.5, 0.5), 400^3 cells over [-0.5, 1.5]^3)
  uniform 10M, rc = 0.02   (50^3 cells, about 335 partners per particle)
  512 uneven systems in one batched step (36 of them checked: both distributions, the whole range
  of sizes)

Bit-exact: counts, offsets, permutation, sorted cell ids, sorted coordinates, cell descriptors,
the candidate count and the interacting-pair count.  Every particle's energy and force within the
FP32 tolerances of test_gpu_parity (error over the conditioning scale, norm-wise force error), and
the total energy within 1e-6 of FP64.  Particles whose FP64 results exceed the float range
(near-coincident pairs of the random inputs) are left out of the float comparisons and counted."""
import numpy as np
import pytest

import ljoracle as O

pytestmark = pytest.mark.gpu

FORCE_SCALED_TOL = 1e-5
ENERGY_SCALED_TOL = 1e-5
FORCE_NORMWISE_TOL = 1e-5
TOTAL_ENERGY_TOL = 1e-6

WORKLOADS = {
    "uniform10M_rc0.01": dict(kind="uniform", n=10_000_000, rc=0.01, lo=(0.0,) * 3, hi=(1.0,) * 3),
    "shell4M_rc0.005": dict(kind="shell", n=4_000_000, rc=0.005, lo=(-0.5,) * 3, hi=(1.5,) * 3),
    "uniform10M_rc0.02": dict(kind="uniform", n=10_000_000, rc=0.02, lo=(0.0,) * 3, hi=(1.0,) * 3),
}


def np_(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module", params=list(WORKLOADS))
def full(request, ctx, torch_cuda):
    import ljcell

    torch = torch_cuda
    w = WORKLOADS[request.param]
    if w["kind"] == "uniform":
        x, y, z = O.generate_uniform(1234, w["n"])
    else:
        x, y, z = O.generate_sphere(1234, w["n"], (0.5, 0.5, 0.5), 1.0)
    g = ljcell.grid_from_box(w["lo"], w["hi"], w["rc"])
    og = O.grid_from_box(w["lo"], w["hi"], w["rc"])
    assert tuple(og.dim) == tuple(g.dim)
    p = ljcell.params(w["rc"])
    d = [torch.from_numpy(a).cuda() for a in (x, y, z)]
    b = ctx.bin(g, *d, order=ljcell.ORDER_X, soa=True, cells=True)
    cand = ctx.count_candidates(g, b.offsets)
    energy, force, tot = ctx.compute(g, p, b)
    ctx.sync()
    n = w["n"]
    # the other sparse-grid kernels (the default there is 12: cell pairs over whole rows; 11: whole
    # rows, one target per lane; 6: row passes)
    extra = {}
    if w["kind"] == "shell":
        for k in (11, 6):
            ctx.set_tuning(k)
            try:
                ek, fk, tk = ctx.compute(g, p, b)
                ctx.sync()
            finally:
                ctx.set_tuning(0)
            extra[k] = (np_(ek)[:n], np_(fk)[:n], ljcell.totals_from_tensor(tk))
    gpu = {
        "counts": np_(b.counts), "offsets": np_(b.offsets), "cells": np_(b.cells).reshape(-1, 2),
        "xyzi": np_(b.xyzi)[:n], "cell": np_(b.cell)[:n],
        "soa": tuple(np_(t)[:n] for t in (b.sx, b.sy, b.sz)),
        "index": np_(b.index)[:n],
        "candidates": int(np_(cand).reshape(-1)[0]),
        "energy": np_(energy)[:n], "force": np_(force)[:n], "totals": ljcell.totals_from_tensor(tot),
        "extra": extra,
    }
    del d, b, cand, energy, force, tot
    torch.cuda.empty_cache()
    ob = O.bin_particles(og, x, y, z, O.ORDER_X)
    ref = O.config_forces(og, ob, w["rc"], 1.0, p.sigma, want32=False)
    yield {"name": request.param, "n": n, "og": og, "ob": ob, "gpu": gpu, "ref": ref,
           "ocand": O.count_candidates(og, ob.offsets)}


def test_binning_bit_exact(full):
    gpu, ob = full["gpu"], full["ob"]
    np.testing.assert_array_equal(gpu["counts"], ob.counts)
    np.testing.assert_array_equal(gpu["offsets"], ob.offsets)
    np.testing.assert_array_equal(gpu["xyzi"][:, 3].view(np.int32), ob.perm)
    np.testing.assert_array_equal(gpu["index"], ob.perm)
    np.testing.assert_array_equal(gpu["cell"], ob.cell_sorted)
    for k, ref in zip(range(3), (ob.sx, ob.sy, ob.sz)):
        np.testing.assert_array_equal(gpu["xyzi"][:, k], ref)
        np.testing.assert_array_equal(gpu["soa"][k], ref)
    np.testing.assert_array_equal(gpu["cells"][:, 0], ob.counts)        # nbParticleInCell
    np.testing.assert_array_equal(gpu["cells"][:, 1], ob.offsets[:-1])  # offsetInContainer


def test_candidate_count_exact(full):
    assert full["gpu"]["candidates"] == full["ocand"]


def test_pair_count_exact(full):
    assert full["gpu"]["totals"]["pairs"] == full["ref"].pairs


def test_every_particle_within_tolerance(full):
    ref, gpu = full["ref"], full["gpu"]
    fe = ref.force_errors(gpu["force"], FORCE_SCALED_TOL)
    ee = ref.energy_errors(gpu["energy"], ENERGY_SCALED_TOL)
    print(full["name"], "force", fe, "energy", ee)
    assert fe["max_scaled_over_tol"] <= 1.0, fe
    assert fe["normwise"] <= FORCE_NORMWISE_TOL, fe
    assert ee["max_scaled_over_tol"] <= 1.0, ee
    assert fe["excluded"] <= 1e-4 * full["n"], fe  # near-coincident pairs only


def test_total_energy(full):
    """E = 1/2 sum of the float per-particle energies, against FP64, over the particles whose FP64
    energies fit in float (all of them when none is excluded, and then also the library's own FP64
    total and virial)."""
    ref, gpu = full["ref"], full["gpu"]
    ok = ref.representable()
    e = gpu["energy"].astype(np.float64)
    assert np.all(np.isfinite(e[ok]))
    got, want = 0.5 * e[ok].sum(), 0.5 * ref.e64[ok].sum()
    assert abs(got - want) <= TOTAL_ENERGY_TOL * abs(want), (got, want)
    if ok.all():
        t = gpu["totals"]
        assert abs(t["energy"] - ref.etot) <= TOTAL_ENERGY_TOL * abs(ref.etot), (t["energy"], ref.etot)
        assert abs(t["virial"] - ref.virial) <= TOTAL_ENERGY_TOL * abs(ref.virial), (t["virial"], ref.virial)


def test_sparse_grid_kernel_on_the_shell(full):
    """Kernels 11 (whole rows) and 6 (row passes) on the shell, where the default is 12: pair count
    exact, every particle within tolerance, total energy within 1e-6."""
    ref, extra = full["ref"], full["gpu"]["extra"]
    if not extra:
        pytest.skip("the sparse-grid kernel is run on the shell workload")
    ok = ref.representable()
    for k, (e, f, t) in extra.items():
        assert t["pairs"] == ref.pairs, k
        fe = ref.force_errors(f, FORCE_SCALED_TOL)
        ee = ref.energy_errors(e, ENERGY_SCALED_TOL)
        assert fe["max_scaled_over_tol"] <= 1.0 and fe["normwise"] <= FORCE_NORMWISE_TOL, (k, fe)
        assert ee["max_scaled_over_tol"] <= 1.0, (k, ee)
        got, want = 0.5 * e[ok].astype(np.float64).sum(), 0.5 * ref.e64[ok].sum()
        assert abs(got - want) <= TOTAL_ENERGY_TOL * abs(want), (k, got, want)


# ------------------------------------------------------------------ 512 uneven systems
def spread(systems, kind, count):
    """`count` systems of one kind, evenly spread over their sizes (smallest and largest included)."""
    ids = sorted((s for s, d in enumerate(systems) if d["kind"] == kind), key=lambda s: systems[s]["n"])
    pick = np.unique(np.round(np.linspace(0, len(ids) - 1, count)).astype(int))
    return [ids[i] for i in pick]


def test_batch_512_systems_against_oracle(ctx, torch_cuda):
    """The batched workload as the benchmark runs it (512 systems, autotuned configuration, one
    graph replay per step): 24 uniform and 12 shell systems over the whole size range, each against
    the oracle on the positions the library generated."""
    import ljcell

    torch = torch_cuda
    w = ljcell.batch_workload()
    b = ljcell.Batch(ctx, w)
    xyz = b.generate()
    ctx.sync()
    b.autotune(*xyz)
    e, f, idx, tot = b.alloc_outputs()
    b.run(*xyz, e, f, idx, tot, mode="graph")
    ctx.sync()
    hx, hy, hz = (np_(t)[:b.ntotal] for t in xyz)
    e, f, idx = np_(e)[:b.ntotal], np_(f)[:b.ntotal], np_(idx)[:b.ntotal]
    totals = ljcell.totals_from_array(tot)
    chosen = spread(w, "uniform", 24) + spread(w, "shell", 12)
    assert len(chosen) >= 32
    sizes = sorted(w[s]["n"] for s in chosen)
    assert sizes[0] < 2000 and sizes[-1] > 150_000   # the range's two ends are covered
    for s in chosen:
        d = w[s]
        fst, n = d["first"], d["n"]
        g = b.grid(s)
        og = O.grid_from_box(d["lo"], d["hi"], g.width)
        assert tuple(og.dim) == tuple(g.dim) and tuple(og.origin) == tuple(g.origin)
        sl = slice(fst, fst + n)
        ob = O.bin_particles(og, hx[sl].copy(), hy[sl].copy(), hz[sl].copy(), O.ORDER_X)
        np.testing.assert_array_equal(idx[sl] - fst, ob.perm)
        p = b.params(s)
        ref = O.config_forces(og, ob, p.cutoff, p.epsilon, p.sigma, want32=False)
        assert totals[s]["pairs"] == ref.pairs, s
        fe = ref.force_errors(f[sl], FORCE_SCALED_TOL)
        ee = ref.energy_errors(e[sl], ENERGY_SCALED_TOL)
        assert fe["max_scaled_over_tol"] <= 1.0 and fe["normwise"] <= FORCE_NORMWISE_TOL, (s, fe)
        assert ee["max_scaled_over_tol"] <= 1.0, (s, ee)
        ok = ref.representable()
        got, want = 0.5 * e[sl][ok].astype(np.float64).sum(), 0.5 * ref.e64[ok].sum()
        assert abs(got - want) <= TOTAL_ENERGY_TOL * abs(want) + 1e-300, (s, got, want)
        if ok.all() and ref.pairs:
            assert abs(totals[s]["energy"] - ref.etot) <= TOTAL_ENERGY_TOL * abs(ref.etot), s
    b.close()
    del xyz
    torch.cuda.empty_cache()
