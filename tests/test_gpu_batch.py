"""GPU: the batched step (many uneven systems in one launch per stage, a
persistent pair kernel fed by a device tile queue, graph replay, autotuner).
Per system, against the CPU oracle: interacting-pair counts bit-exact, forces
and energies within the plain-FP32 tolerance of test_gpu_parity.  Against the
per-system plain launches (lj_batch_run_separate): per-particle outputs bit
for bit (both use the same per-target routine), totals to 1e-12."""
import numpy as np
import pytest

import ljoracle as O

pytestmark = pytest.mark.gpu


def np_(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def small_batch(ctx):
    import ljcell

    w = ljcell.batch_workload(nsys=24, seed=77, n_min=50, n_max=6000, nb_min=10, nb_max=60)
    w.insert(5, {"kind": "uniform", "n": 0, "cutoff": 0.2, "lo": (0, 0, 0), "hi": (1, 1, 1), "seed": 5})  # empty system
    b = ljcell.Batch(ctx, w)
    x, y, z = b.generate()
    ctx.sync()
    yield b, (x, y, z)
    b.close()


def run(b, xyz, mode):
    e, f, idx, tot = b.alloc_outputs()
    b.run(*xyz, e, f, idx, tot, mode=mode)
    b.ctx.sync()
    return np_(e)[:b.ntotal], np_(f)[:b.ntotal], np_(idx)[:b.ntotal], tot


def check_against_oracle(b, xyz, e, f, idx, tot):
    import ljcell

    hx, hy, hz = (np_(t)[:b.ntotal] for t in xyz)
    totals = ljcell.totals_from_array(tot)
    for s, d in enumerate(b.systems):
        fst, n = d["first"], d["n"]
        if n == 0:
            assert totals[s]["pairs"] == 0
            continue
        g = b.grid(s)
        og = O.grid_from_box(d["lo"], d["hi"], g.width)   # the same formula as the library's grid
        assert tuple(og.dim) == tuple(g.dim) and tuple(og.origin) == tuple(g.origin)
        sl = slice(fst, fst + n)
        ob = O.bin_particles(og, hx[sl].copy(), hy[sl].copy(), hz[sl].copy(), O.ORDER_X)
        np.testing.assert_array_equal(idx[sl] - fst, ob.perm)
        p = b.params(s)
        ref = O.config_forces(og, ob, p.cutoff, p.epsilon, p.sigma)
        assert totals[s]["pairs"] == ref.pairs, s
        fe = ref.force_errors(f[sl])
        ee = ref.energy_errors(e[sl])
        assert fe["max_scaled_over_tol"] <= 1.0 and fe["normwise"] <= 1e-5, (s, fe)
        assert ee["max_scaled_over_tol"] <= 1.0, (s, ee)
        if fe["excluded"] == 0 and ref.pairs:
            assert abs(totals[s]["energy"] - ref.etot) <= 1e-6 * abs(ref.etot), s


def test_batch_matches_oracle(small_batch):
    b, xyz = small_batch
    check_against_oracle(b, xyz, *run(b, xyz, "plain"))


def test_batch_equals_separate_launches(small_batch):
    import ljcell

    b, xyz = small_batch
    e1, f1, i1, t1 = run(b, xyz, "plain")
    e2, f2, i2, t2 = run(b, xyz, "separate")
    np.testing.assert_array_equal(i1, i2)
    np.testing.assert_array_equal(e1.view(np.int32), e2.view(np.int32))
    np.testing.assert_array_equal(f1.view(np.int32), f2.view(np.int32))
    for a, c in zip(ljcell.totals_from_array(t1), ljcell.totals_from_array(t2)):
        assert a["pairs"] == c["pairs"]
        assert abs(a["energy"] - c["energy"]) <= 1e-12 * max(abs(c["energy"]), 1e-300)


def test_batch_graph_replay_bitwise(small_batch):
    b, xyz = small_batch
    ref = run(b, xyz, "plain")
    e, f, idx, tot = b.alloc_outputs()
    for _ in range(3):   # the first call captures the graph, later calls replay it (same pointers)
        for t in (e, f, idx, tot):
            t.zero_()
        b.run(*xyz, e, f, idx, tot, mode="graph")
        b.ctx.sync()
        got = (np_(e)[:b.ntotal], np_(f)[:b.ntotal], np_(idx)[:b.ntotal])
        for a, c in zip(ref[:3], got):
            assert np.array_equal(a.view(np.uint8), c.view(np.uint8))
        assert np.array_equal(np_(ref[3]).view(np.uint8), np_(tot).view(np.uint8))


def test_batch_autotune_keeps_results(small_batch):
    b, xyz = small_batch
    cfg, ms = b.autotune(*xyz)
    assert cfg["cell_multiple"] in (1.0, 1.5, 2.0) and cfg["threads"] in (64, 128, 256) and cfg["per_thread"] in (1, 2)
    assert ms > 0 and b.config() == cfg
    check_against_oracle(b, xyz, *run(b, xyz, "graph"))


@pytest.mark.parametrize("cm,threads,ppt", [(1.5, 64, 2), (2.0, 256, 1)])
def test_batch_configs(ctx, cm, threads, ppt):
    import ljcell

    w = ljcell.batch_workload(nsys=8, seed=3, n_min=100, n_max=3000, nb_min=15, nb_max=40)
    b = ljcell.Batch(ctx, w, cell_multiple=cm, threads=threads, per_thread=ppt)
    xyz = b.generate()
    ctx.sync()
    check_against_oracle(b, xyz, *run(b, xyz, "plain"))
    b.close()
