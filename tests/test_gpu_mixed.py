"""GPU: the mixed-precision form (FP32 x + binary16 cell-relative y, z
records; FP32 math; compensated per-particle sums; FP64 totals) against the
oracle's exact restatement: records bit-exact, interacting-pair count
bit-exact under the mixed distance test, forces and energies within the
stated tolerance of FP64 evaluated on the stored positions.  The change of
the inputs themselves (binary16 offsets) is reported, not bounded here."""
import numpy as np
import pytest

import ljoracle as O
from test_gpu_parity import bin_both, np_

pytestmark = pytest.mark.gpu

# compensated sums: same bounds as the plain form's, held here without the sqrt(m) growth allowance
FORCE_SCALED_TOL = 1e-5
FORCE_NORMWISE_TOL = 1e-5
TOTAL_ENERGY_TOL = 1e-6


# 0: default (row passes, two targets per lane); 1 / 2: flat walk, windows in shared memory / in
# registers; 6: row passes, one target per lane
@pytest.mark.parametrize("kernel", [0, 1, 2, 6])
@pytest.mark.parametrize("name", ["uniform_c1", "uniform_dense", "shell", "tiny33"])
def test_mixed_against_oracle(torch_cuda, ctx, name, kernel):
    import ljcell

    (x, y, z), g, og, b, ob, rc = bin_both(torch_cuda, ctx, name, 1)
    p = ljcell.params(rc)
    ctx.set_tuning(kernel)
    rec = ctx.pack_mixed(g, b)
    e, f, tot = ctx.compute_mixed(g, p, b, rec)
    ctx.sync()
    ctx.set_tuning(0)
    n = len(x)
    r = np_(rec)[:n]
    uy, uz = O.pack_mixed(og, ob)
    halves = r[:, 1].copy().view(np.float16).reshape(n, 2).astype(np.float32)
    np.testing.assert_array_equal(r[:, 0], ob.sx)
    np.testing.assert_array_equal(halves[:, 0], uy)
    np.testing.assert_array_equal(halves[:, 1], uz)
    ref = O.mixed_forces(og, ob, uy, uz, rc, 1.0, p.sigma)
    t = ljcell.totals_from_tensor(tot)
    assert t["pairs"] == ref.pairs
    fe = ref.force_errors(np_(f)[:n])
    ee = ref.energy_errors(np_(e)[:n])
    assert fe["max_scaled"] <= FORCE_SCALED_TOL and fe["normwise"] <= FORCE_NORMWISE_TOL, fe
    assert ee["max_scaled"] <= FORCE_SCALED_TOL, ee
    if ref.pairs and fe["excluded"] == 0:
        assert abs(t["energy"] - ref.etot) <= TOTAL_ENERGY_TOL * abs(ref.etot)


def test_mixed_deterministic(torch_cuda, ctx):
    import ljcell

    (x, y, z), g, og, b, ob, rc = bin_both(torch_cuda, ctx, "uniform_c1", 1)
    p = ljcell.params(rc)
    outs = []
    for _ in range(2):
        rec = ctx.pack_mixed(g, b)
        e, f, tot = ctx.compute_mixed(g, p, b, rec)
        ctx.sync()
        outs.append((np_(e), np_(f), np_(tot)))
    for a, c in zip(*outs):
        assert np.array_equal(a.view(np.uint8), c.view(np.uint8))


def test_mixed_dense_sample(torch_cuda, ctx):
    """The dense configuration (10M uniform, rc = 0.02, about 335 neighbours):
    errors of the mixed form on 50,000 targets against FP64 on the stored
    positions, and the effect of the binary16 offsets themselves (stored vs
    unrounded positions), printed for the record."""
    import ljcell

    torch = torch_cuda
    n, rc = 10_000_000, 0.02
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    p = ljcell.params(rc)
    soa, _ = ctx.generate_uniform(1234, n)
    b = ctx.bin(g, soa["x"], soa["y"], soa["z"], order=1)
    rec = ctx.pack_mixed(g, b)
    e, f, tot = ctx.compute_mixed(g, p, b, rec)
    ctx.sync()
    xyzi = np_(b.xyzi)[:n]
    ob = O.Binned(None, np_(b.offsets), xyzi[:, 3].view(np.int32).copy(), np_(b.cell)[:n].copy(),
                  np.ascontiguousarray(xyzi[:, 0]), np.ascontiguousarray(xyzi[:, 1]), np.ascontiguousarray(xyzi[:, 2]))
    og = O.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    uy, uz = O.pack_mixed(og, ob)
    k0, k1 = n // 2, n // 2 + 50_000
    stored = O.mixed_forces(og, ob, uy, uz, rc, 1.0, p.sigma, k0, k1)
    fe = stored.force_errors(np_(f)[k0:k1])
    ee = stored.energy_errors(np_(e)[k0:k1])
    cy = (ob.cell_sorted // og.dim[0]) % og.dim[1]
    cz = ob.cell_sorted // (og.dim[0] * og.dim[1])
    w = np.float32(rc)
    uy32 = ((ob.sy - cy.astype(np.float32) * w) / w).astype(np.float32)
    uz32 = ((ob.sz - cz.astype(np.float32) * w) / w).astype(np.float32)
    orig = O.mixed_forces(og, ob, uy32, uz32, rc, 1.0, p.sigma, k0, k1)
    ok = orig.representable() & stored.representable()
    q = float(np.linalg.norm(stored.f64[ok] - orig.f64[ok]) / np.linalg.norm(orig.f64[ok]))
    print(f"mixed dense sample: force normwise {fe['normwise']:.3e} max scaled {fe['max_scaled']:.3e} "
          f"p99 rel {fe['p99_rel']:.3e}; energy max scaled {ee['max_scaled']:.3e}; "
          f"binary16 input effect on forces {q:.3e}")
    assert fe["normwise"] <= FORCE_NORMWISE_TOL and fe["max_scaled"] <= FORCE_SCALED_TOL, fe
    assert ee["max_scaled"] <= FORCE_SCALED_TOL, ee
    del soa, b, rec, e, f, tot
    torch.cuda.empty_cache()
