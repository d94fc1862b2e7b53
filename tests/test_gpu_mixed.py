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


@pytest.mark.parametrize("kernel", [1, 2])   # windows in shared memory / in registers
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
