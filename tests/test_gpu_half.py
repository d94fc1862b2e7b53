"""GPU: the half-shell pair evaluation (lj_compute_half), each unordered pair once with the reaction
applied to the partner, against the CPU oracle's full-shell evaluation on the same positions: the
ordered pair count bit-exact (twice the unordered count), every particle's energy and force within
the FP32 tolerance of test_gpu_parity, total energy within 1e-6 of FP64, and the same bits on every
run (no float atomics).  Sizes: the small CPU workload (100k, rc = 0.05), the edge cases of the
parity suite, and the 10M uniform workload at rc = 0.01."""
import numpy as np
import pytest

import ljoracle as O
from test_gpu_parity import bin_both, case_positions, dev, np_

pytestmark = pytest.mark.gpu

FORCE_SCALED_TOL = 1e-5
ENERGY_SCALED_TOL = 1e-5
FORCE_NORMWISE_TOL = 1e-5
TOTAL_ENERGY_TOL = 1e-6


def check(ref, e, f, t, n):
    assert t["pairs"] == ref.pairs
    fe = ref.force_errors(f, FORCE_SCALED_TOL)
    ee = ref.energy_errors(e, ENERGY_SCALED_TOL)
    assert fe["max_scaled_over_tol"] <= 1.0, fe
    assert fe["normwise"] <= FORCE_NORMWISE_TOL, fe
    assert ee["max_scaled_over_tol"] <= 1.0, ee
    ok = ref.representable()
    got, want = 0.5 * e[ok].astype(np.float64).sum(), 0.5 * ref.e64[ok].sum()
    assert abs(got - want) <= TOTAL_ENERGY_TOL * abs(want) + 1e-300, (got, want)
    if ok.all() and ref.pairs:
        assert abs(t["energy"] - ref.etot) <= TOTAL_ENERGY_TOL * abs(ref.etot), (t["energy"], ref.etot)
        assert abs(t["virial"] - ref.virial) <= TOTAL_ENERGY_TOL * abs(ref.virial) + 1e-300
    assert abs(t["energy"] - 0.5 * e.astype(np.float64).sum()) <= 1e-12 * abs(t["energy"]) + 1e-300


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("name", ["uniform_c1", "uniform_dense", "shell", "clustered", "outside_and_faces", "tiny1",
                                  "tiny2", "tiny33"])
def test_half_shell_against_oracle(torch_cuda, ctx, name, order):
    import ljcell

    (x, y, z), g, og, b, ob, rc = bin_both(torch_cuda, ctx, name, order)
    p = ljcell.params(rc, sigma=rc / 500 if name == "clustered" else None)
    energy, force, tot = ctx.compute_half(g, p, b)
    ctx.sync()
    n = len(x)
    ref = O.config_forces(og, ob, rc, 1.0, p.sigma, want32=False)
    check(ref, np_(energy)[:n], np_(force)[:n], ljcell.totals_from_tensor(tot), n)


def test_half_shell_matches_full_shell_pair_count_and_is_deterministic(torch_cuda, ctx):
    import ljcell

    torch = torch_cuda
    (x, y, z), (lo, hi), rc = case_positions("uniform_c1")
    g = ljcell.grid_from_box(lo, hi, rc)
    p = ljcell.params(rc)
    b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
    outs = [ctx.compute_half(g, p, b) for _ in range(2)]
    _, _, tfull = ctx.compute(g, p, b)
    ctx.sync()
    (e1, f1, t1), (e2, f2, t2) = [(np_(e), np_(f), np_(t)) for e, f, t in outs]
    assert np.array_equal(e1.view(np.uint32), e2.view(np.uint32))
    assert np.array_equal(f1.view(np.uint32), f2.view(np.uint32))
    assert np.array_equal(t1.view(np.uint8), t2.view(np.uint8))
    assert ljcell.totals_from_tensor(outs[0][2])["pairs"] == ljcell.totals_from_tensor(tfull)["pairs"]


def test_half_shell_uniform_10M(torch_cuda, ctx):
    """The headline workload, 10M uniform particles at rc = 0.01 (100^3 cells), every particle."""
    import ljcell

    torch = torch_cuda
    x, y, z = O.generate_uniform(1234, 10_000_000)
    rc = 0.01
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    p = ljcell.params(rc)
    b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
    energy, force, tot = ctx.compute_half(g, p, b)
    ctx.sync()
    n = len(x)
    e, f, t = np_(energy)[:n], np_(force)[:n], ljcell.totals_from_tensor(tot)
    del b, energy, force
    torch.cuda.empty_cache()
    og = O.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    ob = O.bin_particles(og, x, y, z, O.ORDER_X)
    ref = O.config_forces(og, ob, rc, 1.0, p.sigma, want32=False)
    check(ref, e, f, t, n)
