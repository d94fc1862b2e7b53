"""GPU failure detection without a GPU fault.  The scan's look-back waits are
bounded: with the first tile withheld (a predecessor flag that nothing sets)
every wait gives up, the kernel records a timeout in the context's status
word and returns; lj_sync reports LJ_ETIMEOUT, clears it, and the same
context then computes a correct scan.  Allocation failures are injected on
the host (lj_test_fail_alloc): the call reports LJ_ENOMEM and the context
recovers."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_recovers(torch_cuda, ctx):
    import ljcell

    torch = torch_cuda
    n = 100_000
    counts = torch.randint(0, 5, (n,), dtype=torch.int32, device="cuda")
    out = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    rc = ljcell.lib().lj_test_scan_withheld_tile(ctx.handle, ljcell._ptr(counts), n, ljcell._ptr(out))
    assert rc == ljcell.LJ_OK
    with pytest.raises(ljcell.LJError) as ei:
        ctx.sync()
    waited = time.perf_counter() - t0
    assert ei.value.status == ljcell.LJ_ETIMEOUT
    assert waited < 30.0, waited
    ctx.sync()   # the status word was cleared
    off = ctx.exclusive_scan(counts)
    ctx.sync()
    ref = np.concatenate([[0], np.cumsum(counts.cpu().numpy().astype(np.int64))])
    np.testing.assert_array_equal(off.cpu().numpy(), ref)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_allocation_failure_is_reported_and_the_context_recovers(torch_cuda, ctx, k):
    """A fresh context grows five scratch buffers on its first bin + compute (tickets, unsorted
    records, large-cell list, scan state, reduction partials).  Making the k-th growth fail, as a
    cudaMalloc failure would, gives LJ_ENOMEM from the call that needed it, not a crash; the same
    context then bins and computes with the results of a context that never failed."""
    import ljcell
    from test_gpu_parity import case_positions, dev, np_

    torch = torch_cuda
    (x, y, z), (lo, hi), rc = case_positions("uniform_c1")
    g = ljcell.grid_from_box(lo, hi, rc)
    p = ljcell.params(rc)
    d = [dev(torch, a) for a in (x, y, z)]
    fresh = ljcell.Context(0)
    try:
        ljcell.test_fail_alloc(k)
        try:
            with pytest.raises(ljcell.LJError) as err:
                b = fresh.bin(g, *d, order=1)
                fresh.compute(g, p, b)
                fresh.sync()
            assert err.value.status == ljcell.LJ_ENOMEM
        finally:
            ljcell.test_fail_alloc(0)
        fresh.sync()
        b = fresh.bin(g, *d, order=1)
        e, f, t = fresh.compute(g, p, b)
        fresh.sync()
        b0 = ctx.bin(g, *d, order=1)
        e0, f0, t0 = ctx.compute(g, p, b0)
        ctx.sync()
        n = len(x)
        assert np.array_equal(np_(b.xyzi)[:n].view(np.uint32), np_(b0.xyzi)[:n].view(np.uint32))
        assert np.array_equal(np_(e)[:n].view(np.uint32), np_(e0)[:n].view(np.uint32))
        assert np.array_equal(np_(f)[:n].view(np.uint32), np_(f0)[:n].view(np.uint32))
        assert ljcell.totals_from_tensor(t) == ljcell.totals_from_tensor(t0)
    finally:
        fresh.close()
