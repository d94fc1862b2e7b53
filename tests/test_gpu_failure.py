"""GPU failure detection without a GPU fault.  The scan's look-back waits are
bounded: with the first tile withheld (a predecessor flag that nothing sets)
every wait gives up, the kernel records a timeout in the context's status
word and returns; lj_sync reports LJ_ETIMEOUT, clears it, and the same
context then computes a correct scan."""
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
