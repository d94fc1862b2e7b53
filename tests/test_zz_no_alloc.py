"""GPU: the allocation-free scan, lj_exclusive_scan_noalloc, called through
the C ABI.  It serves callers that cannot allocate device memory (a host whose
memory pool owns the device, or code that must not trigger the device-wide
synchronisation of cudaMalloc / cudaFree) and therefore cannot create an
lj_ctx.  Its result must equal the context-based lj_exclusive_scan on two calls
in a row: the second call is smaller than the first, so state left in the
shared scratch array by the first call would show up as a wrong answer.
This file is named to be collected last."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_scan_matches_context_scan_two_calls(torch_cuda):
    torch = torch_cuda
    import ljcell

    ctx = ljcell.Context(0)
    stream = torch.cuda.current_stream()
    try:
        for trial, (ncells, hi) in enumerate([(3_000_017, 7), (1_000_003, 40)]):
            gen = torch.Generator(device="cuda").manual_seed(100 + trial)
            counts = torch.randint(0, hi, (ncells,), dtype=torch.int32, device="cuda", generator=gen)
            ref = ctx.exclusive_scan(counts)
            ctx.sync()
            out = torch.full((ncells + 1,), -7, dtype=torch.int32, device="cuda")
            rc = ljcell.lib().lj_exclusive_scan_noalloc(_p(counts), ncells, _p(out), C.c_void_p(stream.cuda_stream))
            assert rc == ljcell.LJ_OK, ljcell.status_str(rc)
            torch.cuda.synchronize()
            assert torch.equal(out, ref), f"call {trial}: differs from lj_exclusive_scan"
            assert int(out[-1]) == int(counts.sum())
    finally:
        ctx.close()


def test_noalloc_scan_rejects_too_many_cells(torch_cuda):
    torch = torch_cuda
    import ljcell

    t = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = ljcell.lib().lj_exclusive_scan_noalloc(_p(t), (1 << 26) + 1, _p(t), None)
    assert rc == ljcell.LJ_EUNSUPPORTED


def test_noalloc_scan_timeout_path_then_recovers(torch_cuda):
    """With tile 0 withheld every bounded look-back wait gives up (no fault, no hang): the call marks
    its result invalid with offsets[n] = -1.  The next normal call clears the array's status word
    and counter and returns the correct scan."""
    torch = torch_cuda
    import ljcell

    n = 200_003
    stream = torch.cuda.current_stream()
    counts = torch.randint(0, 9, (n,), dtype=torch.int32, device="cuda")
    out = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    rc = ljcell.lib().lj_test_scan_noalloc_withheld_tile(_p(counts), n, _p(out), C.c_void_p(stream.cuda_stream))
    assert rc == ljcell.LJ_OK, ljcell.status_str(rc)
    torch.cuda.synchronize()
    assert int(out[-1]) == -1
    out2 = torch.full((n + 1,), -7, dtype=torch.int32, device="cuda")
    rc = ljcell.lib().lj_exclusive_scan_noalloc(_p(counts), n, _p(out2), C.c_void_p(stream.cuda_stream))
    assert rc == ljcell.LJ_OK, ljcell.status_str(rc)
    torch.cuda.synchronize()
    ref = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    ref[1:] = torch.cumsum(counts.to(torch.int64), 0)
    assert torch.equal(out2.to(torch.int64), ref)
