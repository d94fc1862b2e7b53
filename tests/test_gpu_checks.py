"""GPU: the bounds-checked debug build (libljcell_checks.so, compiled with -DLJ_CHECKS and loaded when
LJCELL_CHECKS=1).  After each binning stage it checks what the next stage relies on -- counts
non-negative and matching the offsets, every ticket inside its cell, every sorted record inside its
cell's range and in order, the sorted order a permutation -- and lj_sync reports a violation as
LJ_ECHECK.  A child process runs the parity cases (both within-cell orders, a cell beyond the warp
sort, points outside the box), a batched step and time steps through the checked library: no check
fires, and binning and pair outputs carry the bits of the normal build.  A scan of counts with a
negative entry, an input the scan itself does not reject, is reported as LJ_ECHECK by the checked
build and passes unremarked through the normal one."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from test_gpu_parity import case_positions, dev, np_

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "particle-interaction-with-optix_b200")
CASES = [("uniform_c1", 1), ("uniform_c1", 0), ("clustered", 1), ("shell", 1), ("outside_and_faces", 1),
         ("tiny1", 1)]

CHILD = r"""
import json, os, sys
import numpy as np
sys.path[:0] = [os.environ["LJ_TEST_DIR"], os.environ["LJ_PKG"], os.path.join(os.environ["LJ_ROOT"], "oracle")]
import torch
import ljcell
from test_gpu_parity import case_positions, dev, np_
assert ljcell.LIB_PATH.endswith("libljcell_checks.so"), ljcell.LIB_PATH
out = {}
ctx = ljcell.Context(0)
for name, order in json.loads(os.environ["LJ_CASES"]):
    (x, y, z), (lo, hi), rc = case_positions(name)
    g = ljcell.grid_from_box(lo, hi, rc)
    p = ljcell.params(rc, sigma=rc / 500 if name == "clustered" else None)
    b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=order)
    e, f, t = ctx.compute(g, p, b)
    ctx.sync()                                    # raises LJError(LJ_ECHECK) if a check fired
    n = len(x)
    np.savez(os.path.join(os.environ["LJ_OUT"], f"{name}_{order}.npz"), offsets=np_(b.offsets),
             xyzi=np_(b.xyzi)[:n], cell=np_(b.cell)[:n], e=np_(e)[:n], f=np_(f)[:n])
# batched binning (one cell numbering over several systems)
w = ljcell.batch_workload(nsys=8, seed=3, n_min=100, n_max=3000, nb_min=15, nb_max=40)
bt = ljcell.Batch(ctx, w)
xyz = bt.generate()
bt.run(*xyz)
ctx.sync()
bt.close()
# time steps rebin from the previous order
(x, y, z), (lo, hi), rc = case_positions("uniform_dense")
g = ljcell.grid_from_box(lo, hi, rc)
p = ljcell.params(rc)
b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=1)
n = len(x)
force = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
vel = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
ctx.compute(g, p, b, force=force)
for _ in range(3):
    ctx.step_verlet(g, p, b, vel, force, 1e-9)
ctx.sync()
# a negative count: the scan runs, the check reports it
counts = torch.tensor([3, -1, 2, 0], dtype=torch.int32, device="cuda")
offs = ctx.exclusive_scan(counts)
try:
    ctx.sync()
    out["negative_count"] = "ok"
except ljcell.LJError as err:
    out["negative_count"] = int(err.status)
# the status word is cleared: the next clean call passes
ctx.exclusive_scan(torch.tensor([1, 2, 3], dtype=torch.int32, device="cuda"))
ctx.sync()
out["after"] = "ok"
print(json.dumps(out))
"""


def test_checked_build_passes_and_matches(torch_cuda, ctx, tmp_path):
    import ljcell

    torch = torch_cuda
    lib = os.path.join(PKG, "ljcell", "libljcell_checks.so")
    assert os.path.exists(lib), "the bounds-checked library is built by make (target libljcell_checks.so)"
    env = dict(os.environ, LJCELL_CHECKS="1", LJ_TEST_DIR=os.path.dirname(os.path.abspath(__file__)), LJ_PKG=PKG,
               LJ_ROOT=ROOT, LJ_OUT=str(tmp_path), LJ_CASES=json.dumps(CASES))
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["negative_count"] == ljcell.LJ_ECHECK, res
    assert res["after"] == "ok"
    # the same cases through the normal build, in this process: the same bits
    for name, order in CASES:
        (x, y, z), (lo, hi), rc = case_positions(name)
        g = ljcell.grid_from_box(lo, hi, rc)
        p = ljcell.params(rc, sigma=rc / 500 if name == "clustered" else None)
        b = ctx.bin(g, dev(torch, x), dev(torch, y), dev(torch, z), order=order)
        e, f, t = ctx.compute(g, p, b)
        ctx.sync()
        n = len(x)
        got = np.load(tmp_path / f"{name}_{order}.npz")
        assert np.array_equal(got["offsets"], np_(b.offsets)), name
        assert np.array_equal(got["xyzi"].view(np.uint32), np_(b.xyzi)[:n].view(np.uint32)), name
        assert np.array_equal(got["cell"], np_(b.cell)[:n]), name
        assert np.array_equal(got["e"].view(np.uint32), np_(e)[:n].view(np.uint32)), name
        assert np.array_equal(got["f"].view(np.uint32), np_(f)[:n].view(np.uint32)), name


def test_normal_build_does_not_check(torch_cuda, ctx):
    """The product library runs no consistency checks: the same negative count scans without remark."""
    torch = torch_cuda
    counts = torch.tensor([3, -1, 2, 0], dtype=torch.int32, device="cuda")
    offs = ctx.exclusive_scan(counts)
    ctx.sync()
    assert np_(offs).tolist() == [0, 3, 2, 4, 4]
