"""Velocity-Verlet time step with rebinning (lj_step_verlet).  One step is
checked against the oracle's single-precision restatement of the drift
(positions and the carried ids and half-kicked velocities bit-exact, the new
sorted order bit-exact against the oracle's binning of the moved positions),
the new forces against the FP64 oracle within the plain form's tolerance, and
the closing half kick bit-exact given those forces.  Many steps are checked
through a size-independent property: the energy of the truncated law,
shifted by the cutoff jump of every interacting pair, stays constant."""
import numpy as np
import pytest

import ljoracle as O

FORCE_NORMWISE_TOL = 1e-5


def lattice(side: int, jitter: float, seed: int):
    """Jittered cubic lattice in [0, 1)^3 with spacing 1 / side, float32."""
    rng = np.random.default_rng(seed)
    a = 1.0 / side
    g = (np.arange(side) + 0.5) * a
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    p += rng.uniform(-jitter * a, jitter * a, p.shape)
    return p.astype(np.float32), a


def setup(torch, ctx, side=20, seed=5):
    import ljcell

    p, a = lattice(side, 0.05, seed)
    sigma = a / 1.12
    rc = 2.5 * sigma
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    prm = ljcell.params(rc, sigma=sigma)
    d = [torch.from_numpy(p[:, i].copy()).cuda() for i in range(3)]
    b = ctx.bin(g, *d, order=ljcell.ORDER_X)
    e, f, tot = ctx.compute(g, prm, b)
    rng = np.random.default_rng(seed + 1)
    v = (rng.standard_normal(p.shape) * 0.5).astype(np.float32)   # in original order
    perm = b.xyzi.cpu().numpy()[:len(p), 3].copy().view(np.int32)
    vel = torch.from_numpy(v[perm].copy()).cuda()
    ctx.sync()
    return g, prm, b, vel, f, e, tot, sigma, rc


def test_oracle_drift_is_single_precision_mul_then_add():
    x = np.array([[0.1, 0.2, 0.3]], np.float32)
    v = np.array([[1.0, -2.0, 0.5]], np.float32)
    f = np.array([[3.0, 0.0, -1.0]], np.float32)
    x2, v2, h = O.verlet_drift(x, v, f, 1e-3, 2.0)
    assert h == np.float32(np.float32(0.5) * np.float32(1e-3) / np.float32(2.0))
    assert v2[0, 0] == np.float32(np.float32(1.0) + np.float32(h * np.float32(3.0)))
    assert x2[0, 2] == np.float32(np.float32(0.3) + np.float32(np.float32(1e-3) * v2[0, 2]))


def test_step_verlet_rejects_bad_arguments():
    import ljcell

    assert ljcell.lib().lj_step_verlet(None, None, None, 0, 1.0, 1.0, None, None, None, None, None, None, None,
                                       None) == 1  # LJ_EINVAL


@pytest.mark.gpu
def test_step_verlet_one_step_against_oracle(torch_cuda, ctx):
    import ljcell

    torch = torch_cuda
    g, prm, b, vel, f, e, tot, sigma, rc = setup(torch, ctx)
    n = b.n
    dt, mass = 2e-4, 1.0
    rec0 = b.xyzi.cpu().numpy()[:n].copy()
    v0 = vel.cpu().numpy().copy()
    f0 = f.cpu().numpy()[:n].copy()
    ctx.step_verlet(g, prm, b, vel, f, dt, mass, e, tot)
    ctx.sync()
    # drift: the oracle's restatement in the old sorted order, then the oracle's binning of it
    x2, vh, h = O.verlet_drift(rec0[:, :3], v0, f0, dt, mass)
    og = O.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    ob = O.bin_particles(og, x2[:, 0].copy(), x2[:, 1].copy(), x2[:, 2].copy(), O.ORDER_X)
    rec1 = b.xyzi.cpu().numpy()[:n]
    np.testing.assert_array_equal(b.offsets.cpu().numpy(), ob.offsets)
    np.testing.assert_array_equal(rec1[:, :3], x2[ob.perm])
    ids0 = rec0[:, 3].copy().view(np.int32)
    np.testing.assert_array_equal(rec1[:, 3].copy().view(np.int32), ids0[ob.perm])
    # new forces against FP64, then the closing half kick bit-exact given them
    ref = O.config_forces(og, ob, rc, 1.0, sigma)
    f1 = f.cpu().numpy()[:n]
    fe = ref.force_errors(f1)
    assert fe["normwise"] <= FORCE_NORMWISE_TOL, fe
    assert ljcell.totals_from_tensor(tot)["pairs"] == ref.pairs
    v1 = vel.cpu().numpy()
    np.testing.assert_array_equal(v1, (vh[ob.perm] + h * f1).astype(np.float32))


@pytest.mark.gpu
def test_step_verlet_conserves_energy(torch_cuda, ctx):
    import ljcell

    torch = torch_cuda
    g, prm, b, vel, f, e, tot, sigma, rc = setup(torch, ctx, side=24, seed=9)
    mass, dt = 1.0, 2e-5

    # The law is truncated without a shift: a pair crossing the cutoff changes the potential energy by
    # V(rc) with no force impulse, so the conserved quantity is KE + PE - (interacting pairs) V(rc).
    s6 = (sigma / rc) ** 6
    v_rc = 4.0 * (s6 * s6 - s6)

    def total_energy():
        ctx.sync()
        ke = 0.5 * mass * float((vel.double() ** 2).sum())
        t = ljcell.totals_from_tensor(tot)
        return ke + t["energy"] - 0.5 * t["pairs"] * v_rc, ke

    e0, ke0 = total_energy()
    assert ke0 > 0
    for _ in range(100):
        ctx.step_verlet(g, prm, b, vel, f, dt, mass, e, tot)
    e1, ke1 = total_energy()
    assert ke1 != ke0                       # the particles moved
    assert abs(e1 - e0) <= 1e-3 * abs(ke0), (e0, e1, ke0)
