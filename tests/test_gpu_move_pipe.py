"""The persistent TMA-pipelined kick-drift-rebin kernel (lf2_move_pipe.cu)
against the per-brick kernel and the oracle: identical particles (bit-exact,
compared by id), identical fixed-point deposits, identical max |v|.  Cases
cover partial bricks on the upper periodic boundary (lattice sizes that are
not multiples of 16), bricks with several chunks of particles (clustered
particles), per-particle masses, and repeated steps with brick changes."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import by_id, small_case

pytestmark = pytest.mark.gpu


def _pair(n, cell, off, vel, mass):
    import latfield2_b200 as L
    ids = np.arange(cell.shape[0], dtype=np.int64)
    out = []
    for which in (2, 1):
        ctx = L.Context(n, box=tuple(v / n[0] for v in n), mode=1)
        gm = 0.0 if mass is not None else 1.0 / len(cell)
        ctx.set_particles(cell, off, vel, mass=mass, global_mass=gm, ids=ids)
        ctx.set_move_kernel(which)
        out.append(ctx)
    return out


@pytest.mark.parametrize("n,npart,clustered,with_mass", [
    ((32, 32, 32), 30000, False, False),
    ((48, 40, 36), 50000, False, True),
    ((64, 64, 64), 200000, True, False),
    ((64, 48, 80), 120000, True, True),
])
def test_pipelined_move_equals_per_brick_and_oracle(cuda, n, npart, clustered, with_mass):
    import torch
    cell, off, vel = small_case(n, npart, seed=101, vel_sigma=0.03, clustered=clustered)
    rng = np.random.default_rng(5)
    mass = (1.0 + 0.1 * rng.random(npart)).astype(np.float32) / npart if with_mass else None
    F = rng.standard_normal((3, n[2], n[1], n[0])).astype(np.float32)
    a, b = _pair(n, cell, off, vel, mass)
    Ft = torch.from_numpy(F).cuda()
    Fa, Fb = a.field(3, Ft), b.field(3, Ft)
    ra, rb = a.field(1), b.field(1)
    res = 1.0 / n[0]
    c, o, v = cell.copy(), off.copy(), vel.copy()
    movers = 0
    for _ in range(3):
        a.step(Fa, 0.05, 0.2, ra)
        b.step(Fb, 0.05, 0.2, rb)
        movers += a.rebin_stats()[2]
        v = O.state_kick(n, c, o, v, F, np.float32(0.05))
        c, o, _ = O.state_drift(n, c, o, v, np.float32(0.2 / res))
    assert movers > 0
    assert a.count() == npart and b.count() == npart
    ga = by_id(a.get_particles(mass=with_mass, ids=True))
    gb = by_id(b.get_particles(mass=with_mass, ids=True))
    for k in ("cell", "off", "vel"):
        np.testing.assert_array_equal(ga[k], gb[k])
    if with_mass:
        np.testing.assert_array_equal(ga["mass"], gb["mass"])
        np.testing.assert_array_equal(ga["mass"], mass)
    np.testing.assert_array_equal(ga["id"], np.arange(npart))
    np.testing.assert_array_equal(ga["vel"], v)
    np.testing.assert_array_equal(ga["cell"], c)
    np.testing.assert_array_equal(ga["off"], o)
    np.testing.assert_array_equal(ra.export_internal(), rb.export_internal())
    np.testing.assert_array_equal(a.cell_counts(), np.bincount(c, minlength=int(np.prod(n))))
    # FP64 sums over particles whose order within a brick may differ
    ca, cb = a.conservation(), b.conservation()
    assert ca[0] == pytest.approx(cb[0], rel=1e-12) and ca[2] == cb[2]
    np.testing.assert_allclose(ca[1], cb[1], rtol=1e-9, atol=1e-12 * np.abs(cb[1]).max())
    assert a.flags() & ~0x8 == 0 and b.flags() & ~0x8 == 0


def test_pipelined_move_refuses_unsupported_lattice(cuda):
    import latfield2_b200 as L
    import torch
    n = (24, 24, 24)
    cell, off, vel = small_case(n, 1000, seed=3)
    ctx = L.Context(n, box=1.0, mode=1)
    ctx.set_particles(cell, off, vel, global_mass=1e-3)
    ctx.set_move_kernel(2)
    F = ctx.field(3, torch.zeros(3, 24, 24, 24, device="cuda"))
    with pytest.raises(L.LF2Error):
        ctx.step(F, 0.1, 0.1)
    ctx.set_move_kernel(0)  # automatic: the per-brick kernel serves this lattice
    ctx.step(F, 0.1, 0.1)
    assert ctx.count() == 1000


def test_pipelined_move_long_run_equals_per_brick(cuda):
    """Sixty steps of lf2_step on a log-normal 256^3 case (the statistics of
    the throughput workload, half the particles), pipelined kernel against
    per-brick kernel: identical particles by id, identical fixed-point
    density, clean flags, cell counts that match the particles.  Long runs
    turn the pipelined kernel's chunk and tile buffers over many thousands
    of times and go through brick relocations."""
    import torch
    import latfield2_b200 as L
    import latfield2_b200.workloads as W
    n = (256, 256, 256)
    npart = 256 ** 3 // 2
    cell, off = W.lognormal(n, npart, seed=13, device="cuda")
    vel = W.velocities(npart, 0.02, seed=14, device="cuda")
    F = W.grf_gradient(n, seed=15, device="cuda", amplitude=0.01)
    ids = torch.arange(npart, dtype=torch.int64, device="cuda")
    dtau = 0.1 * 64.0 / 256
    out = []
    for which in (2, 1):
        ctx = L.Context(n, box=1.0, mode=L.DEPOSIT_FIXED64)
        ctx.set_particles(cell, off, vel, global_mass=1.0 / npart, ids=ids)
        ctx.set_move_kernel(which)
        Fh, rho = ctx.field(3, F), ctx.field(1)
        for _ in range(60):
            ctx.step(Fh, dtau, dtau, rho)
        assert ctx.last_move_kernel() == which
        ctx.synchronize()
        assert ctx.flags() & ~0x8 == 0
        p = ctx.get_particles(ids=True)
        k = np.argsort(p["id"])
        counts = ctx.cell_counts()
        np.testing.assert_array_equal(counts, np.bincount(p["cell"], minlength=256 ** 3))
        out.append(({kk: v[k] for kk, v in p.items()}, rho.export_internal(), ctx.rebin_stats()))
        del ctx, Fh, rho
        torch.cuda.empty_cache()
    (a, ra, sa), (b, rb, sb) = out
    np.testing.assert_array_equal(a["id"], np.arange(npart))
    for kk in ("cell", "off", "vel"):
        np.testing.assert_array_equal(a[kk], b[kk])
    np.testing.assert_array_equal(ra, rb)
    assert sa[1] > 0  # bricks were relocated


def test_a_wait_that_runs_out_is_reported_and_the_context_recovers(cuda):
    """The bounded-wait path: with the consumers stalled on a barrier that
    nothing completes and a limit of about 10 us, the pass gives up (the
    producer waits for its copies first), the status is LF2_ERR_STATE with
    LF2_FLAG_TIMEOUT, and after a reload the same context steps bit-exactly
    against the oracle with the default limit."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200 import _lib
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 20000, seed=7, vel_sigma=0.03)
    F = np.random.default_rng(8).standard_normal((3, 32, 32, 32)).astype(np.float32)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    ctx = L.Context(n, box=1.0, mode=1)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / 20000, ids=ids)
    ctx.set_move_kernel(2)
    Fh = ctx.field(3, torch.from_numpy(F).cuda())
    rho = ctx.field(1)
    ctx.set_wait_limit(20000, stall=True)
    ctx.step(Fh, 0.05, 0.2, rho)
    with pytest.raises(_lib.LF2Error) as err:
        ctx.synchronize()
    assert err.value.status == _lib.LF2_ERR_STATE
    assert ctx.flags() & _lib.FLAG_TIMEOUT
    ctx.set_wait_limit(0)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / 20000, ids=ids)
    assert ctx.flags() == 0
    ctx.step(Fh, 0.05, 0.2, rho)
    ctx.synchronize()
    assert ctx.last_move_kernel() == 2
    got = by_id(ctx.get_particles(ids=True))
    v = O.state_kick(n, cell, off, vel, F, np.float32(0.05))
    c, o, _ = O.state_drift(n, cell, off, v, np.float32(0.2 * 32))
    np.testing.assert_array_equal(got["vel"], v)
    np.testing.assert_array_equal(got["cell"], c)
    np.testing.assert_array_equal(got["off"], o)


@pytest.mark.parametrize("n,npart,clustered,with_mass,dtau", [
    ((32, 32, 32), 30000, False, False, 0.2),
    ((48, 40, 36), 50000, False, True, 0.2),
    ((64, 64, 64), 200000, True, False, 0.2),
    ((64, 48, 80), 120000, True, True, 0.2),
    ((32, 32, 32), 30000, False, False, 60.0),  # particles cross several cells: the redo path
])
def test_fused_deposit_equals_the_separate_deposit_and_the_oracle(cuda, n, npart, clustered,
                                                                   with_mass, dtau):
    """lf2_step with the fixed-point deposit fused into the pipelined pass
    (kernel 3) against the pipelined pass followed by the tile deposit
    (kernel 2): the same particles and the same density bits, step after step,
    and the oracle's integer deposit of the oracle's particles."""
    import torch
    cell, off, vel = small_case(n, npart, seed=202, vel_sigma=0.03, clustered=clustered)
    rng = np.random.default_rng(6)
    mass = (1.0 + 0.1 * rng.random(npart)).astype(np.float32) / npart if with_mass else None
    F = rng.standard_normal((3, n[2], n[1], n[0])).astype(np.float32)
    a, b = _pair(n, cell, off, vel, mass)
    a.set_move_kernel(3)
    b.set_move_kernel(2)
    Ft = torch.from_numpy(F).cuda()
    Fa, Fb = a.field(3, Ft), b.field(3, Ft)
    ra, rb = a.field(1), b.field(1)
    res = 1.0 / n[0]
    c, o, v = cell.copy(), off.copy(), vel.copy()
    for _ in range(3):
        a.step(Fa, 0.05, dtau, ra)
        b.step(Fb, 0.05, dtau, rb)
        assert a.last_move_kernel() == 3 and b.last_move_kernel() == 2
        v = O.state_kick(n, c, o, v, F, np.float32(0.05))
        c, o, _ = O.state_drift(n, c, o, v, np.float32(dtau / res))
        np.testing.assert_array_equal(ra.export_internal(), rb.export_internal())
    a.synchronize()
    b.synchronize()
    ga = by_id(a.get_particles(ids=True))
    np.testing.assert_array_equal(ga["cell"], c)
    np.testing.assert_array_equal(ga["off"], o)
    np.testing.assert_array_equal(ga["vel"], v)
    unit = 1.0 / npart
    mrel = None
    if with_mass:
        unit = float(np.sum(mass.astype(np.float64)) / npart)
        mrel = (mass * np.float32(1.0 / unit)).astype(np.float32)
    exact = O.fixed_to_f32(O.state_deposit_fixed(n, c, o, mrel),
                           np.float32(2.0 ** -32 * unit / res ** 3))
    np.testing.assert_array_equal(ra.export_internal().reshape(-1), exact)
