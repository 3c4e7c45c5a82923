"""GPU checks of the hand-written adjoint kernels and of the differentiable
multi-step chain (latfield2_b200.autodiff.PMChain) against the FP64
restatement in oracle/pm_chain.py (torch autograd in float64) and against
FP64 central finite differences along random directions.

Tolerances: single adjoint kernels 2e-5 of the gradient's norm; the 8-step
chain 2e-3 of each gradient's norm (FP32 particle state through 8 steps);
directional derivatives within 5e-3 of the rms directional derivative."""
import numpy as np
import pytest

from oracle import pm_chain as P

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.double().reshape(-1)
    b = b.double().reshape(-1)
    return float((a - b).norm() / max(float(b.norm()), 1e-300))


def _case(n, npart, seed, device):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    pos = torch.rand(npart, 3, generator=g, dtype=torch.float64)
    vel = 0.02 * torch.randn(npart, 3, generator=g, dtype=torch.float64)
    m = (1.0 + 0.1 * (2 * torch.rand(npart, generator=g, dtype=torch.float64) - 1)) / npart
    S = 0.02 * torch.randn(81, generator=g, dtype=torch.float64)
    w = torch.randn(n ** 3, generator=g, dtype=torch.float64)
    return [t.to(device) for t in (pos, vel, m, S, w)]


def _state(pos, n):
    from latfield2_b200.autodiff import positions_to_state
    return positions_to_state(pos, (n, n, n), 1.0 / n)


def test_single_adjoint_kernels(cuda):
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import _Ops
    n, npart = 24, 5000
    pos, vel, m, S, w = _case(n, npart, 1, "cuda")
    ctx = L.Context((n, n, n), box=1.0)
    ops = _Ops(ctx)
    cell, off = _state(pos, n)
    # the FP64 positions the device sees
    posd = ((torch.stack([cell.long() % n, (cell.long() // n) % n, cell.long() // (n * n)], 1)
             .double() + off.double()) / n)
    m32 = m.float().contiguous()
    nn = (n, n, n)
    # deposit adjoint
    g_rho = torch.randn(n ** 3, dtype=torch.float64, device="cuda")
    x = posd.clone().requires_grad_(True)
    mm = m32.double().clone().requires_grad_(True)
    (P.deposit(x, mm, nn) * g_rho).sum().backward()
    g_off = torch.zeros(npart, 3, device="cuda")
    g_m = torch.zeros(npart, device="cuda")
    ops.deposit_adj(cell, off, m32, g_rho.float().contiguous(), g_off, g_m)
    assert _rel(g_off * n, x.grad) < 2e-5
    assert _rel(g_m, mm.grad) < 2e-5
    # gather adjoint
    F = torch.randn(3, n ** 3, dtype=torch.float64, device="cuda")
    gG = torch.randn(npart, 3, dtype=torch.float64, device="cuda")
    x = posd.clone().requires_grad_(True)
    Fr = F.clone().requires_grad_(True)
    (P.gather(x, Fr, nn) * gG).sum().backward()
    F4 = torch.zeros(n ** 3, 4, device="cuda")
    F4[:, :3] = F.float().t()
    g_F4 = torch.zeros(n ** 3, 4, device="cuda")
    g_off = torch.zeros(npart, 3, device="cuda")
    ops.gather_adj(cell, off, F4, gG.float().contiguous(), g_F4, g_off)
    assert _rel(g_off * n, x.grad) < 2e-5
    assert _rel(g_F4[:, :3].t(), Fr.grad) < 2e-5
    assert float(g_F4[:, 3].abs().max()) == 0.0
    # gather and deposit forward
    G = torch.empty(npart, 3, device="cuda")
    ops.gather(cell, off, F4, G)
    assert _rel(G, P.gather(posd, F, nn)) < 2e-6
    rho = torch.zeros(n ** 3, device="cuda")
    ops.deposit(cell, off, m32, rho)
    assert _rel(rho, P.deposit(posd, m32.double(), nn)) < 2e-6
    # stencil and its adjoint
    r = torch.randn(n ** 3, dtype=torch.float64, device="cuda")
    F32 = torch.empty(n ** 3, 4, device="cuda")
    ops.stencil(r.float().contiguous(), S.float().contiguous(), F32)
    assert _rel(F32[:, :3].t(), P.stencil(r, S, nn)) < 2e-6
    gF = torch.randn(3, n ** 3, dtype=torch.float64, device="cuda")
    rr = r.clone().requires_grad_(True)
    Sr = S.clone().requires_grad_(True)
    (P.stencil(rr, Sr, nn) * gF).sum().backward()
    g_r = torch.zeros(n ** 3, device="cuda")
    g_S = torch.zeros(81, device="cuda")
    gF4 = torch.zeros(n ** 3, 4, device="cuda")
    gF4[:, :3] = gF.float().t()
    ops.stencil_adj(r.float().contiguous(), S.float().contiguous(), gF4, g_r, g_S)
    assert _rel(g_r, rr.grad) < 2e-5
    assert _rel(g_S, Sr.grad) < 2e-5


@pytest.mark.parametrize("n,npart,ndir", [(32, 20000, 1000)])
def test_chain_gradients_against_fp64(cuda, n, npart, ndir):
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import pm_chain_loss
    steps, dt = 8, 0.1
    pos, vel, m, S, w = _case(n, npart, 7, "cuda")
    # FP64 chain on the positions the device represents (FP32 offsets)
    cell, off = _state(pos, n)
    posd = ((torch.stack([cell.long() % n, (cell.long() // n) % n, cell.long() // (n * n)], 1)
             .double() + off.double()) / n)
    vel = vel.float().double()
    m = m.float().double()
    S = S.float().double()
    w = w.float().double()
    ctx = L.Context((n, n, n), box=1.0)
    leaves = [t.clone().requires_grad_(True) for t in (posd, vel, m, S, w)]
    loss = pm_chain_loss(ctx, *leaves, steps=steps, dt=dt, checkpoint_every=2)
    loss.backward()
    got = [t.grad for t in leaves]
    ref_leaves = [t.clone().requires_grad_(True) for t in (posd, vel, m, S, w)]
    ref_loss = P.chain_loss(*ref_leaves, (n, n, n), steps, dt)
    ref = torch.autograd.grad(ref_loss, ref_leaves)
    assert float(loss.detach()) == pytest.approx(float(ref_loss.detach()), rel=2e-4)
    for name, a, b in zip(("pos", "vel", "mass", "stencil", "weights"), got, ref):
        assert _rel(a, b) < 2e-3, name
    # FP64 central differences of the FP64 chain along random directions
    rng = np.random.default_rng(11)
    base = [posd, vel, m, S]
    fd, an_dev, an_ref = [], [], []
    for _ in range(ndir):
        us = [torch.from_numpy(rng.standard_normal(tuple(t.shape))).to("cuda") for t in base]
        nrm = float(torch.sqrt(sum((u ** 2).sum() for u in us)))
        us = [u / nrm for u in us]
        with torch.no_grad():
            d, _ = P.directional_fd(base, us, w, (n, n, n), steps, dt, eps=1e-7)
        assert d is not None  # an eps without face crossings exists
        fd.append(d)
        an_dev.append(float(sum((g * u).sum() for g, u in zip(got[:4], us))))
        an_ref.append(float(sum((g * u).sum() for g, u in zip(ref[:4], us))))
    fd, an_dev, an_ref = map(np.array, (fd, an_dev, an_ref))
    scale = np.sqrt(np.mean(fd ** 2))
    assert np.max(np.abs(an_ref - fd)) < 1e-5 * scale  # the FP64 reference gradient
    assert np.max(np.abs(an_dev - fd)) < 5e-3 * scale  # the CUDA adjoint


COUPLING = 4 * np.pi  # lap phi = 4 pi G rho with G = 1


def test_pm_force4_and_its_adjoint(cuda):
    """lf2_pm_force4 against the FP64 PM force, and lf2_pm_force4_adjoint
    against its autograd gradient (2e-5 of the norm)."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import _Ops
    for n in (24, 32):
        ctx = L.Context((n, n, n), box=1.0)
        ops = _Ops(ctx)
        g = torch.Generator(device="cpu").manual_seed(n)
        rho = (1.0 + torch.randn(n ** 3, generator=g, dtype=torch.float64)).to("cuda")
        F4 = torch.full((n ** 3, 4), 7.0, device="cuda")
        ops.pm_force(rho.float().contiguous(), F4, COUPLING)
        ref = P.pm_force(rho, (n, n, n), COUPLING)
        assert _rel(F4[:, :3].t(), ref) < 2e-5
        assert float(F4[:, 3].abs().max()) == 0.0
        gF = torch.randn(3, n ** 3, generator=g, dtype=torch.float64).to("cuda")
        r = rho.clone().requires_grad_(True)
        (P.pm_force(r, (n, n, n), COUPLING) * gF).sum().backward()
        gF4 = torch.zeros(n ** 3, 4, device="cuda")
        gF4[:, :3] = gF.float().t()
        gF4[:, 3] = 5.0  # not read
        g_rho = torch.ones(n ** 3, device="cuda")
        ops.pm_force_adj(gF4, g_rho, COUPLING)
        assert _rel(g_rho - 1.0, r.grad) < 2e-5  # accumulated
        ctx.close()


def test_pm_chain_gradients_against_fp64(cuda):
    """The 8-step chain with the PM force as grid operator: gradients for
    positions, velocities, masses and loss weights against the FP64 chain
    (2e-3 of each norm) and central differences along 200 random
    directions (5e-3 of their rms)."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import pm_chain_loss
    n, npart, ndir, steps, dt = 32, 20000, 200, 8, 0.1
    pos, vel, m, S, w = _case(n, npart, 9, "cuda")
    cell, off = _state(pos, n)
    posd = ((torch.stack([cell.long() % n, (cell.long() // n) % n, cell.long() // (n * n)], 1)
             .double() + off.double()) / n)
    vel, m, w = vel.float().double(), m.float().double(), w.float().double()
    ctx = L.Context((n, n, n), box=1.0)
    leaves = [t.clone().requires_grad_(True) for t in (posd, vel, m, w)]
    loss = pm_chain_loss(ctx, leaves[0], leaves[1], leaves[2], None, leaves[3], steps=steps,
                         dt=dt, checkpoint_every=2, operator="pm", coupling=COUPLING)
    loss.backward()
    got = [t.grad for t in leaves]
    ref_leaves = [t.clone().requires_grad_(True) for t in (posd, vel, m, w)]
    ref_loss = P.chain_loss(ref_leaves[0], ref_leaves[1], ref_leaves[2], None, ref_leaves[3],
                            (n, n, n), steps, dt, coupling=COUPLING)
    ref = torch.autograd.grad(ref_loss, ref_leaves)
    assert float(loss.detach()) == pytest.approx(float(ref_loss.detach()), rel=2e-4)
    for name, a, b in zip(("pos", "vel", "mass", "weights"), got, ref):
        assert _rel(a, b) < 2e-3, name
    rng = np.random.default_rng(12)
    base = [posd, vel, m]
    fd, an_dev, an_ref = [], [], []
    for _ in range(ndir):
        us = [torch.from_numpy(rng.standard_normal(tuple(t.shape))).to("cuda") for t in base]
        nrm = float(torch.sqrt(sum((u ** 2).sum() for u in us)))
        us = [u / nrm for u in us]
        with torch.no_grad():
            d, _ = P.directional_fd(base + [None], us + [None], w, (n, n, n), steps, dt,
                                    eps=1e-7, coupling=COUPLING)
        assert d is not None
        fd.append(d)
        an_dev.append(float(sum((g * u).sum() for g, u in zip(got[:3], us))))
        an_ref.append(float(sum((g * u).sum() for g, u in zip(ref[:3], us))))
    fd, an_dev, an_ref = map(np.array, (fd, an_dev, an_ref))
    scale = np.sqrt(np.mean(fd ** 2))
    assert np.max(np.abs(an_ref - fd)) < 1e-5 * scale
    assert np.max(np.abs(an_dev - fd)) < 5e-3 * scale
    ctx.close()


@pytest.mark.parametrize("masses", [False, True])
def test_fixed_point_chain_deposit(cuda, masses):
    """The chain's deposit in a context of the fixed-point mode: integer sums
    of the library's corner weights (times the mass relative to the call's
    largest mass), so the density is the same bits in any particle order and
    within 1e-6 of the FP64 deposit; the 8-step chain's gradients match the
    FP64 gradient as the FP32-mode chain's do (the adjoint kernels are
    shared)."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import _Ops, pm_chain_loss
    from tests.helpers import precision
    n, npart = 32, 60000
    pos, vel, m, S, w = _case(n, npart, 5, "cuda")
    # a clump on top of the uniform particles: dense vertices
    pos[: npart // 3] = (0.5 + 0.02 * torch.randn(npart // 3, 3, dtype=torch.float64,
                                                  device="cuda")) % 1.0
    ctx = L.Context((n, n, n), box=1.0, mode=L.DEPOSIT_FIXED64)
    ops = _Ops(ctx)
    cell, off = _state(pos, n)
    m32 = m.float().contiguous()
    gm = 1.0 / npart
    posd = ((torch.stack([cell.long() % n, (cell.long() // n) % n, cell.long() // (n * n)], 1)
             .double() + off.double()) / n)
    mass = m32.double() if masses else torch.full((npart,), gm, dtype=torch.float64, device="cuda")
    ref = P.deposit(posd, mass, (n, n, n)).cpu().numpy()
    outs = []
    for perm in (torch.arange(npart, device="cuda"), torch.randperm(npart, device="cuda")):
        rho = torch.zeros(n ** 3, dtype=torch.float32, device="cuda")
        if masses:
            ops.deposit(cell[perm].contiguous(), off[perm].contiguous(), m32[perm].contiguous(), rho)
        else:
            rc = ops.lib.lf2_pm_deposit(ctx.h, npart, ops_ptr(cell[perm].contiguous()),
                                        ops_ptr(off[perm].contiguous()), None, gm, ops_ptr(rho))
            assert rc == 0
        torch.cuda.synchronize()
        outs.append(rho.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])  # order-free integer sums
    p = precision(outs[0], ref)
    assert p["norm_max"] <= 1e-6 and p["cell_max"] <= 1e-6, p
    ctx.synchronize()
    ctx.close()
    # the 8-step chain with the fixed-point deposits against the FP64 gradient
    # (uniform particles, the tolerance of the FP32-mode chain's test)
    n, npart = 32, 20000
    pos, vel, m, S, w = _case(n, npart, 7, "cuda")
    cell, off = _state(pos, n)
    posd = ((torch.stack([cell.long() % n, (cell.long() // n) % n, cell.long() // (n * n)], 1)
             .double() + off.double()) / n)
    vel, m, S, w = vel.float().double(), m.float().double(), S.float().double(), w.float().double()
    ctx = L.Context((n, n, n), box=1.0, mode=L.DEPOSIT_FIXED64)
    leaves = [t.clone().requires_grad_(True) for t in (posd, vel, m, S, w)]
    pm_chain_loss(ctx, *leaves, steps=8, dt=0.1, checkpoint_every=2).backward()
    ref_leaves = [t.clone().requires_grad_(True) for t in (posd, vel, m, S, w)]
    ref = torch.autograd.grad(P.chain_loss(*ref_leaves, (n, n, n), 8, 0.1), ref_leaves)
    for name, a, b in zip(("pos", "vel", "mass", "stencil", "weights"), leaves, ref):
        assert _rel(a.grad, b) < 2e-3, name
    ctx.close()


def ops_ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("n", [48, 64])
def test_chain_state_kernels_match_the_torch_restatement(cuda, n):
    """lf2_pm_state_pack / lf2_pm_state_unpack / lf2_pm_grads_unorder (the
    chain's particle state and its gradients' way back) bit for bit against
    the torch expressions they replace: positions_to_state, the permutation
    by order, and the scatter of the FP64 gradients; the sort key (brick,
    then cell in the brick).  Positions include cell faces, the box's faces
    and periodic images outside [0, 1)."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import _Ops
    npart = 20000
    g = torch.Generator(device="cpu").manual_seed(5)
    pos = torch.rand(npart, 3, generator=g, dtype=torch.float64) * 3.0 - 1.0
    pos[:500] = torch.randint(-n, 2 * n, (500, 3), generator=g).double() / n  # cell faces
    pos[500:600] = torch.nextafter(pos[500:600], torch.full_like(pos[500:600], -10.0))
    vel = torch.randn(npart, 3, generator=g, dtype=torch.float64)
    m = torch.rand(npart, generator=g, dtype=torch.float64) + 0.5
    pos, vel, m = pos.cuda(), vel.cuda(), m.cuda()
    res = 1.0 / n
    ctx = L.Context((n, n, n), box=1.0)
    ops = _Ops(ctx)
    cell_t, off_t = _state(pos, n)
    key, rec = ops.state_pack(pos, vel, m, 1.0 / res)
    c = cell_t.long()
    x, y, z = c % n, (c // n) % n, c // (n * n)
    nb = -(-n // 16)
    want_key = (((x // 16) + nb * ((y // 16) + nb * (z // 16))) * 4096 + x % 16
                + 16 * (y % 16 + 16 * (z % 16)))
    assert torch.equal(key.long(), want_key)
    order = torch.argsort(key)
    cell, off, vel32, m32 = ops.state_unpack(order, rec)
    assert torch.equal(cell, cell_t[order])
    assert torch.equal(off, off_t[order])
    assert torch.equal(vel32, vel.float()[order])
    assert torch.equal(m32, m.float()[order])
    g_off = torch.randn(npart, 3, generator=g).cuda()
    g_v = torch.randn(npart, 3, generator=g).cuda()
    g_m = torch.randn(npart, generator=g).cuda()
    g_pos, g_vel, g_mass = ops.grads_unorder(order, g_off, g_v, g_m, 1.0 / res)
    want = torch.empty(npart, 3, dtype=torch.float64, device="cuda")
    want[order] = g_off.to(torch.float64) / res
    assert torch.equal(g_pos, want)
    want = torch.empty(npart, 3, dtype=torch.float64, device="cuda")
    want[order] = g_v.to(torch.float64)
    assert torch.equal(g_vel, want)
    want = torch.empty(npart, dtype=torch.float64, device="cuda")
    want[order] = g_m.to(torch.float64)
    assert torch.equal(g_mass, want)


@pytest.mark.parametrize("mode", ["fixed", "fp32"])
def test_brick_tiled_chain_deposit_matches_the_per_particle_one(cuda, mode):
    """lf2_pm_deposit_bricks (particles grouped by brick, brick_start from
    lf2_pm_brick_start) against lf2_pm_deposit on the same particles: the
    same sums in the fixed-point mode, within 1e-5 of the maximum in the FP32
    mode (FP32 atomics in two orders); again after a drift has moved
    particles out of their groups' bricks."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import _Ops
    n, npart = 40, 300000
    g = torch.Generator(device="cpu").manual_seed(9)
    pos = (0.5 + 0.15 * torch.randn(npart, 3, generator=g, dtype=torch.float64)) % 1.0
    vel = torch.randn(npart, 3, generator=g, dtype=torch.float64)
    m = (torch.rand(npart, generator=g, dtype=torch.float64) + 0.5) / npart
    pos, vel, m = pos.cuda(), vel.cuda(), m.cuda()
    ctx = L.Context((n, n, n), box=1.0, mode=L.DEPOSIT_FIXED64 if mode == "fixed" else L.DEPOSIT_FP32)
    ops = _Ops(ctx)
    key, rec = ops.state_pack(pos, vel, m, float(n))
    order = torch.argsort(key)
    cell, off, vel32, m32 = ops.state_unpack(order, rec)
    bs = ops.brick_start(cell)
    c = cell.long()
    nb = -(-n // 16)
    brick = (c % n) // 16 + nb * (((c // n) % n) // 16 + nb * ((c // (n * n)) // 16))
    assert torch.equal(bs, torch.searchsorted(brick, torch.arange(nb ** 3 + 1, device="cuda")))
    for drift in (0.0, 0.4 / n):
        if drift:
            ops.kick_drift(cell, off, vel32, None, drift)
            c = cell.long()
            now = (c % n) // 16 + nb * (((c // n) % n) // 16 + nb * ((c // (n * n)) // 16))
            assert int((now != brick).sum()) > 1000  # strays
        a = torch.zeros(n ** 3, dtype=torch.float32, device="cuda")
        b = torch.zeros(n ** 3, dtype=torch.float32, device="cuda")
        ops.bricks = None
        ops.deposit(cell, off, m32, a)
        ops.bricks = bs
        ops.deposit(cell, off, m32, b)
        if mode == "fixed":
            assert torch.equal(a, b)
        else:
            assert float((a - b).abs().max()) <= 1e-5 * float(a.abs().max())
        total = float(m32.double().sum())
        assert abs(float(b.double().sum()) / n ** 3 - total) <= 1e-5 * total


def test_fused_chain_step_equals_gather_then_kick_drift(cuda):
    """lf2_pm_step (gather, kick and drift in one pass) gives the cells,
    offsets and velocities of lf2_pm_gather followed by lf2_pm_kick_drift
    bit for bit, face crossings and the periodic wrap included."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import _Ops
    n, npart = 24, 50000
    pos, vel, m, S, w = _case(n, npart, 21, "cuda")
    ctx = L.Context((n, n, n), box=1.0)
    ops = _Ops(ctx)
    cell, off = _state(pos, n)
    v = (vel * 20).float().contiguous()
    F4 = torch.randn(4 * n ** 3, generator=torch.Generator(device="cpu").manual_seed(3)).cuda()
    a = (cell.clone(), off.clone(), v.clone())
    b = (cell.clone(), off.clone(), v.clone())
    G = torch.empty_like(v)
    ops.gather(a[0], a[1], F4, G)
    ops.kick_drift(a[0], a[1], a[2], G, 0.05)
    ops.step(b[0], b[1], b[2], F4, 0.05)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    assert int((a[0] != cell).sum()) > 1000
