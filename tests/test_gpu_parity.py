"""GPU parity of the CUDA path (called through the C ABI) against the CPU
oracle.

Tolerances
  - fixed-point scalar deposit: bit-exact against the oracle's restatement of
    the integer arithmetic; within 1e-6 (normalized) of the FP64 reference.
  - FP32-mode deposits (compensated shared atomics): within 1e-6 of the FP64
    reference, normalized by the field's maximum (|got-ref|max / |ref|max).
    The plain FP32 mode (unordered atomics, no compensation) is held to 1e-5
    in tests/test_gpu_precision.py, which covers every projection in every
    mode.
  - kick, drift, rebin: bit-exact against the oracle's FP32 restatement;
    within 2e-6 (velocity) / 1e-6 res (position) of the FP64 reference.
  - cell assignment and particle counts per cell: exact.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import (by_id, internal_to_reference, mean_relative_error, normalized_error,
                           positions, small_case)

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8, 8), (16, 16, 16), (20, 20, 20), (33, 17, 24), (48, 48, 48)]


def _ctx(n, mode=0):
    import latfield2_b200 as L
    box = tuple(v / n[0] for v in n)
    return L.Context(n, box=box, mode=mode)


def _load(ctx, cell, off, vel, gm, mass=None):
    ids = np.arange(cell.shape[0], dtype=np.int64)
    ctx.set_particles(cell, off, vel, mass=mass, global_mass=0.0 if mass is not None else gm,
                      ids=ids)


def fixed_scale(unit_mass, res):
    """FP32 scale of the fixed-point accumulator, formed as the device does."""
    return np.float32(2.0 ** -32 * unit_mass / (res * res * res))


def _ref_lists(n, res, cell, off, vel, mass=None):
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    v = vel.astype(np.float64)[order]
    pm = None if mass is None else mass.astype(np.float64)[order]
    return cs, pos, v, pm


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("clustered", [False, True])
def test_scalar_deposit_fp32(cuda, n, clustered):
    cell, off, vel = small_case(n, 6000, seed=1, clustered=clustered)
    res = 1.0 / n[0]
    gm = 1.0 / 6000
    ctx = _ctx(n, 0)
    _load(ctx, cell, off, vel, gm)
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    got = rho.export_internal()[0]
    cs, pos, v, _ = _ref_lists(n, res, cell, off, vel)
    ref = O.interior(O.scalar_cic(n, 1, res, cs, pos, None, gm), n, 1)[0]
    assert normalized_error(got, ref) < 1e-6
    assert np.sum(got, dtype=np.float64) * res ** 3 == pytest.approx(1.0, rel=1e-6)


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("clustered", [False, True])
def test_scalar_deposit_fixed_is_bit_exact(cuda, n, clustered):
    cell, off, vel = small_case(n, 6000, seed=2, clustered=clustered)
    res = 1.0 / n[0]
    gm = 1.0 / 6000
    ctx = _ctx(n, 1)
    _load(ctx, cell, off, vel, gm)
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    got = rho.export_internal()[0].reshape(-1)
    exact = O.fixed_to_f32(O.state_deposit_fixed(n, cell, off), fixed_scale(gm, res))
    np.testing.assert_array_equal(got, exact)
    ref = O.state_deposit_f64(n, cell, off, res, gmass=gm)
    assert normalized_error(got, ref) < 1e-6
    assert ctx.flags() == 0


def test_fixed_deposit_is_independent_of_input_order(cuda):
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 40000, seed=9, clustered=True)
    gm = 1.0 / 40000
    outs = []
    for perm_seed in (0, 1, 2):
        p = np.random.default_rng(perm_seed).permutation(cell.shape[0])
        ctx = _ctx(n, 1)
        _load(ctx, cell[p], off[p], vel[p], gm)
        rho = ctx.field(1)
        ctx.deposit_scalar(rho)
        ctx.deposit_scalar(rho)
        outs.append(rho.export_internal())
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


def test_individual_mass_deposits(cuda):
    n = (24, 24, 24)
    cell, off, vel = small_case(n, 5000, seed=4)
    rng = np.random.default_rng(5)
    m = ((1.0 + 0.1 * rng.uniform(-1, 1, 5000)) / 5000).astype(np.float32)
    res = 1.0 / 24
    ref = O.state_deposit_f64(n, cell, off, res, mass=m)
    for mode in (0, 1):
        ctx = _ctx(n, mode)
        _load(ctx, cell, off, vel, 0.0, mass=m)
        rho = ctx.field(1)
        ctx.deposit_scalar(rho)
        got = rho.export_internal()[0].reshape(-1)
        assert normalized_error(got, ref) < 1e-6
        if mode == 1:
            # the device forms the relative mass as m * (1/unit) in FP32
            unit = float(np.sum(m.astype(np.float64)) / 5000)
            mrel = (m * np.float32(1.0 / unit)).astype(np.float32)
            exact = O.fixed_to_f32(O.state_deposit_fixed(n, cell, off, mrel), fixed_scale(unit, res))
            np.testing.assert_array_equal(got, exact)


@pytest.mark.parametrize("n", [(8, 8, 8), (20, 20, 20), (33, 17, 24)])
def test_vector_and_tensor_deposits(cuda, n):
    cell, off, vel = small_case(n, 5000, seed=7, vel_sigma=0.2, clustered=True)
    res = 1.0 / n[0]
    gm = 1.0 / 5000
    ctx = _ctx(n, 0)
    _load(ctx, cell, off, vel, gm)
    vf, tf = ctx.field(3), ctx.field(6)
    ctx.deposit_vector(vf)
    ctx.deposit_symtensor(tf)
    cs, pos, v, _ = _ref_lists(n, res, cell, off, vel)
    vref = O.interior(O.vector_cicngp(n, 1, res, cs, pos, v, gmass=gm), n, 1)
    tref = O.interior(O.symtensor_cicngp(n, 1, res, cs, pos, v, gmass=gm), n, 1)
    vg, tg = vf.export_internal(), tf.export_internal()
    for c in range(3):
        assert normalized_error(vg[c], vref[c]) < 1e-6, c
    for c in range(6):
        assert normalized_error(tg[c], tref[c]) < 1e-6, c


@pytest.mark.parametrize("n", [(16, 16, 16), (20, 20, 20), (40, 40, 40)])
def test_gather_kick_bit_exact_and_reference(cuda, n):
    import torch
    cell, off, vel = small_case(n, 8000, seed=11, vel_sigma=0.02)
    res = 1.0 / n[0]
    F = np.random.default_rng(3).standard_normal((3, n[2], n[1], n[0])).astype(np.float32)
    ctx = _ctx(n, 0)
    _load(ctx, cell, off, vel, 1.0 / 8000)
    Ft = torch.from_numpy(F).cuda()
    Fh = ctx.field(3, Ft)
    dtau = 0.05
    maxv = ctx.gather_kick(Fh, dtau, want_max_v=True)
    got = by_id(ctx.get_particles(ids=True))
    exact = O.state_kick(n, cell, off, vel, F, np.float32(dtau))
    np.testing.assert_array_equal(got["vel"], exact)
    np.testing.assert_array_equal(got["cell"], cell)
    np.testing.assert_array_equal(got["off"], off)
    # the reference's updateVel with the CIC gather-kick callback, in double
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    vref = vel.astype(np.float64)[order].copy()
    mref, _ = O.update_vel_cic(n, 1, cs, pos, vref, internal_to_reference(F.astype(np.float64), 1),
                               dtau)
    vback = np.empty_like(vref)
    vback[order] = vref
    assert normalized_error(got["vel"], vback) < 2e-6
    assert maxv == pytest.approx(mref, rel=2e-6)


@pytest.mark.parametrize("n", [(16, 16, 16), (20, 20, 20), (33, 17, 24)])
@pytest.mark.parametrize("dtau", [0.1, 3.0])
def test_drift_rebin_bit_exact(cuda, n, dtau):
    cell, off, vel = small_case(n, 8000, seed=12, vel_sigma=0.05)
    res = 1.0 / n[0]
    ctx = _ctx(n, 0)
    _load(ctx, cell, off, vel, 1.0 / 8000)
    ctx.drift_rebin(dtau)
    assert ctx.count() == 8000
    got = by_id(ctx.get_particles(ids=True))
    c2, o2, bad = O.state_drift(n, cell, off, vel, np.float32(dtau / res))
    assert bad == 0
    np.testing.assert_array_equal(got["cell"], c2)
    np.testing.assert_array_equal(got["off"], o2)
    np.testing.assert_array_equal(got["vel"], vel)
    np.testing.assert_array_equal(ctx.cell_counts(), np.bincount(c2, minlength=int(np.prod(n))))
    assert ctx.flags() & ~0x8 == 0


def test_drift_matches_reference_move(cuda):
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 20000, seed=19, vel_sigma=0.02)
    res = 1.0 / 32
    dtau = 0.1
    ctx = _ctx(n, 0)
    _load(ctx, cell, off, vel, 1.0 / 20000)
    ctx.drift_rebin(dtau)
    got = by_id(ctx.get_particles(ids=True))
    pos = positions(n, res, cell, off)
    new_cell = O.move_simple(n, 1.0, pos, vel.astype(np.float64), dtau)
    u = pos / res
    near = np.any(np.abs(u - np.round(u)) < 1e-4, axis=1)
    assert np.all((got["cell"] == new_cell) | near)
    d = np.abs(positions(n, res, got["cell"], got["off"]) - pos)
    assert np.minimum(d, 1 - d).max() < 1e-6 * 32


def test_fused_step_equals_kick_then_drift(cuda):
    import torch
    n = (24, 24, 24)
    cell, off, vel = small_case(n, 10000, seed=23, vel_sigma=0.03)
    F = np.random.default_rng(6).standard_normal((3, 24, 24, 24)).astype(np.float32)
    res = 1.0 / 24
    a, b = _ctx(n, 1), _ctx(n, 1)
    for c in (a, b):
        _load(c, cell, off, vel, 1.0 / 10000)
    Ft = torch.from_numpy(F).cuda()
    Fa, Fb = a.field(3, Ft), b.field(3, Ft)
    ra, rb = a.field(1), b.field(1)
    for _ in range(3):
        a.step(Fa, 0.05, 0.2, ra)
        b.gather_kick(Fb, 0.05)
        b.drift_rebin(0.2)
        b.deposit_scalar(rb)
    ga, gb = by_id(a.get_particles(ids=True)), by_id(b.get_particles(ids=True))
    for k in ("cell", "off", "vel"):
        np.testing.assert_array_equal(ga[k], gb[k])
    np.testing.assert_array_equal(ra.export_internal(), rb.export_internal())
    # and against the oracle, step by step
    c, o, v = cell.copy(), off.copy(), vel.copy()
    for _ in range(3):
        v = O.state_kick(n, c, o, v, F, np.float32(0.05))
        c, o, _ = O.state_drift(n, c, o, v, np.float32(0.2 / res))
    np.testing.assert_array_equal(ga["vel"], v)
    np.testing.assert_array_equal(ga["cell"], c)
    np.testing.assert_array_equal(ga["off"], o)
    exact = O.fixed_to_f32(O.state_deposit_fixed(n, c, o), fixed_scale(1.0 / 10000, res))
    np.testing.assert_array_equal(ra.export_internal().reshape(-1), exact)


def test_repack_when_bricks_overflow(cuda):
    """All particles converge into one brick: its slots run out and the store
    is repacked without losing or duplicating a particle."""
    n = (64, 64, 64)
    rng = np.random.default_rng(31)
    npart = 30000
    pos = rng.random((npart, 3))
    target = np.array([0.5, 0.5, 0.5])
    dtau = 1.0
    vel = ((target + 0.01 * rng.standard_normal((npart, 3)) - pos) / dtau).astype(np.float32)
    u = pos * 64
    cell = (np.floor(u[:, 0]) + 64 * (np.floor(u[:, 1]) + 64 * np.floor(u[:, 2]))).astype(np.int32)
    off = (u - np.floor(u)).astype(np.float32)
    ctx = _ctx(n, 1)
    _load(ctx, cell, off, vel, 1.0 / npart)
    ctx.drift_rebin(dtau)
    repacks, relocations, movers = ctx.rebin_stats()
    assert repacks + relocations > 0 and movers > 0
    assert ctx.flags() & ~0x8 == 0
    got = by_id(ctx.get_particles(ids=True))
    np.testing.assert_array_equal(got["id"], np.arange(npart))
    c2, o2, _ = O.state_drift(n, cell, off, vel, np.float32(dtau * 64))
    np.testing.assert_array_equal(got["cell"], c2)
    np.testing.assert_array_equal(got["off"], o2)
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    exact = O.fixed_to_f32(O.state_deposit_fixed(n, c2, o2), fixed_scale(1.0 / npart, 1.0 / 64))
    np.testing.assert_array_equal(rho.export_internal().reshape(-1), exact)
    # move back out: the repacked store keeps working
    ctx.drift_rebin(-dtau)
    back = by_id(ctx.get_particles(ids=True))
    c3, o3, _ = O.state_drift(n, c2, o2, vel, np.float32(-dtau * 64))
    np.testing.assert_array_equal(back["cell"], c3)
    np.testing.assert_array_equal(back["off"], o3)


def test_single_brick_relocation(cuda):
    """A modest flux into one brick overflows only that brick: it is moved
    to the relocation region on its own, without a full repack."""
    n = (64, 64, 64)
    rng = np.random.default_rng(8)
    npart = 30000
    pos = rng.random((npart, 3))
    vel = np.zeros((npart, 3), np.float32)
    # 300 particles of the brick above brick 0 (in z) fall into brick 0
    above = np.where((pos[:, 0] < 0.25) & (pos[:, 1] < 0.25) & (pos[:, 2] >= 0.25) &
                     (pos[:, 2] < 0.5))[0][:300]
    vel[above, 2] = -0.25 / 1.0
    u = pos * 64
    cell = (np.floor(u[:, 0]) + 64 * (np.floor(u[:, 1]) + 64 * np.floor(u[:, 2]))).astype(np.int32)
    off = (u - np.floor(u)).astype(np.float32)
    ctx = _ctx(n, 1)
    _load(ctx, cell, off, vel, 1.0 / npart)
    ctx.drift_rebin(1.0)
    repacks, relocations, movers = ctx.rebin_stats()
    assert repacks == 0 and relocations >= 1 and movers >= 300
    got = by_id(ctx.get_particles(ids=True))
    c2, o2, _ = O.state_drift(n, cell, off, vel, np.float32(64.0))
    np.testing.assert_array_equal(got["cell"], c2)
    np.testing.assert_array_equal(got["off"], o2)
    np.testing.assert_array_equal(ctx.cell_counts(), np.bincount(c2, minlength=64 ** 3))
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    exact = O.fixed_to_f32(O.state_deposit_fixed(n, c2, o2), fixed_scale(1.0 / npart, 1.0 / 64))
    np.testing.assert_array_equal(rho.export_internal().reshape(-1), exact)
    # and again: the relocated brick keeps working and can move back out
    ctx.drift_rebin(-1.0)
    back = by_id(ctx.get_particles(ids=True))
    c3, o3, _ = O.state_drift(n, c2, o2, vel, np.float32(-64.0))
    np.testing.assert_array_equal(back["cell"], c3)
    np.testing.assert_array_equal(back["off"], o3)


def test_empty_and_single_cell(cuda):
    n = (16, 16, 16)
    ctx = _ctx(n, 1)
    e = np.zeros(0, np.int32)
    ctx.set_particles(e, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32),
                      global_mass=1.0)
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    assert not np.any(rho.export_internal())
    ctx.drift_rebin(0.1)
    assert ctx.count() == 0
    # many particles in one cell (dense cell) at the upper corner: periodic fold
    k = 5000
    cell = np.full(k, 15 + 16 * (15 + 16 * 15), np.int32)
    off = np.random.default_rng(0).random((k, 3)).astype(np.float32)
    _load(ctx, cell, off, np.zeros((k, 3), np.float32), 1.0 / k)
    ctx.deposit_scalar(rho)
    exact = O.fixed_to_f32(O.state_deposit_fixed(n, cell, off), fixed_scale(1.0 / k, 1.0 / 16))
    np.testing.assert_array_equal(rho.export_internal().reshape(-1), exact)


def test_tiny_lattices(cuda):
    for n in ((1, 1, 1), (2, 3, 1), (5, 5, 5)):
        cell, off, vel = small_case(n, 300, seed=3)
        res = 1.0 / n[0]
        ctx = _ctx(n, 1)
        _load(ctx, cell, off, vel, 1.0 / 300)
        rho = ctx.field(1)
        ctx.deposit_scalar(rho)
        exact = O.fixed_to_f32(O.state_deposit_fixed(n, cell, off), fixed_scale(1.0 / 300, res))
        np.testing.assert_array_equal(rho.export_internal().reshape(-1), exact)


def test_export_with_halo_is_update_halo(cuda):
    import torch
    n = (12, 10, 9)
    F = np.random.default_rng(8).standard_normal((3, 9, 10, 12)).astype(np.float32)
    ctx = _ctx(n, 0)
    f = ctx.field(3, torch.from_numpy(F).cuda())
    for halo in (1, 2):
        for dt in (np.float32, np.float64):
            out = f.export(halo=halo, dtype=dt, fill_halo=True)
            np.testing.assert_array_equal(out, internal_to_reference(F, halo).astype(dt))
            z = f.export(halo=halo, dtype=dt, fill_halo=False)
            ref = O.projection_init(n, halo, 3)
            ref[halo:-halo, halo:-halo, halo:-halo] = F.transpose(1, 2, 3, 0)
            np.testing.assert_array_equal(z, ref.astype(dt))
    g = ctx.field(3)
    g.import_(internal_to_reference(F, 2).astype(np.float64), halo=2)
    np.testing.assert_array_equal(g.export_internal(), F)
    # in-place halo fill of a device array in the reference layout
    dev = torch.zeros((9 + 2, 10 + 2, 12 + 2, 3), dtype=torch.float64, device="cuda")
    dev[1:-1, 1:-1, 1:-1] = torch.from_numpy(F.transpose(1, 2, 3, 0).astype(np.float64)).cuda()
    ctx.halo_fill(dev, 3, 1)
    np.testing.assert_array_equal(dev.cpu().numpy(), internal_to_reference(F, 1).astype(np.float64))


def test_conservation_sums(cuda):
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 30000, seed=41, vel_sigma=0.1)
    m = np.random.default_rng(1).uniform(0.5, 1.5, 30000).astype(np.float32)
    ctx = _ctx(n, 0)
    _load(ctx, cell, off, vel, 0.0, mass=m)
    mass, mom, maxv = ctx.conservation()
    md = m.astype(np.float64)
    assert mass == pytest.approx(md.sum(), rel=1e-12)
    np.testing.assert_allclose(mom, (md[:, None] * vel.astype(np.float64)).sum(0), rtol=1e-10,
                               atol=1e-12)
    assert maxv == pytest.approx(np.sqrt((vel.astype(np.float64) ** 2).sum(1)).max(), rel=1e-12)


def test_set_from_positions_matches_get_pos(cuda):
    n = (20, 20, 20)
    rng = np.random.default_rng(2)
    pos = rng.random((3000, 3))
    vel = 0.01 * rng.standard_normal((3000, 3))
    ctx = _ctx(n, 0)
    ctx.set_positions(pos, vel, global_mass=1.0, ids=np.arange(3000, dtype=np.int64))
    p2, v2, ids = ctx.get_positions(ids=True)
    order = np.argsort(ids)
    np.testing.assert_allclose(p2[order], pos, atol=1e-7)
    np.testing.assert_allclose(v2[order], vel, rtol=1e-6, atol=1e-9)
    counts = ctx.cell_counts()
    u = np.floor(pos * 20).astype(np.int64)
    np.testing.assert_array_equal(counts, np.bincount(u[:, 0] + 20 * (u[:, 1] + 20 * u[:, 2]),
                                                      minlength=8000))


def test_bad_input_is_reported_not_faulted(cuda):
    import latfield2_b200 as L
    n = (8, 8, 8)
    ctx = _ctx(n, 0)
    cell = np.array([0, 600], np.int32)  # 600 is outside the lattice
    off = np.zeros((2, 3), np.float32)
    with pytest.raises(L.LF2Error):
        ctx.set_particles(cell, off, off.copy(), global_mass=1.0)
    off2 = np.array([[0.5, 1.0, 0.2]], np.float32)  # offset must be < 1
    with pytest.raises(L.LF2Error):
        ctx.set_particles(np.array([0], np.int32), off2, off2.copy(), global_mass=1.0)
    ok_cell, ok_off, ok_vel = small_case(n, 100, seed=1)
    ok_vel[3, 1] = np.nan
    ctx.set_particles(ok_cell, ok_off, ok_vel, global_mass=1.0)
    ctx.drift_rebin(0.1)
    assert ctx.flags(clear=True) & 0x1
    assert ctx.count() == 100


@pytest.mark.parametrize("mode", [0, 1])
def test_medium_lattice_mass_and_properties(cuda, mode):
    """A 128^3 lattice with 2M clustered particles: conservation and
    fixed/FP32 agreement (size-independent properties)."""
    import torch
    import latfield2_b200.workloads as W
    n = (128, 128, 128)
    cell, off = W.clumps(n, 1 << 21, 64, 0.01, seed=5, device="cuda")
    vel = W.velocities(1 << 21, 0.01, seed=6, device="cuda")
    ctx = _ctx(n, mode)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / (1 << 21))
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    res = 1.0 / 128
    got = rho.export_internal()
    assert got.sum(dtype=np.float64) * res ** 3 == pytest.approx(1.0, rel=1e-6)
    counts = ctx.cell_counts()
    ref_counts = torch.bincount(cell.long(), minlength=128 ** 3).cpu().numpy()
    np.testing.assert_array_equal(counts, ref_counts)
    ref = O.state_deposit_f64(n, cell.cpu().numpy(), off.cpu().numpy(), res, gmass=1.0 / (1 << 21))
    assert normalized_error(got.reshape(-1), ref) < (1e-6 if mode == 1 else 1e-5)
    assert mean_relative_error(got.reshape(-1), ref) < (1e-5 if mode == 1 else 1e-4)


def test_last_max_velocity_matches_the_kick(cuda):
    """lf2_last_max_velocity after lf2_step equals what lf2_gather_kick with
    dtau 0 returns on the same particles (the same per-brick maxima), on the
    host path and, written in stream order, on the device path."""
    import torch
    n = (64, 64, 64)
    cell, off, vel = small_case(n, 120000, seed=41, vel_sigma=0.03)
    F = np.random.default_rng(4).standard_normal((3, 64, 64, 64)).astype(np.float32)
    ctx = _ctx(n, 1)
    _load(ctx, cell, off, vel, 1.0 / 120000)
    Fh = ctx.field(3, torch.from_numpy(F).cuda())
    rho = ctx.field(1)
    ctx.step(Fh, 0.05, 0.2, rho)
    host = ctx.last_max_velocity()
    dev = ctx.last_max_velocity(torch.zeros(1, dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    assert float(dev[0]) == host
    assert ctx.gather_kick(Fh, 0.0, want_max_v=True) == host
    v = ctx.get_particles()["vel"].astype(np.float64)
    assert host == pytest.approx(float(np.sqrt((v ** 2).sum(1).max())), rel=1e-6)
