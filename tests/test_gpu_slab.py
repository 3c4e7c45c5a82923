"""GPU side of the slab decomposition: lf2_particles_extract_z and
lf2_particles_add, the migration records of lf2_slab_count / lf2_slab_extract
/ lf2_slab_insert through the C ABI, and latfield2_b200.distributed.SlabDomain
on the CUDA engine with one rank (its neighbours are itself), against the
plain single-GPU path on the same particles.

Particles bit-exact by id (migration moves state, it does not recompute it);
the density within 1e-6 of its maximum (the fold adds FP32 values).
"""
import numpy as np
import pytest

from tests.helpers import small_case

pytestmark = pytest.mark.gpu


def _ctx(n, mode=1):
    import latfield2_b200 as L
    return L.Context(n, box=tuple(v / n[0] for v in n), mode=mode)


def _by_id(d):
    o = np.argsort(d["id"])
    return {k: np.asarray(v)[o] for k, v in d.items()}


def _np(t):
    return {k: v.cpu().numpy() for k, v in t.items()}


def test_extract_and_add_back():
    n = (32, 24, 40)
    cell, off, vel = small_case(n, 50000, seed=5)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    ctx = _ctx(n)
    ctx.set_particles(cell, off, vel, global_mass=1e-5, ids=ids)
    before = _by_id(ctx.get_particles(ids=True))
    counts0 = ctx.cell_counts()
    out = _np(ctx.extract_z(7, 29, ids=True))
    z = out["cell"] // (n[0] * n[1])
    assert z.shape[0] > 10000 and np.all((z < 7) | (z > 29))
    rest = ctx.get_particles(ids=True)
    zr = rest["cell"] // (n[0] * n[1])
    assert np.all((zr >= 7) & (zr <= 29))
    assert ctx.count() == rest["cell"].shape[0] == cell.shape[0] - out["cell"].shape[0]
    both = {k: np.concatenate([rest[k], out[k]]) for k in ("cell", "off", "vel", "id")}
    both = _by_id(both)
    for k in before:
        np.testing.assert_array_equal(both[k], before[k])
    # back in (device arrays), and the store is whole again
    import torch
    t = {k: torch.from_numpy(v).cuda() for k, v in out.items()}
    ctx.add_particles(t["cell"], t["off"], t["vel"], ids=t["id"])
    after = _by_id(ctx.get_particles(ids=True))
    for k in before:
        np.testing.assert_array_equal(after[k], before[k])
    np.testing.assert_array_equal(ctx.cell_counts(), counts0)
    # nothing outside: an empty result, no change
    assert _np(ctx.extract_z(0, n[2] - 1, ids=True))["cell"].shape[0] == 0
    assert ctx.count() == cell.shape[0]
    # adding nothing is allowed (empty arrays, null pointers)
    e = _np(ctx.extract_z(0, n[2] - 1, ids=True))
    ctx.add_particles(e["cell"], e["off"], e["vel"], ids=e["id"])
    assert ctx.count() == cell.shape[0]


def test_add_beyond_the_store_reloads_and_bad_input_adds_nothing():
    import latfield2_b200 as L
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 1000, seed=6)
    ids = np.arange(1000, dtype=np.int64)
    ctx = _ctx(n)
    ctx.set_particles(cell, off, vel, global_mass=1e-3, ids=ids)
    c2, o2, v2 = small_case(n, 200000, seed=7, clustered=True)
    ids2 = np.arange(1000, 201000, dtype=np.int64)
    ctx.add_particles(c2, o2, v2, ids=ids2)
    got = _by_id(ctx.get_particles(ids=True))
    np.testing.assert_array_equal(got["id"], np.arange(201000))
    np.testing.assert_array_equal(got["cell"], np.concatenate([cell, c2]))
    np.testing.assert_array_equal(got["off"], np.concatenate([off, o2]))
    bad_cell = np.array([0, n[0] * n[1] * n[2]], np.int32)
    with pytest.raises(L.LF2Error, match="out of range"):
        ctx.add_particles(bad_cell, np.zeros((2, 3), np.float32), np.zeros((2, 3), np.float32),
                          ids=np.array([-1, -2], np.int64))
    assert ctx.count() == 201000
    ctx.synchronize()
    # the same bad input through the mover path (room in the store): intact
    ctx2 = _ctx(n)
    ctx2.set_particles(cell, off, vel, global_mass=1e-3, ids=ids)
    with pytest.raises(L.LF2Error, match="out of range"):
        ctx2.add_particles(bad_cell, np.full((2, 3), 0.5, np.float32),
                           np.zeros((2, 3), np.float32), ids=np.array([-1, -2], np.int64))
    kept = _by_id(ctx2.get_particles(ids=True))
    np.testing.assert_array_equal(kept["id"], ids)
    np.testing.assert_array_equal(kept["cell"], cell)
    ctx2.synchronize()


@pytest.mark.parametrize("n", [(32, 32, 32), (40, 24, 20)])
def test_one_rank_slab_domain_equals_the_single_gpu_step(n):
    """SlabDomain with one rank: ghost planes, migration across the periodic
    z face (through extract/add) and the folded deposit give what lf2_step
    gives on the whole lattice."""
    import torch
    from latfield2_b200 import _lib
    from latfield2_b200.distributed import SlabDomain
    steps, dtk, dtd = 5, 0.05, 0.02
    res = 1.0 / n[0]
    cell, off, _ = small_case(n, 60000, seed=11)
    rng = np.random.default_rng(12)
    vel = (rng.uniform(-0.55, 0.55, (cell.shape[0], 3)) * res / dtd).astype(np.float32)
    F = (0.1 * rng.standard_normal((3, n[2], n[1], n[0]))).astype(np.float32)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    gm = 1.0 / cell.shape[0]

    ref = _ctx(n)
    ref.set_particles(cell, off, vel, global_mass=gm, ids=ids)
    Fh = ref.field(3, torch.from_numpy(F).cuda())
    rho_ref = ref.field(1)
    for k in range(steps):
        ref.step(Fh, dtk, dtd, rho_ref if k == steps - 1 else None)
    want = _by_id(ref.get_particles(ids=True))

    d = SlabDomain(n, box=1.0, mode=_lib.DEPOSIT_FIXED64)
    d.set_particles(cell, off, vel, gm, ids=ids)
    Ff = d.field(3)
    d.set_own_planes(Ff, F)
    rho = d.field(1)
    for k in range(steps):
        d.step(Ff, dtk, dtd, rho if k == steps - 1 else None)
    got = _by_id(d.particles_global())
    for k in ("id", "cell", "off", "vel"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    r = d.own_planes(rho)[0]
    w = rho_ref.export_internal()[0]
    assert np.abs(r - w).max() <= 1e-6 * np.abs(w).max()
    zs = cell // (n[0] * n[1])
    zf = want["cell"] // (n[0] * n[1])
    assert np.sum(np.abs(zs[want["id"]] - zf) > n[2] // 2) > 50  # crossed the periodic z face


@pytest.mark.parametrize("n", [(32, 32, 32), (40, 24, 20)])
def test_one_rank_slab_projections_equal_the_single_gpu_deposits(n):
    """SlabDomain.project with one rank (both folds go to itself) against the
    library's deposits on the whole lattice: vector and symtensor CIC-NGP,
    full-CIC vector and VecVec, within 1e-5 of each component's maximum
    (FP32 shared atomics in another order, plus the FP32 fold)."""
    from latfield2_b200 import _lib
    from latfield2_b200.distributed import SlabDomain
    cell, off, vel = small_case(n, 60000, seed=13)
    gm = 1.0 / cell.shape[0]
    ref = _ctx(n)
    ref.set_particles(cell, off, vel, global_mass=gm)
    d = SlabDomain(n, box=1.0, mode=_lib.DEPOSIT_FIXED64)
    d.set_particles(cell, off, vel, gm)
    for kind, (comps, _) in SlabDomain.PROJECTIONS.items():
        want = ref.field(comps)
        getattr(ref, "deposit_" + kind)(want)
        w = want.export_internal()
        f = d.field(comps)
        d.project(kind, f)
        got = d.own_planes(f)
        for c in range(comps):
            assert np.abs(got[c] - w[c]).max() <= 1e-5 * np.abs(w[c]).max(), (kind, c)


@pytest.mark.parametrize("n", [32, 48])
def test_one_rank_slab_pm_force_equals_the_single_gpu_operator(n):
    """SlabDomain.pm_force with one rank (the slab transforms through
    lf2_slab_fft_*, lf2_slab_green and lf2_pm_gradient) against lf2_pm_force
    on the whole lattice and against the FP64 oracle: 1e-5 of the maximum."""
    import torch
    from latfield2_b200 import _lib
    from latfield2_b200.distributed import SlabDomain
    from oracle import fft_oracle as FO
    coupling = 4 * np.pi
    rng = np.random.default_rng(n)
    rho_g = (1.0 + rng.standard_normal((n, n, n))).astype(np.float32)
    ref = _ctx((n, n, n))
    Fr = ref.field(3)
    ref.pm_force(ref.field(1, torch.from_numpy(rho_g.reshape(-1)).cuda()), Fr, coupling)
    want = Fr.export_internal()
    phi64, F64 = FO.pm_force(rho_g, 1.0 / n, coupling)
    d = SlabDomain((n, n, n), box=1.0, mode=_lib.DEPOSIT_FIXED64)
    rho = d.field(1)
    d.set_own_planes(rho, rho_g[None])
    F, phi = d.field(3), d.field(1)
    d.pm_force(rho, F, coupling, phi)
    got = d.own_planes(F)
    for c in range(3):
        scale = np.abs(F64[c]).max()
        assert np.abs(got[c] - want[c]).max() <= 1e-5 * scale, c
        assert np.abs(got[c] - F64[c]).max() <= 1e-5 * scale, c
    assert np.abs(d.own_planes(phi)[0] - phi64).max() <= 1e-5 * np.abs(phi64).max()


@pytest.mark.parametrize("ranks", [2, 4])
def test_slab_pieces_with_several_ky_slabs_on_one_gpu(ranks):
    """lf2_slab_fft_* and lf2_slab_green for 2 and 4 z slabs emulated in one
    process on one GPU (the ranks one after the other, transposes by slicing;
    nothing waits on another launch): k_y slabs with ky0 > 0, against the FP64
    operator (1e-5 of the maximum).  The same emulation runs on the CPU in
    tests/test_slab.py with the numpy engine."""
    import torch
    from latfield2_b200.distributed import CudaEngine
    from oracle import fft_oracle as FO
    from tests.helpers import slab_potential_emulated
    n, coupling = 32, 4 * np.pi
    rng = np.random.default_rng(70 + ranks)
    rho = (1.0 + rng.standard_normal((n, n, n))).astype(np.float32)
    phi = slab_potential_emulated(CudaEngine, torch.from_numpy(rho).cuda(), ranks, coupling,
                                  device=0).cpu().numpy()
    want = FO.pm_force(rho, 1.0 / n, coupling)[0]
    assert np.abs(phi - want).max() <= 1e-5 * np.abs(want).max()


def test_one_rank_exact_slab_deposit_is_the_single_gpu_deposit():
    """SlabDomain.deposit(exact=True) with one rank (ghost copies of its own
    top plane on plane 0, no FP32 fold) equals lf2_deposit_scalar on the
    whole lattice bit for bit, and leaves the particle count unchanged."""
    from latfield2_b200 import _lib
    from latfield2_b200.distributed import SlabDomain
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 60000, seed=17, clustered=True)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    gm = 1.0 / cell.shape[0]
    ref = _ctx(n)
    ref.set_particles(cell, off, vel, global_mass=gm, ids=ids)
    want = ref.field(1)
    ref.deposit_scalar(want)
    d = SlabDomain(n, box=1.0, mode=_lib.DEPOSIT_FIXED64)
    d.set_particles(cell, off, vel, gm, ids=ids)
    rho = d.field(1)
    d.deposit(rho, exact=True)
    np.testing.assert_array_equal(d.own_planes(rho)[0], want.export_internal()[0])
    assert d.count() == cell.shape[0]


def _records(rec, has_mass, has_id):
    """Migration records (int32 words) as separate numpy arrays."""
    r = np.ascontiguousarray(rec.cpu().numpy())
    out = {"cell": r[:, 0].copy(), "off": np.ascontiguousarray(r[:, 1:4]).view(np.float32),
           "vel": np.ascontiguousarray(r[:, 4:7]).view(np.float32)}
    w = 7
    if has_mass:
        out["mass"] = np.ascontiguousarray(r[:, w]).view(np.float32)
        w += 1
    if has_id:
        out["id"] = np.ascontiguousarray(r[:, w:w + 2]).view(np.int64)[:, 0]
    return out


@pytest.mark.parametrize("masses", [False, True])
def test_migration_records_count_extract_insert(masses):
    """lf2_slab_count / lf2_slab_extract / lf2_slab_insert (the migration
    without host waits): the counts, the records (bit-exact state, cell index
    moved by -+nz planes into the neighbour's lattice), the store without
    them, and the store with the records inserted."""
    import torch
    n = (32, 24, 40)
    plane = n[0] * n[1]
    cell, off, vel = small_case(n, 50000, seed=5)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    mass = (np.random.default_rng(3).uniform(0.5, 2.0, cell.shape[0]).astype(np.float32)
            if masses else None)
    ctx = _ctx(n)
    ctx.set_particles(cell, off, vel, mass=mass, global_mass=0.0 if masses else 1e-5, ids=ids)
    assert ctx.slab_record_words() == 7 + masses + 2
    z = cell // plane
    zlo, zhi = 7, 29
    nz = zhi - zlo + 1
    lo, hi = z < zlo, z > zhi
    counts = ctx.slab_count(zlo, zhi, torch.zeros(4, dtype=torch.int64, device="cuda"))
    want = [lo.sum(), hi.sum(), ((z < zlo - 1) | (z > zhi + 1)).sum()]
    assert counts.cpu().tolist() == [int(v) for v in want] + [0]  # no kick yet
    # max |v|^2 of a kick (of nothing, no drift) as float bits
    F0 = ctx.field(3, torch.zeros((3, n[2], n[1], n[0]), dtype=torch.float32, device="cuda"))
    ctx.step(F0, 0.0, 0.0)
    c4 = ctx.slab_count(zlo, zhi, torch.zeros(4, dtype=torch.int64, device="cuda")).cpu().tolist()
    assert c4[:3] == [int(v) for v in want]
    v2 = np.array([c4[3]], np.uint32).view(np.float32)[0]
    assert np.sqrt(np.float64(v2)) == ctx.last_max_velocity()
    below, above = ctx.slab_extract(zlo, zhi, int(want[0]), int(want[1]))
    rb, ra = _records(below, masses, True), _records(above, masses, True)
    for r, sel, dz in ((rb, lo, nz), (ra, hi, -nz)):
        o = np.argsort(r["id"])
        r = {k: v[o] for k, v in r.items()}
        np.testing.assert_array_equal(r["id"], ids[sel])
        np.testing.assert_array_equal(r["cell"], cell[sel] + dz * plane)
        np.testing.assert_array_equal(r["off"], off[sel])
        np.testing.assert_array_equal(r["vel"], vel[sel])
        if masses:
            np.testing.assert_array_equal(r["mass"], mass[sel])
    inside = ~(lo | hi)
    rest = _by_id(ctx.get_particles(mass=masses, ids=True))
    np.testing.assert_array_equal(rest["id"], ids[inside])
    np.testing.assert_array_equal(rest["cell"], cell[inside])
    assert ctx.count() == int(inside.sum())
    # the records back in, at their moved cells: the store holds every particle
    ctx.slab_insert(above, below)
    got = _by_id(ctx.get_particles(mass=masses, ids=True))
    moved = cell + np.where(lo, nz, np.where(hi, -nz, 0)) * plane
    np.testing.assert_array_equal(got["id"], ids)
    np.testing.assert_array_equal(got["cell"], moved)
    np.testing.assert_array_equal(got["off"], off)
    np.testing.assert_array_equal(got["vel"], vel)
    if masses:
        np.testing.assert_array_equal(got["mass"], mass)
    np.testing.assert_array_equal(ctx.cell_counts(), np.bincount(moved, minlength=np.prod(n)))
    assert ctx.count() == cell.shape[0]
    ctx.synchronize()


def test_migration_records_reload_bad_record_and_short_counts():
    """Insert beyond the store's room goes through the reloading add; a
    record out of range raises LF2_FLAG_BAD_CELL; counts short of
    slab_count's raise LF2_FLAG_CAPACITY (nothing is written past them)."""
    import torch
    import latfield2_b200 as L
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 1000, seed=6)
    ids = np.arange(1000, dtype=np.int64)
    ctx = _ctx(n)
    ctx.set_particles(cell, off, vel, global_mass=1e-3, ids=ids)
    c2, o2, v2 = small_case(n, 200000, seed=7, clustered=True)
    ids2 = np.arange(1000, 201000, dtype=np.int64)
    rec = np.concatenate([c2[:, None], o2.view(np.int32), v2.view(np.int32),
                          ids2.view(np.int32).reshape(-1, 2)], axis=1)
    rec = torch.from_numpy(np.ascontiguousarray(rec)).cuda()
    ctx.slab_insert(rec[:150000], rec[150000:])
    got = _by_id(ctx.get_particles(ids=True))
    np.testing.assert_array_equal(got["id"], np.arange(201000))
    np.testing.assert_array_equal(got["cell"], np.concatenate([cell, c2]))
    np.testing.assert_array_equal(got["vel"], np.concatenate([vel, v2]))
    ctx.synchronize()
    # a record out of range is dropped and reported
    bad = rec[:4].clone()
    bad[1, 0] = n[0] * n[1] * n[2]
    ctx.slab_insert(bad, bad[:0])
    with pytest.raises(L.LF2Error):
        ctx.synchronize()
    # short counts: the particles beyond them are reported
    ctx3 = _ctx(n)
    ctx3.set_particles(cell, off, vel, global_mass=1e-3, ids=ids)
    z = cell // (n[0] * n[1])
    nb = int((z < 4).sum())
    assert nb > 2
    ctx3.slab_extract(4, 31, nb - 2, 0)
    with pytest.raises(L.LF2Error):
        ctx3.synchronize()
