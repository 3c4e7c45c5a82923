"""The slab decomposition (latfield2_b200/distributed.py) on CPU processes:
the exchange logic (ghost planes of the force field, migration of particles
that crossed a slab face, the upper-plane fold of the deposit) with the
oracle's restatement of the device arithmetic as the local engine
(tests/slab_oracle_engine.py), over gloo with 1, 2 and 4 ranks.

Against a single-domain run of the same arithmetic on the whole lattice:
particles (by id) bit-exact after several steps (the kick reads the same
force values, the drift is per particle); the density within 1e-6 of its
maximum (the fold adds two FP32 values where one domain converts one exact
integer sum).  The vector and symtensor CIC-NGP projections and the full-CIC
vector and VecVec projections of the final state, each folded across the
slab faces, within 1e-6 of their maximum of the oracle's FP64 projection on
the whole lattice.
"""
import os
import socket

import numpy as np
import pytest

from latfield2_b200 import _lib
from oracle import oracle as O
from tests.helpers import small_case

N = (16, 12, 16)
STEPS = 4
DTK, DTD = 0.05, 0.02
KINDS = {"vector": (3, O.vector_cicngp), "symtensor": (6, O.symtensor_cicngp),
         "vector_cic": (3, O.vector_cic), "vecvec_cic": (6, O.vecvec_cic)}


def _case():
    """Uniform particles whose velocities move them up to 0.55 cells per step
    and component (|v| dtau under one cell, the decomposition's limit; the
    kick adds little), so that many cross slab faces."""
    cell, off, _ = small_case(N, 3000, seed=21)
    rng = np.random.default_rng(22)
    res = 1.0 / N[0]
    vel = (rng.uniform(-0.55, 0.55, (cell.shape[0], 3)) * res / DTD).astype(np.float32)
    F = (0.1 * rng.standard_normal((3, N[2], N[1], N[0]))).astype(np.float32)
    return cell, off, vel, F, np.arange(cell.shape[0], dtype=np.int64)


def _single_domain(cell, off, vel, F):
    res = 1.0 / N[0]
    c, o, v = cell.copy(), off.copy(), vel.copy()
    for _ in range(STEPS):
        v = O.state_kick(N, c, o, v, F, np.float32(DTK))
        c, o, _ = O.state_drift(N, c, o, v, np.float32(DTD / res))
    gm = 1.0 / cell.shape[0]
    scale = np.float32(2.0 ** -32 * gm / res ** 3)
    rho = O.fixed_to_f32(O.state_deposit_fixed(N, c, o), scale).reshape(N[2], N[1], N[0])
    return c, o, v, rho


def _run_domain(dist_initialised):
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    cell, off, vel, F, ids = _case()
    d = SlabDomain(N, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=OracleEngine)
    d.set_particles(cell, off, vel, 1.0 / cell.shape[0], ids=ids)
    Ff = d.field(3)
    d.set_own_planes(Ff, F)
    rho = d.field(1)
    for k in range(STEPS):
        d.step(Ff, DTK, DTD, rho if k == STEPS - 1 else None)
    p = d.particles_global()
    proj = {}
    for kind, (comps, _) in KINDS.items():
        f = d.field(comps)
        d.project(kind, f)
        proj[kind] = d.own_planes(f)
    return d.rank, d.z0, d.nz, p, d.own_planes(rho)[0], proj


def _check(results):
    cell, off, vel, F, ids = _case()
    c1, o1, v1, rho1 = _single_domain(cell, off, vel, F)
    got = {k: np.concatenate([r[3][k] for r in results]) for k in ("cell", "off", "vel", "id")}
    order = np.argsort(got["id"])
    np.testing.assert_array_equal(got["id"][order], ids)
    np.testing.assert_array_equal(got["cell"][order], c1)
    np.testing.assert_array_equal(got["off"][order], o1)
    np.testing.assert_array_equal(got["vel"][order], v1)
    rho = np.zeros_like(rho1)
    for _, z0, nz, _, r, _ in results:
        rho[z0:z0 + nz] = r
    assert np.abs(rho - rho1).max() <= 1e-6 * np.abs(rho1).max()
    res = 1.0 / N[0]
    cs, order = O.lists_from_insertion(N, c1)
    pos = O.state_to_pos(N, res, c1, o1)[order]
    vv = v1.astype(np.float64)[order]
    for kind, (comps, fn) in KINDS.items():
        want = O.interior(fn(N, 1, res, cs, pos, vv, gmass=1.0 / cell.shape[0]), N, 1)
        got = np.zeros_like(want)
        for _, z0, nz, _, _, proj in results:
            got[:, z0:z0 + nz] = proj[kind]
        for c in range(comps):
            assert np.abs(got[c] - want[c]).max() <= 1e-6 * np.abs(want[c]).max(), (kind, c)
    # many particles changed slab (the periodic face included)
    nz = results[0][2]
    moved = (cell // (N[0] * N[1]) // nz) != (c1 // (N[0] * N[1]) // nz)
    assert len(results) == 1 or moved.sum() > 100


def test_one_rank_exchanges_with_itself():
    """Without a process group the domain is one rank whose neighbours are
    itself: the periodic single-domain result."""
    _check([_run_domain(False)])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out, fn="_run_domain"):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out.put(globals()[fn](True))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_ranks_over_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    _check(res)


def test_too_fast_a_particle_is_refused():
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    cell, off, vel, F, ids = _case()
    d = SlabDomain(N, engine=OracleEngine)
    d.set_particles(cell, off, vel * 2.0, 1.0 / cell.shape[0], ids=ids)
    Ff = d.field(3)
    d.set_own_planes(Ff, F)
    with pytest.raises(RuntimeError, match="less than one cell"):
        d.step(Ff, DTK, DTD)


NPM = 16
COUPLING = 4 * np.pi


def _pm_field():
    rng = np.random.default_rng(31)
    return (1.0 + rng.standard_normal((NPM, NPM, NPM))).astype(np.float32)


def _run_pm(dist_initialised):
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    d = SlabDomain((NPM,) * 3, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=OracleEngine)
    rho = d.field(1)
    d.set_own_planes(rho, _pm_field()[None])
    F, phi = d.field(3), d.field(1)
    d.pm_force(rho, F, COUPLING, phi)
    return d.rank, d.z0, d.nz, F[0].numpy().copy(), phi[0].numpy().copy()


def _check_pm(results):
    from oracle import fft_oracle as FO
    phi_ref, F_ref = FO.pm_force(_pm_field(), 1.0 / NPM, COUPLING)
    for _, z0, nz, F, phi in results:
        planes = [(z0 - 1 + p) % NPM for p in range(nz + 2)]  # ghost planes included
        for c in range(3):
            assert np.abs(F[c] - F_ref[c][planes]).max() <= 1e-5 * np.abs(F_ref[c]).max(), c
        assert np.abs(phi[0] - phi_ref[planes]).max() <= 1e-5 * np.abs(phi_ref).max()


@pytest.mark.parametrize("world", [1, 2, 4])
def test_pm_force_over_slabs(world):
    """SlabDomain.pm_force (plane transforms, all-to-all transposes, line
    transforms, Green's function, gradient with ghost planes) against the
    single-domain FP64 PM force, on 1, 2 and 4 gloo ranks."""
    if world == 1:
        _check_pm([_run_pm(False)])
        return
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, "_run_pm"))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    _check_pm(res)


def _run_pm_steps(dist_initialised):
    """Three self-consistent PM steps of clustered particles on the cubic
    lattice NPM^3."""
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    cell, off, _ = small_case((NPM,) * 3, 4000, seed=51, clustered=True)
    rng = np.random.default_rng(52)
    vel = (0.1 * rng.standard_normal((cell.shape[0], 3)) / NPM / DTD).astype(np.float32)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    d = SlabDomain((NPM,) * 3, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=OracleEngine)
    d.set_particles(cell, off, vel, 1.0 / cell.shape[0], ids=ids)
    rho, F = d.field(1), d.field(3)
    for _ in range(3):
        d.pm_step(rho, F, 0.002, DTD, COUPLING)
    return d.rank, d.particles_global()


@pytest.mark.parametrize("world", [2, 4])
def test_pm_steps_agree_on_any_number_of_ranks(world):
    """pm_step (deposit, slab PM force, kick-drift, migration) on `world`
    gloo ranks against one rank.  The transforms are per plane and per line,
    so the rank count changes no FFT arithmetic; the deposit's fold at each
    slab face adds two FP32 values where one rank converts one exact integer
    sum, so forces, and the particles after three steps, agree to FP32
    rounding (positions within 1e-6 of the box, velocities within 1e-5 of
    their maximum), not bit for bit."""
    from latfield2_b200 import snapshot as S
    one = _run_pm_steps(False)[1]
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, "_run_pm_steps"))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = {k: np.concatenate([r[1][k] for r in res]) for k in ("id", "cell", "off", "vel")}
    o1, o2 = np.argsort(one["id"]), np.argsort(got["id"])
    np.testing.assert_array_equal(got["id"][o2], one["id"][o1])
    res_ = 1.0 / NPM
    p1 = S.cells_to_positions(one["cell"][o1], one["off"][o1], (NPM,) * 3, res_)
    p2 = S.cells_to_positions(got["cell"][o2], got["off"][o2], (NPM,) * 3, res_)
    d = np.abs(p1 - p2)
    assert np.minimum(d, 1.0 - d).max() < 1e-6
    v1, v2 = one["vel"][o1], got["vel"][o2]
    assert np.abs(v1 - v2).max() <= 1e-5 * np.abs(v1).max()
    assert (got["cell"][o2] != one["cell"][o1]).sum() <= 2  # a face crossing may differ


def test_bad_requests_are_refused():
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    d = SlabDomain(N, engine=OracleEngine)  # N is not cubic
    with pytest.raises(ValueError, match="cubic"):
        d.pm_force(d.field(1), d.field(3), COUPLING)
    with pytest.raises(ValueError, match="unknown projection"):
        d.project("scalar", d.field(1))
    with pytest.raises(ValueError, match="3 components"):
        d.project("vector_cic", d.field(6))


def _run_exact(dist_initialised):
    """Two exact pm_steps of clustered particles, then an exact deposit."""
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    cell, off, _ = small_case((NPM,) * 3, 4000, seed=61, clustered=True)
    rng = np.random.default_rng(62)
    vel = (0.1 * rng.standard_normal((cell.shape[0], 3)) / NPM / DTD).astype(np.float32)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    d = SlabDomain((NPM,) * 3, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=OracleEngine)
    d.set_particles(cell, off, vel, 1.0 / cell.shape[0], ids=ids)
    rho, F = d.field(1), d.field(3)
    for _ in range(2):
        d.pm_step(rho, F, 0.002, DTD, COUPLING, exact=True)
    d.deposit(rho, exact=True)
    return d.rank, d.z0, d.nz, d.particles_global(), d.own_planes(rho)[0], d.count()


@pytest.mark.parametrize("world", [2, 4])
def test_exact_deposits_make_the_steps_independent_of_the_rank_count(world):
    """With exact=True the slab density is the single-domain fixed-point
    deposit bit for bit, so pm_steps on 1, 2 and 4 ranks give the same
    particles bit for bit; the ghost copies leave the stores again."""
    one = _run_exact(False)
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, "_run_exact"))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=180) for _ in range(world)], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = {k: np.concatenate([r[3][k] for r in res]) for k in ("id", "cell", "off", "vel")}
    assert sum(r[5] for r in res) == one[5] == got["id"].shape[0]
    o1, o2 = np.argsort(one[3]["id"]), np.argsort(got["id"])
    for k in ("id", "cell", "off", "vel"):
        np.testing.assert_array_equal(got[k][o2], one[3][k][o1], err_msg=k)
    # the density: bit-identical to the single-domain fixed-point deposit
    c, o = one[3]["cell"], one[3]["off"]
    scale = np.float32(2.0 ** -32 * (1.0 / 4000) / (1.0 / NPM) ** 3)
    want = O.fixed_to_f32(O.state_deposit_fixed((NPM,) * 3, c, o), scale).reshape((NPM,) * 3)
    rho = np.zeros_like(want)
    for _, z0, nz, _, r, _ in res:
        rho[z0:z0 + nz] = r
    np.testing.assert_array_equal(rho, want)
    np.testing.assert_array_equal(one[4], want)


def test_exact_deposit_needs_the_fixed_point_mode():
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    d = SlabDomain((NPM, NPM, 1), engine=OracleEngine)  # one plane per rank
    with pytest.raises(ValueError, match="exact"):
        d.deposit(d.field(1), exact=True)


def _run_fast_on_one_rank(dist_initialised):
    """Only the upper half of the box holds a particle that moves more than a
    cell per step; every rank must raise, none may wait in the migration."""
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    cell, off, vel, F, ids = _case()
    vel = vel * 0.5
    z = cell // (N[0] * N[1])
    fast = np.flatnonzero(z >= N[2] // 2)[0]
    vel[fast] = np.array([0, 0, 3.0 / N[0] / DTD], np.float32)
    d = SlabDomain(N, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=OracleEngine)
    d.set_particles(cell, off, vel, 1.0 / cell.shape[0], ids=ids)
    m, mom, vmax = d.conservation()
    Ff = d.field(3)
    d.set_own_planes(Ff, F)
    try:
        d.step(Ff, DTK, DTD)
        outcome = "stepped"
    except RuntimeError as e:
        outcome = "raised" if "less than one cell" in str(e) else str(e)
    return d.rank, outcome, m, mom, vmax


def test_a_too_fast_particle_on_one_rank_stops_every_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, "_run_fast_on_one_rank"))
             for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == ["raised", "raised"]
    # the conservation sums are global and the same on every rank
    cell, off, vel, F, ids = _case()
    v = (vel * 0.5).astype(np.float64)
    v[np.flatnonzero(cell // (N[0] * N[1]) >= N[2] // 2)[0]] = [0, 0, np.float32(3.0 / N[0] / DTD)]
    for _, _, m, mom, vmax in res:
        assert m == pytest.approx(1.0, rel=1e-12)
        np.testing.assert_allclose(mom, v.sum(axis=0) / cell.shape[0], rtol=1e-10, atol=1e-15)
        assert vmax == pytest.approx(float(np.sqrt((v * v).sum(axis=1).max())), rel=1e-12)


@pytest.mark.parametrize("ranks", [2, 4])
def test_slab_potential_emulated_in_one_process(ranks):
    """The emulation that tests/test_gpu_slab.py runs on one GPU (k_y slabs
    with ky0 > 0), here with the numpy engine, against the FP64 operator."""
    import torch
    from oracle import fft_oracle as FO
    from tests.helpers import slab_potential_emulated
    from tests.slab_oracle_engine import OracleEngine
    rho = _pm_field()
    phi = slab_potential_emulated(OracleEngine, torch.from_numpy(rho), ranks, COUPLING).numpy()
    want = FO.pm_force(rho, 1.0 / NPM, COUPLING)[0]
    assert np.abs(phi - want).max() <= 1e-5 * np.abs(want).max()


def _run_still(dist_initialised):
    """Particles at rest: the migration finds nobody to send, every message is
    empty, and the particles stay as they were."""
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    cell, off, vel, F, ids = _case()
    vel = np.zeros_like(vel)
    d = SlabDomain(N, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=OracleEngine)
    d.set_particles(cell, off, vel, 1.0 / cell.shape[0], ids=ids)
    Ff = d.field(3)
    d.set_own_planes(Ff, np.zeros_like(F))
    before = d.engine.particles()
    for _ in range(2):
        d.step(Ff, DTK, DTD)
    after = d.engine.particles()
    return d.rank, {k: np.array_equal(before[k], after[k]) for k in before}


def test_a_step_without_migrants_sends_nothing_and_keeps_the_particles():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, "_run_still")) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, same in res:
        assert all(same.values()), same
