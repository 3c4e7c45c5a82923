"""The slab decomposition (latfield2_b200/distributed.py) on CPU processes:
the exchange logic (ghost planes of the force field, migration of particles
that crossed a slab face, the upper-plane fold of the deposit) with the
oracle's restatement of the device arithmetic as the local engine
(tests/slab_oracle_engine.py), over gloo with 1, 2 and 4 ranks.

Against a single-domain run of the same arithmetic on the whole lattice:
particles (by id) bit-exact after several steps (the kick reads the same
force values, the drift is per particle); the density within 1e-6 of its
maximum (the fold adds two FP32 values where one domain converts one exact
integer sum).
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
    return d.rank, d.z0, d.nz, p, d.own_planes(rho)[0]


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
    for _, z0, nz, _, r in results:
        rho[z0:z0 + nz] = r
    assert np.abs(rho - rho1).max() <= 1e-6 * np.abs(rho1).max()
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


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out.put(_run_domain(True))
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
