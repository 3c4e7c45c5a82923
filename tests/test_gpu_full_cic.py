"""GPU parity of the full-CIC projections (vectorProjectionCIC,
VecVecProjectionCIC; projections.hpp:978-1814) against the CPU oracle,
called through the C ABI.

Every case runs in the three deposit modes: FP32 (compensated atomics) and
fixed point within 1e-6 of the FP64 oracle, normalized by the field's
maximum, plain FP32 within 1e-5.  The cases cover ragged
bricks (n not a multiple of 16), lattices one or two bricks wide (a brick is
its own neighbour across the periodic fold), a one-site-wide dim, individual
masses, a dense cell at the lattice corner (both halos fold), an empty store,
an output field that starts with garbage (the deposit overwrites every
site), and the exact sums that hold at any size: the staggered and vertex
weights of a particle each sum to one, so the field sums are the total
momentum and the total m v_i v_j.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import normalized_error, positions, small_case

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8, 8), (16, 16, 16), (20, 18, 17), (33, 16, 2), (1, 3, 2), (48, 48, 48)]
KINDS = [("vector_cic", 3, O.vector_cic), ("vecvec_cic", 6, O.vecvec_cic)]


MODES = [0, 1, 2]


def _tol(mode):
    return 1e-5 if mode == 2 else 1e-6


def _ctx(n, mode=0):
    import latfield2_b200 as L
    return L.Context(n, box=tuple(v / n[0] for v in n), mode=mode)


def _load(ctx, cell, off, vel, gm, mass=None):
    ctx.set_particles(cell, off, vel, mass=mass, global_mass=0.0 if mass is not None else gm,
                      ids=np.arange(cell.shape[0], dtype=np.int64))


def _oracle(fn, n, cell, off, vel, gm, mass=None):
    res = 1.0 / n[0]
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    pm = None if mass is None else mass.astype(np.float64)[order]
    return O.interior(fn(n, 1, res, cs, pos, vel.astype(np.float64)[order], pmass=pm, gmass=gm),
                      n, 1)


def _deposit(ctx, name, comps, field=None):
    f = ctx.field(comps) if field is None else field
    getattr(ctx, "deposit_" + name)(f)
    return f.export_internal()


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("clustered", [False, True])
@pytest.mark.parametrize("name,comps,fn", KINDS, ids=[k[0] for k in KINDS])
@pytest.mark.parametrize("mode", MODES)
def test_full_cic_matches_oracle(cuda, n, clustered, name, comps, fn, mode):
    npart = 6000
    cell, off, vel = small_case(n, npart, seed=11, vel_sigma=0.3, clustered=clustered)
    gm = 1.0 / npart
    ctx = _ctx(n, mode)
    _load(ctx, cell, off, vel, gm)
    got = _deposit(ctx, name, comps)
    ref = _oracle(fn, n, cell, off, vel, gm)
    for c in range(comps):
        assert normalized_error(got[c], ref[c]) < _tol(mode), (name, c)


@pytest.mark.parametrize("name,comps,fn", KINDS, ids=[k[0] for k in KINDS])
@pytest.mark.parametrize("mode", MODES)
def test_full_cic_individual_mass(cuda, name, comps, fn, mode):
    n = (24, 24, 24)
    cell, off, vel = small_case(n, 5000, seed=4, vel_sigma=0.2, clustered=True)
    m = ((1.0 + 0.5 * np.random.default_rng(5).uniform(-1, 1, 5000)) / 5000).astype(np.float32)
    ctx = _ctx(n, mode)
    _load(ctx, cell, off, vel, 0.0, mass=m)
    got = _deposit(ctx, name, comps)
    ref = _oracle(fn, n, cell, off, vel, 0.0, mass=m)
    for c in range(comps):
        assert normalized_error(got[c], ref[c]) < _tol(mode), (name, c)


@pytest.mark.parametrize("name,comps,fn", KINDS, ids=[k[0] for k in KINDS])
@pytest.mark.parametrize("mode", MODES)
def test_full_cic_dense_corner_cell_and_empty(cuda, name, comps, fn, mode):
    n = (32, 32, 32)
    ctx = _ctx(n, mode)
    e = np.zeros(0, np.int32)
    ctx.set_particles(e, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32),
                      global_mass=1.0)
    assert not np.any(_deposit(ctx, name, comps))
    # every particle in cell (31, 31, 31) or (0, 0, 0): offsets below and
    # above 1/2 reach the links of both neighbours across the periodic fold
    k = 4000
    rng = np.random.default_rng(2)
    cell = np.where(rng.random(k) < 0.5, 31 + 32 * (31 + 32 * 31), 0).astype(np.int32)
    off = rng.random((k, 3)).astype(np.float32)
    vel = (0.5 * rng.standard_normal((k, 3))).astype(np.float32)
    _load(ctx, cell, off, vel, 1.0 / k)
    got = _deposit(ctx, name, comps)
    ref = _oracle(fn, n, cell, off, vel, 1.0 / k)
    for c in range(comps):
        assert normalized_error(got[c], ref[c]) < _tol(mode), (name, c)


@pytest.mark.parametrize("name,comps,fn", KINDS, ids=[k[0] for k in KINDS])
@pytest.mark.parametrize("mode", MODES)
def test_full_cic_overwrites_the_field_and_repeats(cuda, name, comps, fn, mode):
    import torch
    n = (40, 40, 40)
    cell, off, vel = small_case(n, 20000, seed=9, vel_sigma=0.3, clustered=True)
    ctx = _ctx(n, mode)
    _load(ctx, cell, off, vel, 1.0 / 20000)
    buf = torch.full((comps, n[2], n[1], n[0]), 1e30, dtype=torch.float32, device="cuda")
    f = ctx.field(comps, buf)
    first = _deposit(ctx, name, comps, f)
    second = _deposit(ctx, name, comps, f)
    ref = _oracle(fn, n, cell, off, vel, 1.0 / 20000)
    for got in (first, second):
        for c in range(comps):
            assert normalized_error(got[c], ref[c]) < _tol(mode), (name, c)


def test_full_cic_sums_at_size(cuda):
    """Field sums equal the particle sums (FP64 on the host) at ~128^3 with
    4M uniform particles and ragged edges.  (A case that piles millions of
    particles onto a few vertices measures FP32 accumulation error instead:
    the positive T_ii terms then drift by ~1e-3.)"""
    n = (130, 128, 127)
    npart = 1 << 22
    cell, off, vel = small_case(n, npart, seed=13, vel_sigma=0.3, clustered=False)
    gm = 1.0 / npart
    res = 1.0 / n[0]
    ctx = _ctx(n)
    _load(ctx, cell, off, vel, gm)
    scale = gm / res ** 3
    v = vel.astype(np.float64)
    vf = _deposit(ctx, "vector_cic", 3).astype(np.float64)
    want = scale * v.sum(axis=0)
    got = vf.reshape(3, -1).sum(axis=1)
    assert np.abs(got - want).max() <= 1e-5 * scale * np.abs(v).sum(axis=0).max()
    tf = _deposit(ctx, "vecvec_cic", 6).astype(np.float64)
    pairs = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))
    got = tf.reshape(6, -1).sum(axis=1)
    for c, (i, j) in enumerate(pairs):
        want = scale * (v[:, i] * v[:, j]).sum()
        assert abs(got[c] - want) <= 1e-5 * scale * np.abs(v[:, i] * v[:, j]).sum(), c
