"""Deposit precision of the three modes against the FP64 references of the
reference's own projections (projections.hpp, restated in oracle layer A),
and bit-exactness of the fixed-point mode against the oracle's integer
restatement (layer B), for every projection:

  kind 0  scalarProjectionCIC          kind 1  vectorProjectionCICNGP
  kind 2  symtensorProjectionCICNGP    kind 3  vectorProjectionCIC
  kind 4  VecVecProjectionCIC

Tolerances (tests.helpers.precision):
  - FP32 mode (compensated atomics) and fixed-point mode: error <= 1e-6 of the
    field maximum, and <= 1e-6 of the vertex's sum of |contributions| on every
    vertex where that sum exceeds 1e-2 of its mean (the relative error of a
    sum, defined where signed momenta cancel).
  - fixed point: bit-exact against the oracle; the same bits for any particle
    order.
  - plain FP32 mode: 1e-5 of the field maximum (unordered FP32 atomics).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import positions, precision, small_case

pytestmark = pytest.mark.gpu

KINDS = {1: ("deposit_vector", 3, O.vector_cicngp), 2: ("deposit_symtensor", 6, O.symtensor_cicngp),
         3: ("deposit_vector_cic", 3, O.vector_cic), 4: ("deposit_vecvec_cic", 6, O.vecvec_cic)}


def _ctx(n, mode):
    import latfield2_b200 as L
    return L.Context(n, box=tuple(v / n[0] for v in n), mode=mode)


def _deposit(n, mode, kind, cell, off, vel, gm, perm=None):
    ctx = _ctx(n, mode)
    if perm is not None:
        cell, off, vel = cell[perm], off[perm], vel[perm]
    ctx.set_particles(cell, off, vel, global_mass=gm)
    if kind == 0:
        f = ctx.field(1)
        ctx.deposit_scalar(f)
    else:
        name, comps, _ = KINDS[kind]
        f = ctx.field(comps)
        getattr(ctx, name)(f)
    out = f.export_internal()
    assert ctx.flags() == 0
    ctx.close()
    return out


def _fp64(n, kind, cell, off, vel, gm):
    """FP64 reference of the projection and its |contribution| sums."""
    res = 1.0 / n[0]
    if kind == 0:
        ref = O.state_deposit_f64(n, cell, off, res, gmass=gm).reshape(1, n[2], n[1], n[0])
        return ref, np.abs(ref)
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    v = vel.astype(np.float64)[order]
    fn = KINDS[kind][2]
    ref = O.interior(fn(n, 1, res, cs, pos, v, gmass=gm), n, 1)
    mag = O.interior(fn(n, 1, res, cs, pos, np.abs(v), gmass=gm), n, 1)
    return ref, mag


CASES = [((8, 8, 8), 5000, False), ((20, 20, 20), 5000, True), ((33, 17, 24), 8000, True),
         ((32, 32, 32), 120000, True)]


@pytest.mark.parametrize("n,npart,clustered", CASES)
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("mode", [0, 1])
def test_deposits_within_1e6_of_fp64(cuda, n, npart, clustered, kind, mode):
    cell, off, vel = small_case(n, npart, seed=17 + kind, vel_sigma=0.2, clustered=clustered)
    gm = 1.0 / npart
    got = _deposit(n, mode, kind, cell, off, vel, gm)
    ref, mag = _fp64(n, kind, cell, off, vel, gm)
    for c in range(ref.shape[0]):
        p = precision(got[c], ref[c], mag[c])
        assert p["norm_max"] <= 1e-6, (c, p)
        assert p["cell_max"] <= 1e-6, (c, p)


@pytest.mark.parametrize("n,npart,clustered", CASES)
@pytest.mark.parametrize("kind", [1, 2, 3, 4])
def test_fixed_point_momentum_and_stress_are_bit_exact(cuda, n, npart, clustered, kind):
    cell, off, vel = small_case(n, npart, seed=29 + kind, vel_sigma=0.3, clustered=clustered)
    gm = 1.0 / npart
    got = _deposit(n, 1, kind, cell, off, vel, gm)
    acc, e = O.state_deposit_fixed_kind(kind, n, cell, off, vel)
    want = O.fixed_kind_to_f32(acc, kind, e, gm, 1.0 / n[0])
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
def test_fixed_point_momentum_and_stress_ignore_particle_order(cuda, kind):
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 60000, seed=41, vel_sigma=0.1, clustered=True)
    outs = [_deposit(n, 1, kind, cell, off, vel, 1.0 / 60000,
                     perm=np.random.default_rng(s).permutation(cell.shape[0]))
            for s in (0, 1, 2)]
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_plain_fp32_mode(cuda, kind):
    import latfield2_b200 as L
    n = (20, 20, 20)
    cell, off, vel = small_case(n, 6000, seed=3, vel_sigma=0.2, clustered=True)
    got = _deposit(n, L.DEPOSIT_FP32_PLAIN, kind, cell, off, vel, 1.0 / 6000)
    ref, _ = _fp64(n, kind, cell, off, vel, 1.0 / 6000)
    for c in range(ref.shape[0]):
        assert precision(got[c], ref[c])["norm_max"] < 1e-5, c


def test_individual_masses_in_the_fixed_point_momentum(cuda):
    """Per-particle masses: the relative mass m / unit (unit = mean mass)
    scales each contribution; bit-exact against the oracle."""
    n = (24, 24, 24)
    cell, off, vel = small_case(n, 5000, seed=4, vel_sigma=0.1)
    rng = np.random.default_rng(5)
    m = ((1.0 + 0.1 * rng.uniform(-1, 1, 5000)) / 5000).astype(np.float32)
    unit = float(np.sum(m.astype(np.float64)) / 5000)
    mrel = (m * np.float32(1.0 / unit)).astype(np.float32)
    for kind in (1, 2, 3, 4):
        name, comps, _ = KINDS[kind]
        ctx = _ctx(n, 1)
        ctx.set_particles(cell, off, vel, mass=m)
        f = ctx.field(comps)
        getattr(ctx, name)(f)
        acc, e = O.state_deposit_fixed_kind(kind, n, cell, off, vel, mrel=mrel)
        want = O.fixed_kind_to_f32(acc, kind, e, unit, 1.0 / 24)
        np.testing.assert_array_equal(f.export_internal(), want)
        ctx.close()
