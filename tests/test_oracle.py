"""CPU tests of the oracle: analytic known answers of the CIC projections
(derived from particles/projections.hpp:142-179), conservation laws and the
agreement of the two oracle layers.  No GPU needed."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import (cell_xyz, internal_to_reference, normalized_error, positions,
                           small_case)

N8 = (8, 8, 8)


def _ref_scalar(n, cell, off, gmass, prec="d", halo=1, pmass=None):
    res = 1.0 / n[0]
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    pm = None if pmass is None else np.asarray(pmass, np.float64)[order]
    rho = O.scalar_cic(n, halo, res, cs, pos, pm, gmass, prec=prec)
    return O.interior(rho, n, halo)[0]


def test_vertex_particle_deposits_everything_on_its_vertex():
    n = N8
    cell = np.array([3 + 8 * (4 + 8 * 5)], np.int32)
    off = np.zeros((1, 3), np.float32)
    rho = _ref_scalar(n, cell, off, gmass=2.0)
    res = 1.0 / 8
    assert rho[5, 4, 3] == pytest.approx(2.0 / res ** 3, rel=1e-14)
    assert np.count_nonzero(rho) == 1


def test_cell_centre_particle_splits_in_eight():
    n = N8
    x, y, z = 7, 0, 7  # upper corner: exercises the periodic fold
    cell = np.array([x + 8 * (y + 8 * z)], np.int32)
    off = np.full((1, 3), 0.5, np.float32)
    rho = _ref_scalar(n, cell, off, gmass=1.0)
    res = 1.0 / 8
    expect = 1.0 / (8 * res ** 3)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                assert rho[(z + dz) % 8, (y + dy) % 8, (x + dx) % 8] == pytest.approx(expect, rel=1e-13)
    assert np.count_nonzero(rho) == 8


@pytest.mark.parametrize("prec", ["d", "f"])
def test_one_particle_per_cell_gives_uniform_density(prec):
    n = (6, 5, 7)
    nc = n[0] * n[1] * n[2]
    cell = np.arange(nc, dtype=np.int32)
    off = np.full((nc, 3), 0.25, np.float32)
    res = 1.0 / 6
    rho = _ref_scalar(n, cell, off, gmass=0.5, prec=prec) if n[0] == 6 else None
    tol = 1e-12 if prec == "d" else 3e-6
    np.testing.assert_allclose(rho, 0.5 / res ** 3, rtol=tol)


@pytest.mark.parametrize("prec", ["d", "f"])
def test_scalar_mass_conservation(prec):
    n = (12, 12, 12)
    cell, off, _ = small_case(n, 3000, seed=5)
    res = 1.0 / 12
    rho = _ref_scalar(n, cell, off, gmass=1.0 / 3000, prec=prec)
    tol = 1e-12 if prec == "d" else 2e-6
    assert np.sum(rho, dtype=np.float64) * res ** 3 == pytest.approx(1.0, rel=tol)


def test_fold_equals_direct_periodic_deposit():
    """project + comm of the reference layout == periodic deposit (layer B)."""
    for n, halo in (((8, 8, 8), 1), ((9, 7, 5), 2), ((16, 16, 16), 1)):
        cell, off, _ = small_case(n, 2000, seed=11, clustered=True)
        res = 1.0 / n[0]
        rho = _ref_scalar(n, cell, off, gmass=1e-3, halo=halo)
        direct = O.state_deposit_f64(n, cell, off, res, gmass=1e-3).reshape(n[2], n[1], n[0])
        assert normalized_error(rho, direct) < 1e-13


def test_individual_mass_deposit():
    n = (8, 8, 8)
    cell, off, _ = small_case(n, 500, seed=3)
    rng = np.random.default_rng(4)
    m = (1.0 + 0.1 * rng.uniform(-1, 1, 500)).astype(np.float32) / 500
    res = 1.0 / 8
    rho = _ref_scalar(n, cell, off, gmass=0.0, pmass=m)
    direct = O.state_deposit_f64(n, cell, off, res, mass=m).reshape(8, 8, 8)
    assert normalized_error(rho, direct) < 1e-13
    assert np.sum(rho) * res ** 3 == pytest.approx(np.sum(m, dtype=np.float64), rel=1e-12)


def test_fixed_point_weights_are_exact_partitions():
    rng = np.random.default_rng(0)
    for _ in range(200):
        f = rng.random(3).astype(np.float32)
        tot = sum(O.fixed_weight(f[0], f[1], f[2], (k >> 2) & 1, (k >> 1) & 1, k & 1)
                  for k in range(8))
        assert abs(tot - 2 ** 32) <= 4
    assert O.fixed_weight(0.0, 0.0, 0.0, 0, 0, 0) == 2 ** 32
    assert O.fixed_weight(0.5, 0.5, 0.5, 1, 0, 1) == 2 ** 29


def test_fixed_point_deposit_matches_fp64():
    n = (16, 16, 16)
    cell, off, _ = small_case(n, 20000, seed=8, clustered=True)
    res = 1.0 / 16
    gm = 1.0 / 20000
    acc = O.state_deposit_fixed(n, cell, off)
    assert abs(int(acc.sum()) - 20000 * 2 ** 32) <= 8 * 20000
    scale = np.float32(2.0 ** -32 * gm / res ** 3)
    rho = O.fixed_to_f32(acc, scale)
    ref = O.state_deposit_f64(n, cell, off, res, gmass=gm)
    assert normalized_error(rho, ref) < 1e-6


def test_vector_and_tensor_conserve_momentum_and_stress():
    n = (10, 12, 8)
    cell, off, vel = small_case(n, 1500, seed=21, vel_sigma=0.3)
    res = 1.0 / 10
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    v = vel.astype(np.float64)[order]
    gm = 2e-3
    vec = O.interior(O.vector_cicngp(n, 1, res, cs, pos, v, gmass=gm), n, 1)
    ten = O.interior(O.symtensor_cicngp(n, 1, res, cs, pos, v, gmass=gm), n, 1)
    for c in range(3):
        assert vec[c].sum() * res ** 3 == pytest.approx(gm * v[:, c].sum(), rel=1e-11)
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    for k, (i, j) in enumerate(pairs):
        assert ten[k].sum() * res ** 3 == pytest.approx(gm * (v[:, i] * v[:, j]).sum(), rel=1e-11)


def test_vector_ngp_direction():
    """A particle at offset (0.3, 0.6, 0.9) puts v_x only on its own x vertex."""
    n = (8, 8, 8)
    cell = np.array([2 + 8 * (3 + 8 * 4)], np.int32)
    off = np.array([[0.3, 0.6, 0.9]], np.float32)
    vel = np.array([[1.0, 0.0, 0.0]])
    res = 1.0 / 8
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)
    vec = O.interior(O.vector_cicngp(n, 1, res, cs, pos, vel, gmass=1.0), n, 1)
    nz = np.argwhere(vec[0] != 0)
    assert set(map(tuple, nz[:, [2]])) == {(2,)}  # x stays at the particle's cell
    assert len(nz) == 4
    assert np.count_nonzero(vec[1]) == 0 and np.count_nonzero(vec[2]) == 0


def test_update_halo_is_periodic_image():
    n = (5, 6, 7)
    rng = np.random.default_rng(1)
    inner = rng.standard_normal((3,) + (n[2], n[1], n[0]))
    for halo in (1, 2):
        f = np.zeros((n[2] + 2 * halo, n[1] + 2 * halo, n[0] + 2 * halo, 3))
        f[halo:-halo, halo:-halo, halo:-halo, :] = inner.transpose(1, 2, 3, 0)
        O.update_halo(f, n, halo)
        np.testing.assert_array_equal(f, internal_to_reference(inner, halo))


def test_kick_layers_agree():
    """Reference restatement (double, halo'd field) vs device restatement (FP32).
    The reference's gather uses frac = pos * N - coord (LATfield2_Particles.hpp:
    825-828), i.e. a unit box, so the lattice is cubic here."""
    n = (12, 12, 12)
    cell, off, vel = small_case(n, 2000, seed=13)
    F = np.random.default_rng(2).standard_normal((3, n[2], n[1], n[0])).astype(np.float32)
    res = 1.0 / 12
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    v_ref = vel.astype(np.float64)[order].copy()
    Fh = internal_to_reference(F.astype(np.float64), 1)
    maxv, _ = O.update_vel_cic(n, 1, cs, pos, v_ref, Fh, 0.05)
    v_dev = O.state_kick(n, cell, off, vel, F, np.float32(0.05))[order]
    np.testing.assert_allclose(v_dev, v_ref, rtol=0, atol=2e-6 * np.abs(v_ref).max())
    assert maxv == pytest.approx(np.sqrt((v_ref ** 2).sum(1)).max(), rel=1e-12)


def test_drift_layers_agree_except_on_faces():
    n = (16, 16, 16)
    cell, off, vel = small_case(n, 5000, seed=17, vel_sigma=0.05)
    res = 1.0 / 16
    dtau = 0.3
    pos = positions(n, res, cell, off)
    new_cell_ref = O.move_simple(n, 1.0, pos, vel.astype(np.float64), dtau)
    c2, o2, bad = O.state_drift(n, cell, off, vel, np.float32(dtau / res))
    assert bad == 0
    u = pos / res
    near_face = np.any(np.abs(u - np.round(u)) < 1e-4, axis=1)
    assert np.all((c2 == new_cell_ref) | near_face)
    assert np.mean(c2 != cell) > 0.05  # some particles changed cell
    pos_dev = positions(n, res, c2, o2)
    d = np.abs(pos_dev - pos)
    d = np.minimum(d, 1.0 - d)
    assert d.max() < 1e-6


def test_rebin_lists_is_a_permutation_in_new_cells():
    n = (6, 6, 6)
    cell, off, vel = small_case(n, 800, seed=2)
    cs, order = O.lists_from_insertion(n, cell)
    newc = np.roll(cell, 7)
    cs2, order2 = O.rebin_lists(n, cs, order, newc)
    assert sorted(order2.tolist()) == list(range(800))
    for c in range(216):
        assert np.all(newc[order2[cs2[c]:cs2[c + 1]]] == c)


def test_cell_xyz_roundtrip():
    n = (5, 7, 3)
    c = np.arange(105)
    xyz = cell_xyz(n, c)
    assert np.all(xyz[:, 0] + 5 * (xyz[:, 1] + 7 * xyz[:, 2]) == c)


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
@pytest.mark.parametrize("clustered", [False, True])
def test_fixed_point_momentum_and_stress_match_the_reference_projections(kind, clustered):
    """The integer restatement of the fixed-point momentum / stress deposits
    (layer B) puts every contribution on the vertex the reference's
    projection does (layer A, FP64), to the quantum of the fixed point."""
    n = (12, 10, 9)
    cell, off, vel = small_case(n, 3000, seed=60 + kind, vel_sigma=0.2, clustered=clustered)
    res = 1.0 / n[0]
    gm = 1.0 / 3000
    acc, e = O.state_deposit_fixed_kind(kind, n, cell, off, vel)
    got = O.fixed_kind_to_f32(acc, kind, e, gm, res)
    cs, order = O.lists_from_insertion(n, cell)
    pos = positions(n, res, cell, off)[order]
    v = vel.astype(np.float64)[order]
    fn = {1: O.vector_cicngp, 2: O.symtensor_cicngp, 3: O.vector_cic, 4: O.vecvec_cic}[kind]
    ref = O.interior(fn(n, 1, res, cs, pos, v, gmass=gm), n, 1)
    for c in range(ref.shape[0]):
        assert normalized_error(got[c], ref[c]) < 1e-6, c


def test_fixed_point_velocity_unit():
    """V = 2^e is the smallest power of two above every |v_i|."""
    for vmax, e in ((0.02, -5), (0.5, 0), (1.0, 1), (3.0, 2), (2.0 ** -30, -29)):
        v = np.array([[vmax, -vmax / 3, 0.0]], np.float32)
        assert O.vexp(v) == e, (vmax, O.vexp(v))
        assert 2.0 ** (e - 1) <= vmax < 2.0 ** e
    assert O.vexp(np.zeros((4, 3), np.float32)) == 0
    assert O.vexp(np.full((1, 3), 1e-35, np.float32)) == -96
