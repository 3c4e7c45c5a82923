"""Pins the oracle (layer A) against the reference itself: the fixtures in
tests/golden/ hold outputs of the reference's own particle path compiled
from its sources (see tests/golden/make_golden.py).

Single-rank cases must match bit for bit: the oracle restates the reference's
arithmetic statement by statement and rebuilds its per-cell list order.  The
2x2-rank cases fold the halos through messages in a different order, so
their deposits are compared to a tight tolerance; their moves are bit-exact.
The full-CIC projections (vectorProjectionCIC, VecVecProjectionCIC) exist only
in the 2x2 cases: their reference folds (sendUpDown) cannot run on a grid with
one rank along a dim.
"""
import glob
import os

import numpy as np
import pytest

from oracle import fft_oracle as FO
from oracle import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(glob.glob(os.path.join(HERE, "*.npz")))


def load(path):
    return dict(np.load(path))


def real_of(path):
    return (np.float32, "f") if path.endswith("_single.npz") else (np.float64, "d")


def ref_cells(n, posR, R):
    """getPartCoord: (int)floor(pos * N) % N in the build's Real
    (LATfield2_Particles.hpp:463-467)."""
    u = np.floor(posR * R(n)).astype(np.int64) % n
    return (u[:, 0] + n * (u[:, 1] + n * u[:, 2])).astype(np.int32)


def test_fixtures_present():
    names = {os.path.basename(p) for p in CASES}
    for case in ("uniform8", "clustered12", "ranks16", "ranks20"):
        for b in ("double", "single"):
            assert f"{case}_{b}.npz" in names
    for b in ("double", "single"):
        for case in ("ranks16", "ranks20"):
            g = load(os.path.join(HERE, f"{case}_{b}.npz"))
            assert "vcic" in g and "vv" in g


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p) for p in CASES])
def test_oracle_matches_reference(path):
    g = load(path)
    R, prec = real_of(path)
    n = int(g["n"])
    halo = int(g["halo"])
    nn = (n, n, n)
    single_rank = int(np.prod(g["grid"])) == 1
    res = R(1.0) / R(n)  # get_lattice_resolution in Real (particles_tools.hpp:6-19)
    posR = g["pos"].astype(R)
    velR = g["vel"].astype(R)
    ids = g["ids"]
    cell = ref_cells(n, posR, R)
    cs, order = O.lists_from_insertion(nn, cell)
    pos_l, vel_l, ids_l = posR[order], velR[order].copy(), ids[order]

    tol = 0.0 if single_rank else (1e-13 if prec == "d" else 1e-6)
    for key, fn in (("rho", O.scalar_cic), ("vec", O.vector_cicngp), ("ten", O.symtensor_cicngp),
                    ("vcic", O.vector_cic), ("vv", O.vecvec_cic)):
        if key not in g:
            continue
        if key == "rho":
            f = fn(nn, halo, res, cs, pos_l.astype(np.float64 if prec == "d" else np.float32),
                   None, float(g["gmass"]), prec=prec)
        else:
            f = fn(nn, halo, res, cs, pos_l, vel_l, None, float(g["gmass"]), prec=prec)
        got = f[halo:halo + n, halo:halo + n, halo:halo + n, :]
        want = g[key]
        if tol == 0.0:
            np.testing.assert_array_equal(got.astype(np.float64), want, err_msg=key)
        else:
            scale = np.abs(want).max()
            assert np.abs(got - want).max() <= tol * scale, key

    if "F_halo" in g:
        F = O.projection_init(nn, halo, 3, prec)
        F[halo:halo + n, halo:halo + n, halo:halo + n, :] = g["F"].astype(R)
        O.update_halo(F, nn, halo, prec)
        np.testing.assert_array_equal(F.astype(np.float64), g["F_halo"])

    if "kick_vel" in g:
        Fh = O.projection_init(nn, halo, 3, prec)
        Fh[halo:halo + n, halo:halo + n, halo:halo + n, :] = g["F"].astype(R)
        O.update_halo(Fh, nn, halo, prec)
        maxv, _ = O.update_vel_cic(nn, halo, cs, pos_l, vel_l, Fh, float(g["dtau_kick"]), prec)
        k = np.argsort(ids_l)
        np.testing.assert_array_equal(ids_l[k], g["kick_id"])
        np.testing.assert_array_equal(vel_l[k].astype(np.float64), g["kick_vel"])
        np.testing.assert_array_equal(pos_l[k].astype(np.float64), g["kick_pos"])
        assert maxv == g["maxv"]

    if "move_pos" in g:
        # moveParticles(move_particles_simple) after the kick, on the 2x2 grid
        k = np.argsort(ids_l)
        p = pos_l[k].copy()
        v = vel_l[k]
        O.move_simple(nn, R(1.0), p, v, float(g["dtau_move"]), prec)
        np.testing.assert_array_equal(g["move_id"], np.sort(ids))
        np.testing.assert_array_equal(p.astype(np.float64), g["move_pos"])
        np.testing.assert_array_equal(v.astype(np.float64), g["move_vel"])


def test_full_cic_projections_conserve_momentum_and_stress():
    """Sum over sites of the vector-CIC field is the total momentum m sum v /
    res^3 and of the VecVec field the total m sum v_i v_j / res^3: the
    staggered weights of a particle sum to one along every dim."""
    for path in CASES:
        g = load(path)
        if "vcic" not in g:
            continue
        n = int(g["n"])
        tol = 1e-12 if path.endswith("_double.npz") else 1e-4
        scale = float(g["gmass"]) * n ** 3
        v = g["vel"]
        mom = scale * v.sum(axis=0)
        np.testing.assert_allclose(g["vcic"].reshape(-1, 3).sum(axis=0), mom,
                                   rtol=tol, atol=tol * np.abs(mom).max())
        pairs = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))
        want = np.array([scale * (v[:, i] * v[:, j]).sum() for i, j in pairs])
        np.testing.assert_allclose(g["vv"].reshape(-1, 6).sum(axis=0), want,
                                   rtol=tol, atol=tol * np.abs(want).max())


@pytest.mark.parametrize("path", [p for p in CASES if "fft_k" in np.load(p)],
                         ids=lambda p: os.path.basename(p))
def test_fft_oracle_matches_reference(path):
    """The reference's PlanFFT (forward and backward) and its Poisson example,
    run on 1x1 and 2x2 grids, against the numpy restatement: round-off only
    (the reference ran over a plain-DFT stand-in of FFTW)."""
    g = load(path)
    R, prec = real_of(path)
    n = int(g["n"])
    rho = g["F"][..., 0].astype(R).astype(np.float64)
    tol = 1e-12 if prec == "d" else 1e-6
    K = FO.rfft_ref(rho)
    assert np.abs(K - g["fft_k"]).max() <= tol * np.abs(K).max()
    back = FO.irfft_ref(g["fft_k"])
    assert np.abs(back - g["fft_back"]).max() <= tol * np.abs(back).max()
    phi = FO.poisson_example(rho, 1.0 / n)
    assert np.abs(phi - g["poisson"]).max() <= tol * np.abs(phi).max()


def test_pm_force_oracle_properties():
    """The force of a point mass points at it and the potential satisfies the
    7-point Poisson equation exactly (to round-off)."""
    n = 16
    res = 1.0 / n
    rho = np.zeros((n, n, n))
    rho[5, 6, 7] = 1.0
    phi, F = FO.pm_force(rho, res, 2.0)
    lap = sum(np.roll(phi, s, a) for a in range(3) for s in (1, -1)) - 6 * phi
    np.testing.assert_allclose(lap / res ** 2, 2.0 * (rho - rho.mean()), atol=1e-9)
    # x+1 neighbour of the mass: force along -x (towards the mass)
    assert F[0][5, 6, 8] < 0 and F[0][5, 6, 6] > 0
    assert abs(F.sum()) < 1e-9


def test_reference_conserves_mass_in_every_fixture():
    for path in CASES:
        g = load(path)
        n = int(g["n"])
        if "rho" in g:
            R, prec = real_of(path)
            tol = 1e-12 if prec == "d" else 1e-5
            assert g["rho"].sum() / n ** 3 == pytest.approx(1.0, rel=tol), path
