"""GPU parity of the PM grid operator (lf2_fft_forward / lf2_fft_backward /
lf2_pm_force, called through the C ABI) against the FP64 numpy oracle
(oracle/fft_oracle.py) and the reference's own PlanFFT outputs
(tests/golden/).

FP32 cuFFT: transforms within 1e-5 of the oracle, normalized by the largest
magnitude of the result; potential and force within 1e-5 of theirs.  The
k-field import/export round trip is exact.
"""
import glob
import os

import numpy as np
import pytest

from oracle import fft_oracle as FO
from tests.helpers import normalized_error, small_case

pytestmark = pytest.mark.gpu

GOLD = sorted(p for p in glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                "golden", "*_double.npz"))
              if "fft_k" in np.load(p))


def _ctx(n):
    import latfield2_b200 as L
    return L.Context((n, n, n), box=1.0, mode=0)


def _real_field(ctx, a):
    """a[z][y][x] (one component) -> a device field."""
    f = ctx.field(1)
    f.import_(np.ascontiguousarray(np.asarray(a, np.float64)[..., None]))
    return f


@pytest.mark.parametrize("n", [8, 16, 48, 64])
def test_forward_and_backward_match_oracle(cuda, n):
    rng = np.random.default_rng(n)
    rho = rng.standard_normal((n, n, n))
    ctx = _ctx(n)
    r = _real_field(ctx, rho)
    k = ctx.kfield(1)
    ctx.fft_forward(r, k)
    got = k.export()[..., 0]
    want = FO.rfft_ref(rho)
    assert normalized_error(got.real, want.real) < 1e-5
    assert normalized_error(got.imag, want.imag) < 1e-5
    back = ctx.field(1)
    ctx.fft_backward(k, back)
    assert normalized_error(back.export()[..., 0], n ** 3 * rho) < 1e-5
    # the k-field is kept by the backward transform
    np.testing.assert_array_equal(k.export()[..., 0], got)


def test_kfield_import_export_round_trip_and_components(cuda):
    n = 16
    ctx = _ctx(n)
    k = ctx.kfield(3)
    rng = np.random.default_rng(1)
    a = (rng.standard_normal((n, n, n // 2 + 1, 3)) +
         1j * rng.standard_normal((n, n, n // 2 + 1, 3))).astype(np.complex64)
    k.import_(a)
    np.testing.assert_array_equal(k.export(np.complex64), a)
    # per-component transforms of a 3-component field
    F = rng.standard_normal((n, n, n, 3))
    f = ctx.field(3)
    f.import_(np.ascontiguousarray(F))
    ctx.fft_forward(f, k)
    got = k.export()
    for c in range(3):
        want = FO.rfft_ref(F[..., c])
        assert normalized_error(got[..., c].real, want.real) < 1e-5
        assert normalized_error(got[..., c].imag, want.imag) < 1e-5


@pytest.mark.parametrize("path", GOLD, ids=lambda p: os.path.basename(p))
def test_fft_and_poisson_match_the_reference(cuda, path):
    """The reference's PlanFFT forward / backward and its Poisson example
    (tests/golden/, 1x1 and 2x2 process grids) against the GPU."""
    g = dict(np.load(path))
    n = int(g["n"])
    rho = g["F"][..., 0]
    ctx = _ctx(n)
    r = _real_field(ctx, rho)
    k = ctx.kfield(1)
    ctx.fft_forward(r, k)
    got = k.export()[..., 0]
    assert normalized_error(got.real, g["fft_k"].real) < 1e-5
    assert normalized_error(got.imag, g["fft_k"].imag) < 1e-5
    k.import_(g["fft_k"][..., None].copy())
    back = ctx.field(1)
    ctx.fft_backward(k, back)
    assert normalized_error(back.export()[..., 0], g["fft_back"]) < 1e-5
    # pm_force's potential with coupling 1 is the example's phi / n^3
    phi, F = ctx.field(1), ctx.field(3)
    ctx.pm_force(r, F, 1.0, phi=phi)
    assert normalized_error(phi.export()[..., 0] * n ** 3, g["poisson"]) < 1e-5


@pytest.mark.parametrize("n", [9, 10, 16, 64])
def test_pm_force_matches_oracle(cuda, n):
    """n = 9: an odd count of k values (the Green's function's last value
    alone) and the one-site gradient path; n = 10: the one-site gradient path;
    16, 64: the four-site path."""
    cell, off, vel = small_case((n, n, n), 20 * n ** 3 // 8, seed=3, clustered=True)
    ctx = _ctx(n)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / cell.shape[0])
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    rho_h = rho.export()[..., 0].astype(np.float64)
    phi, F = ctx.field(1), ctx.field(3)
    ctx.pm_force(rho, F, 4.0, phi=phi)
    want_phi, want_F = FO.pm_force(rho_h, 1.0 / n, 4.0)
    assert normalized_error(phi.export()[..., 0], want_phi) < 1e-5
    got_F = F.export()
    for c in range(3):
        assert normalized_error(got_F[..., c], want_F[c]) < 1e-5, c
    # without phi the same force
    F2 = ctx.field(3)
    ctx.pm_force(rho, F2, 4.0)
    assert normalized_error(F2.export(), got_F) < 1e-6


def test_pm_force_at_size(cuda):
    """256^3, 16M particles: potential and force against the FP64 oracle, and
    the force sums to zero."""
    n = 256
    cell, off, vel = small_case((n, n, n), n ** 3, seed=5, clustered=False)
    ctx = _ctx(n)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / cell.shape[0])
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    phi, F = ctx.field(1), ctx.field(3)
    ctx.pm_force(rho, F, 1.0, phi=phi)
    want_phi, want_F = FO.pm_force(rho.export()[..., 0].astype(np.float64), 1.0 / n, 1.0)
    assert normalized_error(phi.export()[..., 0], want_phi) < 1e-5
    f = F.export().astype(np.float64)
    for c in range(3):
        assert normalized_error(f[..., c], want_F[c]) < 1e-5, c
    assert np.abs(f.reshape(-1, 3).sum(axis=0)).max() < 1e-6 * np.abs(f).sum() / 3


def test_pm_force_into_a_misaligned_field(cuda):
    """A force field wrapped at an address that is not 16-byte aligned takes
    the one-site gradient path and gives the same result."""
    import torch
    n = 32
    cell, off, vel = small_case((n, n, n), 40000, seed=8, clustered=True)
    ctx = _ctx(n)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / cell.shape[0])
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    F = ctx.field(3)
    ctx.pm_force(rho, F, 1.0)
    buf = torch.zeros(3 * n ** 3 + 1, dtype=torch.float32, device="cuda")
    Fm = ctx.field(3, buf[1:])
    ctx.pm_force(rho, Fm, 1.0)
    np.testing.assert_array_equal(Fm.export(), F.export())


def test_non_cubic_lattice_is_refused(cuda):
    import latfield2_b200 as L
    ctx = L.Context((16, 16, 8), box=1.0, mode=0)
    r, k = ctx.field(1), ctx.kfield(1)
    with pytest.raises(L.LF2Error, match="cubic"):
        ctx.fft_forward(r, k)
