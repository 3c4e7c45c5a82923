"""Known-answer tests of the FFT oracle, after the reference's own FFT checks:
a plane wave has its two Fourier coefficients and nothing else
(benchmarks_tests/wave_test.cpp:7,145, TOLERANCE 1e-10), and the Poisson
example on an eigenfunction of the lattice Laplacian returns n^3 times that
eigenfunction over its eigenvalue (examples/poissonSolver.cpp:117-158,
TOLERANCE 1e-11 in double).  The PM force of a plane wave is its analytic
central difference."""
import numpy as np
import pytest

from oracle import fft_oracle as FO

N = 16


def _wave(k):
    z, y, x = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    return 2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) / N


@pytest.mark.parametrize("k", [(1, 0, 0), (3, 2, 0), (2, 5, 7), (0, 0, 8)])
def test_plane_wave_has_two_coefficients(k):
    K = FO.rfft_ref(np.cos(_wave(k)))  # [ky][kz][kx]
    want = np.zeros_like(K)
    for s in (1, -1):  # with k_x = 0 or n/2 both coefficients lie in the stored half
        kx, ky, kz = (s * k[0]) % N, (s * k[1]) % N, (s * k[2]) % N
        if kx <= N // 2:
            want[ky, kz, kx] += N ** 3 / 2
    assert np.abs(K - want).max() <= 1e-10 * N ** 3
    back = FO.irfft_ref(K)
    assert np.abs(back - N ** 3 * np.cos(_wave(k))).max() <= 1e-10 * N ** 3


@pytest.mark.parametrize("k", [(1, 0, 0), (2, 3, 1), (4, 4, 4)])
def test_poisson_example_on_an_eigenfunction(k):
    res = 1.0 / N
    rho = np.cos(_wave(k))
    lam = 2 * (sum(np.cos(2 * np.pi * kd / N) for kd in k) - 3) / res ** 2
    got = FO.poisson_example(rho, res)
    want = N ** 3 * rho / lam
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()


def test_pm_force_of_a_plane_wave():
    res, coupling = 1.0 / N, 4 * np.pi
    k = (2, 1, 3)
    rho = 1.0 + np.cos(_wave(k))  # the mean is removed by the solve
    lam = 2 * (sum(np.cos(2 * np.pi * kd / N) for kd in k) - 3) / res ** 2
    phi, F = FO.pm_force(rho, res, coupling)
    np.testing.assert_allclose(phi, coupling * np.cos(_wave(k)) / lam, rtol=0,
                               atol=1e-12 * abs(coupling / lam))
    for c in range(3):
        # -(cos(a + t) - cos(a - t)) / (2 res) = sin(a) sin(t) / res, t = 2 pi k_c / N
        want = coupling / lam * np.sin(_wave(k)) * np.sin(2 * np.pi * k[c] / N) / res
        assert np.abs(F[c] - want).max() <= 1e-11 * np.abs(want).max()
