"""CPU oracle of the PM grid operator: the reference's real-to-complex
PlanFFT, its Poisson example, and the force the library derives from it.

TEST INFRASTRUCTURE ONLY: imported by tests/ and the smoke check, always as
the checker of the CUDA path.  FP64 numpy.

Reference semantics restated here (pinned against the reference's own
PlanFFT, compiled over the FFTW-interface stand-in oracle/fftw_shim, by the
fixtures of tests/golden/):
  - PlanFFT<Imag>::execute(FFT_FORWARD) (LATfield2_PlanFFT_decl.hpp:855-948):
    K(k) = sum_x rho(x) exp(-2 pi i k.x / n), not normalised, k_x = 0 .. n/2.
    The Fourier lattice (Lattice::initializeRealFFT, LATfield2_Lattice.hpp:
    225-258) has sizes (n/2+1, n, n); rKSite reads coord(1) from storage dim 2
    and coord(2) from storage dim 1 (LATfield2_Site.hpp:319-338), so the
    k-field is stored [k_y][k_z][k_x] (outermost first).
  - execute(FFT_BACKWARD) (:949-1050): the inverse transform, not normalised
    (n^3 times the input after a forward transform).
  - the Poisson example (examples/poissonSolver.cpp): phi_k = rho_k /
    (2 (cos(2 pi k_0/n) + cos(2 pi k_1/n) + cos(2 pi k_2/n) - 3) / res^2),
    phi_0 = 0, then FFT_BACKWARD: n^3 times the solution of the 7-point
    lattice Poisson equation for rho minus its mean.
"""
import numpy as np


def rfft_ref(rho):
    """rho[z][y][x] -> K[ky][kz][kx] (complex128), FFT_FORWARD."""
    return np.ascontiguousarray(np.fft.rfftn(np.asarray(rho, np.float64)).transpose(1, 0, 2))


def irfft_ref(K):
    """K[ky][kz][kx] -> real field [z][y][x], FFT_BACKWARD (not normalised)."""
    K = np.asarray(K).transpose(1, 0, 2)
    n = K.shape[0]
    return np.fft.irfftn(K, s=(n, n, n), axes=(0, 1, 2)) * float(n) ** 3


def laplacian_eigenvalues(n, res):
    """2 (cos(2 pi k_x/n) + cos(2 pi k_y/n) + cos(2 pi k_z/n) - 3) / res^2 on
    the cuFFT/numpy layout [kz][ky][kx]."""
    kz = np.arange(n)[:, None, None]
    ky = np.arange(n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    return 2.0 * (np.cos(2 * np.pi * kx / n) + np.cos(2 * np.pi * ky / n) +
                  np.cos(2 * np.pi * kz / n) - 3.0) / (res * res)


def poisson_example(rho, res):
    """The reference's Poisson example: n^3 phi (see the module docstring)."""
    rho = np.asarray(rho, np.float64)
    n = rho.shape[0]
    K = np.fft.rfftn(rho)
    lam = laplacian_eigenvalues(n, res)
    lam[0, 0, 0] = 1.0
    P = K / lam
    P[0, 0, 0] = 0.0
    return np.fft.irfftn(P, s=(n, n, n), axes=(0, 1, 2)) * float(n) ** 3


def pm_force(rho, res, coupling):
    """The library's PM operator: phi solves the 7-point lattice Poisson
    equation lap(phi) = coupling (rho - mean(rho)) (the example's Green's
    function, normalised), and F_i = -(phi(x + e_i) - phi(x - e_i)) / (2 res),
    periodic.  Returns (phi[z][y][x], F[3][z][y][x])."""
    phi = poisson_example(rho, res) * (coupling / float(np.asarray(rho).shape[0]) ** 3)
    F = np.empty((3,) + phi.shape)
    for c, axis in enumerate((2, 1, 0)):  # x is the last numpy axis
        F[c] = -(np.roll(phi, -1, axis) - np.roll(phi, 1, axis)) / (2.0 * res)
    return phi, F
