"""CPU checks of the FP64 chain that serves as the reference gradient of the
differentiable PM chain: its autograd gradient agrees with central finite
differences along random directions, and its forward conserves mass."""
import numpy as np
import pytest
import torch

from oracle import pm_chain as P


def _setup(n=8, npart=300, seed=0):
    g = torch.Generator().manual_seed(seed)
    pos = torch.rand(npart, 3, generator=g, dtype=torch.float64)
    vel = 0.02 * torch.randn(npart, 3, generator=g, dtype=torch.float64)
    m = (1.0 + 0.1 * (2 * torch.rand(npart, generator=g, dtype=torch.float64) - 1)) / npart
    S = 0.01 * torch.randn(81, generator=g, dtype=torch.float64)
    w = torch.randn(n ** 3, generator=g, dtype=torch.float64)
    return (n, n, n), pos, vel, m, S, w


def test_deposit_conserves_mass():
    n, pos, vel, m, S, w = _setup()
    rho = P.deposit(pos, m, n)
    assert float(rho.sum()) / n[0] ** 3 == pytest.approx(float(m.sum()), rel=1e-13)


def test_stencil_adjoint_identity():
    n, pos, vel, m, S, w = _setup()
    rho = torch.randn(n[0] ** 3, dtype=torch.float64)
    gF = torch.randn(3, n[0] ** 3, dtype=torch.float64)
    # <S rho, gF> = <rho, S^T gF> through autograd
    r = rho.clone().requires_grad_(True)
    (P.stencil(r, S, n) * gF).sum().backward()
    lhs = float((P.stencil(rho, S, n) * gF).sum())
    assert float((r.grad * rho).sum()) == pytest.approx(lhs, rel=1e-12)


def test_fp64_gradient_matches_finite_differences():
    n, pos, vel, m, S, w = _setup(n=8, npart=300, seed=3)
    steps, dt = 4, 0.5
    leaves = [t.clone().requires_grad_(True) for t in (pos, vel, m, S)]
    loss = P.chain_loss(*leaves, w, n, steps, dt)
    grads = torch.autograd.grad(loss, leaves)
    rng = np.random.default_rng(5)
    eps = 1e-7
    for _ in range(20):
        us = [torch.from_numpy(rng.standard_normal(t.shape)) for t in (pos, vel, m, S)]
        norm = float(torch.sqrt(sum((u ** 2).sum() for u in us)))
        us = [u / norm for u in us]
        fd, used = P.directional_fd([pos, vel, m, S], us, w, n, steps, dt, eps=eps)
        assert fd is not None
        an = float(sum((g * u).sum() for g, u in zip(grads, us)))
        assert an == pytest.approx(fd, rel=1e-5, abs=1e-6 * float(torch.sqrt(sum((g ** 2).sum() for g in grads))))


def test_pm_force_matches_the_fft_oracle():
    from oracle import fft_oracle as FO
    n = 16
    rho = torch.rand(n ** 3, generator=torch.Generator().manual_seed(2), dtype=torch.float64)
    F = P.pm_force(rho, (n, n, n), 4 * np.pi)
    _, ref = FO.pm_force(rho.reshape(n, n, n).numpy(), 1.0 / n, 4 * np.pi)
    np.testing.assert_allclose(F.numpy(), ref.reshape(3, -1), rtol=0, atol=1e-14)


def test_pm_force_adjoint_is_divergence_then_the_same_solve():
    """The structure of lf2_pm_force4_adjoint: g_rho = G(div g_F), with
    div_c the transpose of the central difference and G the Green's-function
    solve itself (self-adjoint)."""
    n = 12
    g = torch.Generator().manual_seed(4)
    rho = torch.randn(n ** 3, generator=g, dtype=torch.float64)
    gF = torch.randn(3, n ** 3, generator=g, dtype=torch.float64)
    r = rho.clone().requires_grad_(True)
    (P.pm_force(r, (n, n, n), 3.0) * gF).sum().backward()
    res = 1.0 / n
    gf = gF.reshape(3, n, n, n)
    div = sum(torch.roll(gf[c], -1, axis) - torch.roll(gf[c], 1, axis)
              for c, axis in zip(range(3), (2, 1, 0))) / (2 * res)
    # the forward operator's Green's-function solve, applied to the divergence
    K = torch.fft.rfftn(div)
    k = torch.arange(n, dtype=torch.float64)
    cs = lambda t: torch.cos(2 * torch.pi * t / n)
    lam = 2 * (cs(k[: n // 2 + 1])[None, None, :] + cs(k)[None, :, None] + cs(k)[:, None, None]
               - 3) / res ** 2
    lam[0, 0, 0] = 1.0
    Gk = 3.0 / lam
    Gk[0, 0, 0] = 0.0
    want = torch.fft.irfftn(K * Gk, s=(n, n, n)).reshape(-1)
    np.testing.assert_allclose(r.grad.numpy(), want.numpy(), rtol=0,
                               atol=1e-12 * float(want.abs().max()))


def test_fp64_pm_chain_gradient_matches_finite_differences():
    n, pos, vel, m, S, w = _setup(n=8, npart=300, seed=6)
    steps, dt, coupling = 4, 0.5, 4 * np.pi
    leaves = [t.clone().requires_grad_(True) for t in (pos, vel, m)]
    loss = P.chain_loss(*leaves, S, w, n, steps, dt, coupling=coupling)
    grads = torch.autograd.grad(loss, leaves)
    rng = np.random.default_rng(8)
    gnorm = float(torch.sqrt(sum((g ** 2).sum() for g in grads)))
    for _ in range(20):
        us = [torch.from_numpy(rng.standard_normal(t.shape)) for t in (pos, vel, m)]
        norm = float(torch.sqrt(sum((u ** 2).sum() for u in us)))
        us = [u / norm for u in us] + [torch.zeros_like(S)]
        fd, used = P.directional_fd([pos, vel, m, S], us, w, n, steps, dt, eps=1e-7,
                                    coupling=coupling)
        assert fd is not None
        an = float(sum((g * u).sum() for g, u in zip(grads, us)))
        assert an == pytest.approx(fd, rel=1e-5, abs=1e-6 * gnorm)
