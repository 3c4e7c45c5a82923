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
