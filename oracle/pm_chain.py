"""FP64 restatement of the differentiable particle-mesh chain -- TEST
INFRASTRUCTURE ONLY (the checker of latfield2_b200.autodiff).

The forward operations restate the reference's CIC deposit
(particles/projections.hpp:142-179, rho = m/res^3 * prod of 1-D weights),
the CIC gather of updateVel's kick (LATfield2_Particles.hpp:825-842) and
move_particles_simple (move_function.hpp:30), in float64 torch on positions
in box units of a unit box.  Its gradients come from torch autograd on the
FP64 chain (the FP64 reference gradient) and are themselves checked against
central finite differences.

The grid operator is either the seeded 27-point stencil or the PM force of
the library's lf2_pm_force: the 7-point lattice Poisson equation
lap(phi) = coupling (rho - mean rho) solved by FFT with the Green's function
of the reference's Poisson example (examples/poissonSolver.cpp), then
F = -grad phi by central differences (torch.fft, differentiable; the same
arithmetic as oracle/fft_oracle.pm_force).
"""
import torch


def _corners(x, n):
    """x: (..., 3) float64 box units, res = 1/n[0] -> flat sites (..., 8) and
    weights (..., 8), differentiable in x."""
    u = x * float(n[0])
    c = torch.floor(u).detach()
    f = u - c
    ci = c.to(torch.int64)
    sites, weights = [], []
    for q in range(8):
        b = ((q >> 2) & 1, (q >> 1) & 1, q & 1)
        xyz = [torch.remainder(ci[..., d] + b[d], n[d]) for d in range(3)]
        sites.append(xyz[0] + n[0] * (xyz[1] + n[1] * xyz[2]))
        w = torch.ones_like(f[..., 0])
        for d in range(3):
            w = w * (f[..., d] if b[d] else 1.0 - f[..., d])
        weights.append(w)
    return torch.stack(sites, -1), torch.stack(weights, -1)


def _flat(sites, N):
    """Sites (B, np, 8) of B independent lattices of N sites -> indices into
    the (B * N) concatenation."""
    off = torch.arange(sites.shape[0], device=sites.device, dtype=torch.int64) * N
    return (sites + off[:, None, None]).reshape(-1)


def _deposit_b(sites, w, m, n):
    """Batched deposit: sites, w (B, np, 8), m (B, np) -> rho (B, N)."""
    B = sites.shape[0]
    N = n[0] * n[1] * n[2]
    vol = (1.0 / n[0]) ** 3  # res^3
    rho = torch.zeros(B * N, dtype=w.dtype, device=w.device)
    return rho.index_add(0, _flat(sites, N), (w * (m[..., None] / vol)).reshape(-1)).reshape(B, N)


def deposit(x, m, n):
    sites, w = _corners(x, n)
    return _deposit_b(sites[None], w[None], m[None], n)[0]


def _stencil_b(rho, S, n):
    """Batched stencil: rho (B, N), S (B, 81) -> F (B, 3, N).  Each of the 27
    shifted copies serves the three components; the terms are added in the
    offset order o = 0..26 for every component."""
    B = rho.shape[0]
    r = rho.reshape(B, n[2], n[1], n[0])
    acc = [torch.zeros_like(r) for _ in range(3)]
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                o = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)
                sh = torch.roll(r, shifts=(-dz, -dy, -dx), dims=(1, 2, 3))
                for c in range(3):
                    acc[c] = acc[c] + S[:, c * 27 + o, None, None, None] * sh
    return torch.stack([a.reshape(B, -1) for a in acc], 1)


def stencil(rho, S, n):
    """F_c(g) = sum_o S[c*27 + (dz+1)*9 + (dy+1)*3 + (dx+1)] rho(g + o), periodic."""
    return _stencil_b(rho[None], S[None], n)[0]


def _pm_force_b(rho, n, coupling):
    """Batched PM force: rho (B, N) -> F (B, 3, N) on a cubic lattice,
    res = 1/n[0]."""
    m = n[0]
    res = 1.0 / m
    B = rho.shape[0]
    r = rho.reshape(B, m, m, m)  # [b][z][y][x]
    K = torch.fft.rfftn(r, dim=(1, 2, 3))
    k = torch.arange(m, dtype=rho.dtype, device=rho.device)
    kx = k[: m // 2 + 1]
    c = lambda t: torch.cos(2.0 * torch.pi * t / m)
    lam = 2.0 * (c(kx)[None, None, :] + c(k)[None, :, None] + c(k)[:, None, None] - 3.0) / res ** 2
    zero = torch.zeros_like(lam, dtype=torch.bool)
    zero[0, 0, 0] = True
    G = torch.where(zero, torch.zeros_like(lam), coupling / torch.where(zero, torch.ones_like(lam),
                                                                         lam))
    phi = torch.fft.irfftn(K * G, s=(m, m, m), dim=(1, 2, 3))
    out = []
    for axis in (3, 2, 1):  # x, y, z
        out.append((-(torch.roll(phi, -1, axis) - torch.roll(phi, 1, axis)) / (2.0 * res))
                   .reshape(B, -1))
    return torch.stack(out, 1)


def pm_force(rho, n, coupling):
    """F[3][site] from rho[site] on a cubic lattice, res = 1/n[0]."""
    return _pm_force_b(rho[None], n, coupling)[0]


def _gather_b(sites, w, F, n):
    """Batched gather: sites, w (B, np, 8), F (B, 3, N) -> (B, np, 3)."""
    B = sites.shape[0]
    N = n[0] * n[1] * n[2]
    idx = _flat(sites, N)
    return torch.stack([(w * F[:, c].reshape(-1)[idx].reshape(w.shape)).sum(-1) for c in range(3)],
                       -1)


def gather(x, F, n):
    sites, w = _corners(x, n)
    return _gather_b(sites[None], w[None], F[None], n)[0]


def cells(x, n):
    """Cell index of every particle (the piece of the piecewise-smooth loss);
    x (..., 3)."""
    c = torch.remainder(torch.floor(x * float(n[0])).to(torch.int64),
                        torch.tensor(n, dtype=torch.int64, device=x.device))
    return c[..., 0] + n[0] * (c[..., 1] + n[1] * c[..., 2])


def _chain_b(x, v, m, S, wgt, n, steps, dt, coupling=None, ref_cells=None, record=False):
    """B chains at once: x, v (B, np, 3), m (B, np), S (B, 81) or None.
    Returns the losses (B,) and, with `record`, the cells of every particle
    at every deposit (steps + 1, B, np).  With `ref_cells` (steps + 1, np)
    the evaluation stops at the first deposit where a particle of any chain
    sits in another cell, and returns None."""
    seen = []
    for k in range(steps + 1):
        if record or ref_cells is not None:
            ck = cells(x.detach(), n)
            if record:
                seen.append(ck)
            if ref_cells is not None and not torch.equal(ck, ref_cells[k].expand_as(ck)):
                return None
        sites, w = _corners(x, n)
        rho = _deposit_b(sites, w, m, n)
        if k == steps:
            loss = (wgt.reshape(1, -1) * rho).sum(1)
            break
        F = _stencil_b(rho, S, n) if coupling is None else _pm_force_b(rho, n, coupling)
        v = v + dt * _gather_b(sites, w, F, n)
        x = x + dt * v
    return (loss, torch.stack(seen)) if record else loss


def chain_loss(pos0, vel0, mass, S, wgt, n, steps, dt, return_cells=False, coupling=None):
    """Same chain as latfield2_b200.autodiff.PMChain, in float64: the stencil
    S as grid operator, or the PM force when `coupling` is given (S is then
    not used).  With return_cells the cell of every particle at every
    deposit is returned too, so that a finite-difference check can verify
    that no particle crossed a face between its two evaluations (CIC is only
    piecewise smooth)."""
    r = _chain_b(pos0[None], vel0[None], mass[None], None if S is None else S[None], wgt, n,
                 steps, dt, coupling=coupling, record=return_cells)
    if return_cells:
        return r[0][0], r[1][:, 0]
    return r[0]


def reference_cells(base, wgt, n, steps, dt, coupling=None):
    """Cells of every particle at every deposit of the unperturbed chain
    (base = [pos0, vel0, mass, S]): the pieces a finite difference must stay
    in.  Computed once and passed to directional_fd for many directions."""
    _, c = chain_loss(*base, wgt, n, steps, dt, return_cells=True, coupling=coupling)
    return c


def directional_fd(base, u, wgt, n, steps, dt, eps=1e-7, min_eps=1e-12, coupling=None,
                   ref_cells=None):
    """Central difference of chain_loss along direction u (list matching
    base = [pos0, vel0, mass, S]; S may be None with the PM operator) with
    the largest eps <= `eps` for which no particle changes cell in any step
    between the +eps and -eps evaluations.  The two evaluations run as one
    batched chain that stops at the first deposit where a particle left its
    cell.  `ref_cells` (reference_cells) may be given to skip recomputing
    the unperturbed cells.  Returns (derivative, eps used)."""
    if ref_cells is None:
        ref_cells = reference_cells(base, wgt, n, steps, dt, coupling=coupling)
    while eps >= min_eps:
        pair = [None if t is None else torch.stack([t + eps * d, t - eps * d])
                for t, d in zip(base, u)]
        r = _chain_b(*pair, wgt, n, steps, dt, coupling=coupling, ref_cells=ref_cells)
        if r is not None:
            return float(r[0] - r[1]) / (2 * eps), eps
        eps /= 10.0
    return None, eps
