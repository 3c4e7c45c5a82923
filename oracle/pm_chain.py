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
    """x: (np, 3) float64 box units, res = 1/n[0] -> flat sites (np, 8) and
    weights (np, 8), differentiable in x."""
    nn = torch.tensor(n, dtype=torch.int64, device=x.device)
    u = x * float(n[0])
    c = torch.floor(u).detach()
    f = u - c
    ci = torch.remainder(c.to(torch.int64), nn)
    sites, weights = [], []
    for q in range(8):
        b = ((q >> 2) & 1, (q >> 1) & 1, q & 1)
        xyz = [torch.remainder(ci[:, d] + b[d], n[d]) for d in range(3)]
        sites.append(xyz[0] + n[0] * (xyz[1] + n[1] * xyz[2]))
        w = torch.ones_like(f[:, 0])
        for d in range(3):
            w = w * (f[:, d] if b[d] else 1.0 - f[:, d])
        weights.append(w)
    return torch.stack(sites, 1), torch.stack(weights, 1)


def deposit(x, m, n):
    sites, w = _corners(x, n)
    vol = (1.0 / n[0]) ** 3  # res^3
    rho = torch.zeros(n[0] * n[1] * n[2], dtype=x.dtype, device=x.device)
    return rho.index_add(0, sites.reshape(-1), (w * (m[:, None] / vol)).reshape(-1))


def stencil(rho, S, n):
    """F_c(g) = sum_o S[c*27 + (dz+1)*9 + (dy+1)*3 + (dx+1)] rho(g + o), periodic."""
    r = rho.reshape(n[2], n[1], n[0])
    out = []
    for c in range(3):
        acc = torch.zeros_like(r)
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    o = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)
                    acc = acc + S[c * 27 + o] * torch.roll(r, shifts=(-dz, -dy, -dx), dims=(0, 1, 2))
        out.append(acc.reshape(-1))
    return torch.stack(out)


def pm_force(rho, n, coupling):
    """F[3][site] from rho[site] on a cubic lattice, res = 1/n[0]."""
    m = n[0]
    res = 1.0 / m
    r = rho.reshape(m, m, m)  # [z][y][x]
    K = torch.fft.rfftn(r)
    k = torch.arange(m, dtype=rho.dtype, device=rho.device)
    kx = k[: m // 2 + 1]
    c = lambda t: torch.cos(2.0 * torch.pi * t / m)
    lam = 2.0 * (c(kx)[None, None, :] + c(k)[None, :, None] + c(k)[:, None, None] - 3.0) / res ** 2
    zero = torch.zeros_like(lam, dtype=torch.bool)
    zero[0, 0, 0] = True
    G = torch.where(zero, torch.zeros_like(lam), coupling / torch.where(zero, torch.ones_like(lam),
                                                                         lam))
    phi = torch.fft.irfftn(K * G, s=(m, m, m))
    out = []
    for axis in (2, 1, 0):  # x, y, z
        out.append((-(torch.roll(phi, -1, axis) - torch.roll(phi, 1, axis)) / (2.0 * res))
                   .reshape(-1))
    return torch.stack(out)


def gather(x, F, n):
    sites, w = _corners(x, n)
    return torch.stack([(w * F[c][sites]).sum(1) for c in range(3)], 1)


def cells(x, n):
    """Cell index of every particle (the piece of the piecewise-smooth loss)."""
    c = torch.remainder(torch.floor(x * float(n[0])).to(torch.int64),
                        torch.tensor(n, dtype=torch.int64, device=x.device))
    return c[:, 0] + n[0] * (c[:, 1] + n[1] * c[:, 2])


def chain_loss(pos0, vel0, mass, S, wgt, n, steps, dt, return_cells=False, coupling=None):
    """Same chain as latfield2_b200.autodiff.PMChain, in float64: the stencil
    S as grid operator, or the PM force when `coupling` is given (S is then
    not used).  With return_cells the cell of every particle at every
    deposit is returned too, so that a finite-difference check can verify
    that no particle crossed a face between its two evaluations (CIC is only
    piecewise smooth)."""
    x, v = pos0, vel0
    seen = []
    for _ in range(steps):
        if return_cells:
            seen.append(cells(x.detach(), n))
        rho = deposit(x, mass, n)
        F = stencil(rho, S, n) if coupling is None else pm_force(rho, n, coupling)
        v = v + dt * gather(x, F, n)
        x = x + dt * v
    if return_cells:
        seen.append(cells(x.detach(), n))
    loss = (wgt.reshape(-1) * deposit(x, mass, n)).sum()
    return (loss, torch.stack(seen)) if return_cells else loss


def _shifted(base, u, eps):
    """base + eps u, entry by entry; None entries (an unused S) stay None."""
    return [None if t is None else t + eps * d for t, d in zip(base, u)]


def directional_fd(base, u, wgt, n, steps, dt, eps=1e-7, min_eps=1e-12, coupling=None):
    """Central difference of chain_loss along direction u (list matching
    base = [pos0, vel0, mass, S]; S may be None with the PM operator) with
    the largest eps <= `eps` for which no particle changes cell in any step
    between the +eps and -eps evaluations.  Returns (derivative, eps used)."""
    _, ref_cells = chain_loss(*base, wgt, n, steps, dt, return_cells=True, coupling=coupling)
    while eps >= min_eps:
        lp, cp = chain_loss(*_shifted(base, u, eps), wgt, n, steps, dt, return_cells=True,
                            coupling=coupling)
        lm, cm = chain_loss(*_shifted(base, u, -eps), wgt, n, steps, dt, return_cells=True,
                            coupling=coupling)
        if torch.equal(cp, ref_cells) and torch.equal(cm, ref_cells):
            return float(lp - lm) / (2 * eps), eps
        eps /= 10.0
    return None, eps
