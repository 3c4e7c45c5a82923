"""Seeded synthetic inputs with the shapes and distributions of the
particle-mesh workloads (all in the library's device representation).

Every generator returns int32 cell indices (c = x + n0*(y + n1*z)), FP32
in-cell offsets in [0,1) (shape (np, 3)) and FP32 velocities in box units per
time, as torch tensors on `device` (CPU tensors work for small cases).

  uniform      positions U[0,1)^3 of the box
  clumps       half uniform, half in Gaussian clumps (sigma in box units)
  lognormal    log-normal density: delta_G a Gaussian field with P(k) ~ k^-2,
               rho ~ exp(s*delta_G - s^2/2), cells drawn from rho (multinomial
               by inverse CDF), uniform in-cell offsets
  halos        a uniform fraction plus Gaussian halos
  grf_gradient a Gaussian random scalar field with P(k) ~ k^-2 and its
               central-difference gradient at the vertices (3 components)
"""

import torch


def _gen(seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def positions_to_state(pos, n):
    """pos in box units of a unit box, shape (np, 3) float64 -> cell, off."""
    n_t = torch.tensor(n, dtype=torch.float64, device=pos.device)
    u = pos * n_t
    fl = torch.floor(u)
    off = (u - fl).to(torch.float32)
    carry = (off >= 1.0)
    off = torch.where(carry, torch.zeros_like(off), off)
    fl = fl + carry.to(fl.dtype)
    ci = fl.to(torch.int64)
    ci = torch.remainder(ci, torch.tensor(n, dtype=torch.int64, device=pos.device))
    cell = ci[:, 0] + n[0] * (ci[:, 1] + n[1] * ci[:, 2])
    return cell.to(torch.int32), off.contiguous()


def velocities(npart, sigma, seed, device="cpu"):
    g = _gen(seed, device)
    return (torch.randn(npart, 3, generator=g, device=device, dtype=torch.float32) * sigma).contiguous()


def uniform(n, npart, seed, device="cpu"):
    g = _gen(seed, device)
    pos = torch.rand(npart, 3, generator=g, device=device, dtype=torch.float64)
    return positions_to_state(pos, n)


def clumps(n, npart, nclumps, sigma, seed, device="cpu", frac_uniform=0.5):
    g = _gen(seed, device)
    nu = int(round(npart * frac_uniform))
    nc = npart - nu
    pos_u = torch.rand(nu, 3, generator=g, device=device, dtype=torch.float64)
    centres = torch.rand(nclumps, 3, generator=g, device=device, dtype=torch.float64)
    which = torch.randint(0, nclumps, (nc,), generator=g, device=device)
    pos_c = centres[which] + sigma * torch.randn(nc, 3, generator=g, device=device,
                                                 dtype=torch.float64)
    pos = torch.remainder(torch.cat([pos_u, pos_c]), 1.0)
    return positions_to_state(pos, n)


def halos(n, npart, nhalos, sigma, seed, device="cpu", frac_halo=0.1):
    return clumps(n, npart, nhalos, sigma, seed, device, frac_uniform=1.0 - frac_halo)


def gaussian_field(n, seed, device="cpu", slope=-2.0):
    """Real Gaussian random field on n^3 (unit variance) with P(k) ~ k^slope."""
    g = _gen(seed, device)
    n0, n1, n2 = n
    white = torch.randn(n2, n1, n0, generator=g, device=device, dtype=torch.float32)
    wk = torch.fft.rfftn(white)
    kz = torch.fft.fftfreq(n2, device=device) * n2
    ky = torch.fft.fftfreq(n1, device=device) * n1
    kx = torch.fft.rfftfreq(n0, device=device) * n0
    k2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    amp = torch.where(k2 > 0, k2.clamp_min(1e-12) ** (slope / 4.0), torch.zeros_like(k2))
    f = torch.fft.irfftn(wk * amp, s=(n2, n1, n0))
    f = f - f.mean()
    return (f / f.std()).contiguous()


def lognormal(n, npart, seed, device="cpu", sigma_ln=2.0):
    delta = gaussian_field(n, seed, device)
    rho = torch.exp(sigma_ln * delta.to(torch.float64) - 0.5 * sigma_ln * sigma_ln).reshape(-1)
    # integer weights (2^-20 units of the mean density): their prefix sum is
    # exact in any order, so the particles are the same bits in every run
    # (a floating-point scan on the GPU rounds in a timing-dependent order)
    cdf = torch.cumsum(torch.floor(rho * 1048576.0).to(torch.int64), 0).to(torch.float64)
    cdf = cdf / cdf[-1]
    g = _gen(seed + 1, device)
    u = torch.rand(npart, generator=g, device=device, dtype=torch.float64)
    cell = torch.searchsorted(cdf, u).clamp_max(rho.numel() - 1).to(torch.int32)
    del cdf, rho, delta
    off = torch.rand(npart, 3, generator=g, device=device, dtype=torch.float32)
    off = torch.where(off >= 1.0, torch.zeros_like(off), off)
    return cell, off.contiguous()


def grf_gradient(n, seed, device="cpu", amplitude=1.0):
    """3-component force field (internal layout (3, n2, n1, n0)): central
    differences of a Gaussian random field, scaled to `amplitude` rms."""
    phi = gaussian_field(n, seed, device)
    comps = []
    for axis in (2, 1, 0):  # x is the last torch dim
        comps.append(0.5 * (torch.roll(phi, -1, axis) - torch.roll(phi, 1, axis)))
    F = torch.stack(comps)
    F = F * (amplitude / F.std())
    return F.to(torch.float32).contiguous()


def sort_by_cell(cell, *arrays):
    """Stable sort by cell (useful to build reference-order lists)."""
    order = torch.argsort(cell.to(torch.int64), stable=True)
    return (cell[order],) + tuple(a[order] for a in arrays)


def algorithmic_bytes(npart, nsites, c_dep=1, c_gat=3, per_particle=28, mass_bytes=0):
    """Bytes one full step must move at minimum: particle state read once and
    written once, deposited components written once, gathered read once."""
    return npart * (2 * per_particle + mass_bytes) + nsites * 4 * (c_dep + c_gat)


def ceil_div(a, b):
    return -(-a // b)


__all__ = ["uniform", "clumps", "halos", "lognormal", "grf_gradient", "gaussian_field",
           "velocities", "positions_to_state", "algorithmic_bytes", "sort_by_cell", "math"]
