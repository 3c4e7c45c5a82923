"""Shared helpers of the test suite: seeded small cases and error measures."""
import numpy as np


def small_case(n, npart, seed, vel_sigma=0.01, clustered=False):
    """Particles in the device representation (cell, off, vel) as numpy."""
    rng = np.random.default_rng(seed)
    n = tuple(int(v) for v in n)
    if clustered:
        centre = rng.random(3)
        pos = np.mod(centre + 0.6 / max(n) * rng.standard_normal((npart, 3)), 1.0)
    else:
        pos = rng.random((npart, 3))
    u = pos * np.array(n, np.float64)
    fl = np.floor(u)
    off = (u - fl).astype(np.float32)
    carry = off >= 1.0
    off[carry] = 0.0
    fl = fl + carry
    ci = np.mod(fl.astype(np.int64), np.array(n))
    cell = (ci[:, 0] + n[0] * (ci[:, 1] + n[1] * ci[:, 2])).astype(np.int32)
    vel = (vel_sigma * rng.standard_normal((npart, 3))).astype(np.float32)
    return cell, off, vel


def cell_xyz(n, cell):
    c = np.asarray(cell, np.int64)
    return np.stack([c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1])], axis=1)


def positions(n, res, cell, off):
    return (cell_xyz(n, cell).astype(np.float64) + off.astype(np.float64)) * res


def normalized_error(got, ref):
    """max |got - ref| / max(max |ref|, tiny): the error relative to the
    field's scale (per-vertex relative error is undefined where ref ~ 0)."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    scale = max(np.max(np.abs(ref)), 1e-300)
    return float(np.max(np.abs(got - ref)) / scale)


def mean_relative_error(got, ref, floor_frac=1e-3):
    """Per-vertex relative error where |ref| exceeds floor_frac of its mean |ref|."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    m = np.abs(ref) > floor_frac * np.mean(np.abs(ref))
    if not np.any(m):
        return 0.0
    return float(np.max(np.abs(got[m] - ref[m]) / np.abs(ref[m])))


def precision(got, ref, mag=None, floor_frac=1e-2):
    """Error of a deposited field against its FP64 reference.
      norm_max / norm_rms: |got - ref| over the field's maximum |ref|;
      cell_max / cell_rms: per-vertex |got - ref| / mag, over the vertices
        where mag exceeds floor_frac of its mean.  mag is the vertex's sum of
        |contributions| (the FP64 deposit of |m v|, |m v_i v_j|; for the
        density mag = ref): the relative error of a sum, which stays defined
        where signed contributions cancel.
    """
    got = np.asarray(got, np.float64).reshape(-1)
    ref = np.asarray(ref, np.float64).reshape(-1)
    mag = np.abs(ref) if mag is None else np.asarray(mag, np.float64).reshape(-1)
    d = np.abs(got - ref)
    scale = max(float(np.max(np.abs(ref))), 1e-300)
    m = mag > floor_frac * float(np.mean(mag))
    rel = d[m] / mag[m] if np.any(m) else np.zeros(1)
    return {"norm_max": float(np.max(d) / scale), "norm_rms": float(np.sqrt(np.mean(d * d)) / scale),
            "cell_max": float(np.max(rel)), "cell_rms": float(np.sqrt(np.mean(rel * rel))),
            "floor_frac": floor_frac, "cells_above_floor": int(np.count_nonzero(m))}


def by_id(d, ids_key="id"):
    order = np.argsort(d[ids_key], kind="stable")
    return {k: v[order] for k, v in d.items()}


def internal_to_reference(F, halo):
    """(c, z, y, x) internal -> (z+2h, y+2h, x+2h, c) reference layout, halo filled
    periodically."""
    a = np.ascontiguousarray(np.asarray(F).transpose(1, 2, 3, 0))
    if halo:
        a = np.pad(a, ((halo, halo), (halo, halo), (halo, halo), (0, 0)), mode="wrap")
    return np.ascontiguousarray(a)


def slab_potential_emulated(engine_cls, rho, ranks, coupling, device=None):
    """The potential of the slab PM operator for `ranks` z slabs emulated in
    one process, the ranks one after the other (no collectives, nothing that
    waits): per rank an engine of the rank's local lattice, its plane
    transforms, the all-to-all transposes done here by slicing, the line
    transforms and the Green's function on each rank's k_y slab (ky0 = r nky).
    rho: torch tensor (n, n, n) on the engines' device.  Returns phi (n, n, n)."""
    import torch
    from latfield2_b200 import _lib
    n = int(rho.shape[0])
    nz = nky = n // ranks
    nkx = n // 2 + 1
    res = 1.0 / n
    kw = {} if device is None else {"device": device}
    eng = [engine_cls((n, n, nz + 2), res, _lib.DEPOSIT_FIXED64, **kw) for _ in range(ranks)]
    for e in eng:
        e.fft_prepare(n, nz, nky)
    A = []
    for r, e in enumerate(eng):
        a = e.complex_buffer((nz, n, nkx))
        e.planes_r2c(rho[r * nz:(r + 1) * nz].contiguous(), a)
        A.append(a)
    B = []
    for r, e in enumerate(eng):
        b = torch.cat([A[s][:, r * nky:(r + 1) * nky, :] for s in range(ranks)], 0).contiguous()
        e.lines(b, _lib.FFT_FORWARD)
        e.green(b, r * nky, coupling)
        e.lines(b, _lib.FFT_BACKWARD)
        B.append(b)
    phi = []
    for s, e in enumerate(eng):
        a = torch.cat([B[r][s * nz:(s + 1) * nz] for r in range(ranks)], 1).contiguous()
        p = torch.empty((nz, n, n), dtype=torch.float32, device=rho.device)
        e.planes_c2r(a, p)
        phi.append(p)
    return torch.cat(phi, 0)
