"""Full-size check of the differentiable chain (not collected by pytest):
the CUDA adjoint of the 8-step chain at 128^3 with 2,097,152 particles
against the FP64 reference gradient and FP64 central finite differences
along random directions, with eps chosen per direction so that no particle
changes cell between the two evaluations.

    python tests/adjoint_fd_check.py [--dirs 1000]
"""
import argparse
import json
import os
import sys
import time

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import latfield2_b200 as L  # noqa: E402
from latfield2_b200.autodiff import pm_chain_loss, positions_to_state  # noqa: E402
from oracle import pm_chain as P  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dirs", type=int, default=1000)
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--npart", type=int, default=1 << 21)
    a = ap.parse_args()
    n, npart, steps, dt = a.n, a.npart, 8, 0.1 * 64.0 / a.n
    dev = "cuda"
    g = torch.Generator(device=dev).manual_seed(41)
    pos = torch.rand(npart, 3, generator=g, device=dev, dtype=torch.float64)
    vel = (0.01 * torch.randn(npart, 3, generator=g, device=dev, dtype=torch.float64)).float().double()
    m = ((1.0 + 0.1 * (2 * torch.rand(npart, generator=g, device=dev, dtype=torch.float64) - 1))
         / npart).float().double()
    S = (0.02 * torch.randn(81, generator=g, device=dev, dtype=torch.float64)).float().double()
    w = torch.randn(n ** 3, generator=g, device=dev, dtype=torch.float64).float().double()
    cell, off = positions_to_state(pos, (n, n, n), 1.0 / n)
    c = cell.long()
    pos = (torch.stack([c % n, (c // n) % n, c // (n * n)], 1).double() + off.double()) / n
    ctx = L.Context((n, n, n), box=1.0)
    leaves = [t.clone().requires_grad_(True) for t in (pos, vel, m, S, w)]
    pm_chain_loss(ctx, *leaves, steps=steps, dt=dt).backward()
    got = [t.grad for t in leaves]
    ref_leaves = [t.clone().requires_grad_(True) for t in (pos, vel, m, S, w)]
    ref = torch.autograd.grad(P.chain_loss(*ref_leaves, (n, n, n), steps, dt), ref_leaves)
    rel = {k: float((a_ - b_).norm() / b_.norm())
           for k, a_, b_ in zip(("pos", "vel", "mass", "stencil", "weights"), got, ref)}
    rng = np.random.default_rng(11)
    base = [pos, vel, m, S]
    fd, dv, rf, epss = [], [], [], []
    t0 = time.time()
    for _ in range(a.dirs):
        us = [torch.from_numpy(rng.standard_normal(tuple(t.shape))).to(dev) for t in base]
        nrm = float(torch.sqrt(sum((u ** 2).sum() for u in us)))
        us = [u / nrm for u in us]
        with torch.no_grad():
            d, eps = P.directional_fd(base, us, w, (n, n, n), steps, dt, eps=1e-7)
        if d is None:
            continue
        fd.append(d)
        epss.append(eps)
        dv.append(float(sum((gg * u).sum() for gg, u in zip(got[:4], us))))
        rf.append(float(sum((gg * u).sum() for gg, u in zip(ref[:4], us))))
    fd, dv, rf = map(np.array, (fd, dv, rf))
    scale = float(np.sqrt(np.mean(fd ** 2)))
    out = {"n": n, "particles": npart, "steps": steps, "directions": len(fd),
           "grad_rel_err_vs_fp64": rel,
           "fd_max_err_ref_over_rms": float(np.max(np.abs(rf - fd)) / scale),
           "fd_max_err_cuda_over_rms": float(np.max(np.abs(dv - fd)) / scale),
           "fd_median_rel_err_cuda": float(np.median(np.abs(dv - fd) / np.abs(fd))),
           "eps_used": sorted(set(epss)), "seconds": time.time() - t0}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
