"""The workload configurations at their full sizes on a B200.

C2: 256^3 lattice, 16,777,216 particles (half uniform, half in 64 Gaussian
    clumps of sigma 0.01 box), FP32 mode, the force the central-difference
    gradient of a Gaussian random field.  Ten leapfrog steps (CIC gather-kick,
    drift, rebin), each compared with the oracle's FP32 restatement of the
    device arithmetic bit for bit (cells, offsets, velocities by id); then
    the scalar, vector CIC-NGP and symtensor CIC-NGP deposits of the final
    state against the FP64 references (1e-5 of the field maximum).
C3: 512^3 lattice, 134,217,728 log-normal particles, fixed-point deposit:
    three runs (fresh contexts, the particles loaded in three different
    orders) give the same density bits, after the first deposit and after two
    steps.
"""
import hashlib

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import normalized_error

pytestmark = pytest.mark.gpu


def test_c2_ten_steps_against_the_oracle(cuda):
    import torch
    import latfield2_b200 as L
    import latfield2_b200.workloads as W
    n = (256, 256, 256)
    npart = 256 ** 3
    res = 1.0 / 256
    dtau = 0.1 * 64 / 256
    cell, off = W.clumps(n, npart, 64, 0.01, seed=3, device="cuda")
    vel = W.velocities(npart, 0.01, seed=4, device="cuda")
    F = W.grf_gradient(n, seed=2, device="cuda", amplitude=0.01)
    ids = torch.arange(npart, dtype=torch.int64, device="cuda")
    ctx = L.Context(n, box=1.0, mode=L.DEPOSIT_FP32)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / npart, ids=ids)
    Fh = ctx.field(3, F)
    c, o, v = cell.cpu().numpy(), off.cpu().numpy(), vel.cpu().numpy()
    Fn = F.cpu().numpy()
    moved = 0
    for _ in range(10):
        ctx.step(Fh, dtau, dtau, None)
        v = O.state_kick(n, c, o, v, Fn, np.float32(dtau))
        c_new, o, bad = O.state_drift(n, c, o, v, np.float32(dtau / res))
        assert bad == 0
        moved += int((c_new != c).sum())
        c = c_new
        got = ctx.get_particles(ids=True)
        order = np.argsort(got["id"])
        np.testing.assert_array_equal(got["cell"][order], c)
        np.testing.assert_array_equal(got["off"][order], o)
        np.testing.assert_array_equal(got["vel"][order], v)
    assert moved > 100000  # the rebin had work to do
    gm = 1.0 / npart
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    ref = O.state_deposit_f64(n, c, o, res, gmass=gm)
    assert normalized_error(rho.export_internal().reshape(-1), ref) < 1e-5
    cs, order = O.lists_from_insertion(n, c)
    xyz = np.stack([c % 256, (c // 256) % 256, c // 65536], axis=1).astype(np.float64)
    pos = ((xyz + o.astype(np.float64)) * res)[order]
    vv = v.astype(np.float64)[order]
    vf, tf = ctx.field(3), ctx.field(6)
    ctx.deposit_vector(vf)
    ctx.deposit_symtensor(tf)
    vref = O.interior(O.vector_cicngp(n, 1, res, cs, pos, vv, gmass=gm), n, 1)
    tref = O.interior(O.symtensor_cicngp(n, 1, res, cs, pos, vv, gmass=gm), n, 1)
    vg, tg = vf.export_internal(), tf.export_internal()
    for k in range(3):
        assert normalized_error(vg[k], vref[k]) < 1e-5, k
    for k in range(6):
        assert normalized_error(tg[k], tref[k]) < 1e-5, k


def test_c3_fixed_point_density_is_bit_exact_across_runs(cuda):
    import torch
    import latfield2_b200 as L
    import latfield2_b200.workloads as W
    n = (512, 512, 512)
    npart = 512 ** 3
    dtau = 0.1 * 64 / 512
    cell, off = W.lognormal(n, npart, seed=3, device="cuda")
    vel = W.velocities(npart, 0.01, seed=4, device="cuda")
    F = W.grf_gradient(n, seed=2, device="cuda", amplitude=0.01)
    digests = []
    for run in range(3):
        if run == 0:
            c, o, v = cell, off, vel
        else:
            g = torch.Generator(device="cuda")
            g.manual_seed(100 + run)
            perm = torch.randperm(npart, generator=g, device="cuda")
            c, o, v = cell[perm].contiguous(), off[perm].contiguous(), vel[perm].contiguous()
            del perm
        ctx = L.Context(n, box=1.0, mode=L.DEPOSIT_FIXED64)
        ctx.set_particles(c, o, v, global_mass=1.0 / npart)
        del c, o, v
        rho_t = torch.empty(n[0] * n[1] * n[2], dtype=torch.float32, device="cuda")
        rho = ctx.field(1, rho_t)
        ctx.deposit_scalar(rho)
        ctx.synchronize()
        d0 = hashlib.sha256(rho_t.cpu().numpy().tobytes()).hexdigest()
        Fh = ctx.field(3, F)
        for _ in range(2):
            ctx.step(Fh, dtau, dtau, rho)
        ctx.synchronize()
        d1 = hashlib.sha256(rho_t.cpu().numpy().tobytes()).hexdigest()
        digests.append((d0, d1))
        del rho, Fh
        ctx.close()
        torch.cuda.empty_cache()
    assert digests[0] == digests[1] == digests[2], digests
    assert digests[0][0] != digests[0][1]  # the steps changed the density
