"""The C++ layer with LATfield2's names (include/latfield2_b200.hpp).

CPU: tests/compat/compat_demo.cpp, a particle-mesh loop written like a
reference user's (Lattice, Field, Particles<part_simple, ...>, the
projection functions, updateVel(cic_gather_kick), moveParticles
(move_particles_simple)), builds against the header and liblf2gpu.so in
double and with -DSINGLE.

GPU: the demo's results equal those of the same operations through the
Python binding of the same library: fixed-point density and particles
bit-exact, the FP32 vector and tensor projections (CIC-NGP and full CIC)
within 1e-5 of the field maximum (the order of FP32 additions differs run to
run)."""
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

from tests.helpers import normalized_error

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "compat"))


def _build(tmp_path, single=False):
    import build_demo
    out = str(tmp_path / ("demo_single" if single else "demo_double"))
    return build_demo.build(out, single)


@pytest.mark.parametrize("single", [False, True])
def test_demo_builds_against_the_header(tmp_path, single):
    assert os.path.exists(_build(tmp_path, single))


def _read(path):
    arrays = []
    with open(path, "rb") as f:
        while True:
            h = f.read(8)
            if not h:
                break
            (n,) = struct.unpack("q", h)
            arrays.append(np.frombuffer(f.read(8 * n), dtype=np.float64))
    return arrays


@pytest.mark.gpu
def test_demo_matches_the_python_binding(cuda, tmp_path):
    import torch
    import latfield2_b200 as L
    exe = _build(tmp_path)
    out = str(tmp_path / "demo.bin")
    n, npart = 32, 20000
    r = subprocess.run([exe, str(n), str(npart), out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    (hdr, id0, pos0, vel0, rho0, Fv, id1, pos1, vel1, rho1, B, T, V, VV) = _read(out)
    N, count, dtau, maxv = int(hdr[0]), int(hdr[1]), hdr[2], hdr[3]
    assert N == n and count == npart
    ctx = L.Context((n, n, n), box=1.0, mode=L.DEPOSIT_FIXED64)
    ctx.set_positions(pos0.reshape(-1, 3), vel0.reshape(-1, 3), global_mass=1.0 / npart,
                      ids=id0.astype(np.int64))
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    np.testing.assert_array_equal(rho.export(0, np.float64).reshape(-1), rho0)
    Fi = torch.from_numpy(np.ascontiguousarray(
        Fv.reshape(n, n, n, 3).transpose(3, 0, 1, 2)).astype(np.float32)).cuda()
    F = ctx.field(3, Fi)
    mv = ctx.gather_kick(F, dtau, want_max_v=True)
    assert mv == maxv
    ctx.drift_rebin(dtau)
    ctx.deposit_scalar(rho)
    np.testing.assert_array_equal(rho.export(0, np.float64).reshape(-1), rho1)
    pos, vel, ids = ctx.get_positions(ids=True)
    k, k1 = np.argsort(ids), np.argsort(id1)
    np.testing.assert_array_equal(ids[k], id1[k1].astype(np.int64))
    np.testing.assert_array_equal(pos[k], pos1.reshape(-1, 3)[k1])
    np.testing.assert_array_equal(vel[k], vel1.reshape(-1, 3)[k1])
    v, t = ctx.field(3), ctx.field(6)
    ctx.deposit_vector(v)
    ctx.deposit_symtensor(t)
    assert normalized_error(B, v.export(0, np.float64).reshape(-1)) < 1e-5
    assert normalized_error(T, t.export(0, np.float64).reshape(-1)) < 1e-5
    ctx.deposit_vector_cic(v)
    ctx.deposit_vecvec_cic(t)
    assert normalized_error(V, v.export(0, np.float64).reshape(-1)) < 1e-5
    assert normalized_error(VV, t.export(0, np.float64).reshape(-1)) < 1e-5
