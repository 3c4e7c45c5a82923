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


@pytest.mark.parametrize("single", [False, True])
def test_poisson_demo_builds_against_the_header(tmp_path, single):
    import build_demo
    out = str(tmp_path / ("poisson_single" if single else "poisson_double"))
    assert os.path.exists(build_demo.build(out, single, "poisson_demo.cpp"))


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


@pytest.mark.gpu
@pytest.mark.parametrize("khalo", [0, 1])
def test_poisson_demo_matches_the_oracle(cuda, tmp_path, khalo):
    """The reference-style Poisson program (rKSite loop, PlanFFT forward and
    backward, updateHalo) on the GPU path: its rho_k is the oracle's forward
    transform in the reference's storage order, its phi the oracle's Poisson
    solution, and its own Laplacian check holds."""
    import build_demo
    from oracle import fft_oracle as FO
    exe = build_demo.build(str(tmp_path / "poisson"), False, "poisson_demo.cpp")
    out = str(tmp_path / "poisson.bin")
    n = 32
    r = subprocess.run([exe, str(n), out, str(khalo)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert float(r.stdout.split()[3]) < 1e-4, r.stdout
    (hdr, rho, rhok, phi) = _read(out)
    assert int(hdr[0]) == n
    rho = rho.reshape(n, n, n)
    k = (rhok[0::2] + 1j * rhok[1::2]).reshape(n, n, n // 2 + 1)
    want = FO.rfft_ref(rho)
    assert normalized_error(k.real, want.real) < 1e-5
    assert normalized_error(k.imag, want.imag) < 1e-5
    assert normalized_error(phi.reshape(n, n, n), FO.poisson_example(rho, 1.0 / n)) < 1e-5


def test_restart_demo_builds_against_the_header(tmp_path):
    import build_demo
    assert os.path.exists(build_demo.build(str(tmp_path / "restart_demo"),
                                           source="restart_demo.cpp"))


@pytest.mark.gpu
def test_restart_through_particles_save_and_load(cuda, tmp_path):
    """Particles::saveHDF5 / loadHDF5 of the C++ layer: a set restored from
    the file continues bit for bit (tests/compat/restart_demo.cpp)."""
    import build_demo
    exe = build_demo.build(str(tmp_path / "restart_demo"), source="restart_demo.cpp")
    r = subprocess.run([exe, "24", "20000", str(tmp_path)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
    assert os.path.exists(tmp_path / "run.lf2c")


def test_outputs_demo_builds_against_the_header(tmp_path):
    import build_demo
    for single in (False, True):
        out = str(tmp_path / ("outputs_single" if single else "outputs_double"))
        assert os.path.exists(build_demo.build(out, single, "outputs_demo.cpp"))


@pytest.mark.gpu
def test_update_vel_outputs_mapping_overload_and_oset(cuda, tmp_path):
    """tests/compat/outputs_demo.cpp: updateVel's SUM / MIN / MAX outputs of
    the kick's |v|^2 (FP64 on the GPU) against FP64 sums of the Python
    binding's velocities; the mappingClass overload kicks like the plain one;
    a projection with the part_info mass at its offset, doubled, gives twice
    the density bit for bit; offsets the GPU store does not hold are
    refused."""
    import torch
    import build_demo
    import latfield2_b200 as L
    exe = build_demo.build(str(tmp_path / "outputs"), False, "outputs_demo.cpp")
    out = str(tmp_path / "outputs.bin")
    n, npart = 32, 20000
    r = subprocess.run([exe, str(n), str(npart), out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    hdr, id0, pos0, vel0, Fv, rho, rho2, B = _read(out)
    dtau = hdr[2]
    assert int(hdr[10]) == 2  # both bad offsets refused
    ctx = L.Context((n, n, n), box=1.0, mode=L.DEPOSIT_FIXED64)
    ctx.set_positions(pos0.reshape(-1, 3), vel0.reshape(-1, 3), global_mass=1.0 / npart,
                      ids=id0.astype(np.int64))
    Fi = torch.from_numpy(np.ascontiguousarray(
        Fv.reshape(n, n, n, 3).transpose(3, 0, 1, 2)).astype(np.float32)).cuda()
    F = ctx.field(3, Fi)
    sums = []
    for k in range(2):
        mv = ctx.gather_kick(F, dtau, want_max_v=True)
        assert mv == hdr[3 + k]
        _, vel, _ = ctx.get_positions(ids=True)
        v2 = np.sum(vel.astype(np.float64) ** 2, axis=1)
        sums.append((v2.sum(), v2.min(), v2.max()))
    assert hdr[5] == pytest.approx(sums[0][0], rel=1e-12)
    assert hdr[6] == sums[0][1] and hdr[7] == sums[0][2]
    assert hdr[8] == sums[1][2] and hdr[9] == pytest.approx(sums[1][0], rel=1e-12)
    d = ctx.field(1)
    ctx.deposit_scalar(d)
    np.testing.assert_array_equal(d.export(0, np.float64).reshape(-1), rho)
    np.testing.assert_array_equal(rho2, 2 * rho)
    v = ctx.field(3)
    ctx.deposit_vector(v)
    np.testing.assert_array_equal(v.export(0, np.float64).reshape(-1), B)


def test_device_physics_demo_builds_with_nvcc(tmp_path):
    import build_demo
    for single in (False, True):
        out = str(tmp_path / ("device_single" if single else "device_double"))
        assert os.path.exists(build_demo.build(out, single, "device_physics_demo.cu"))


@pytest.mark.gpu
def test_user_physics_runs_on_the_gpu(cuda, tmp_path):
    """tests/compat/device_physics_demo.cu: a user's kick and drift, written as
    functors with __device__ operator() and the reference's callback
    arguments, run through updateVel / moveParticles on the GPU.  They compute
    the CIC kick and pos += dtau vel in double, so they agree with the
    library's FP32 kick and drift to FP32 rounding: velocities within 1e-6 of
    their scale, positions within 1e-6 of a cell; the SUM and MAX outputs of
    |v|^2 match FP64 sums of the velocities."""
    import torch
    import build_demo
    import latfield2_b200 as L
    exe = build_demo.build(str(tmp_path / "device_physics"), False, "device_physics_demo.cu")
    out = str(tmp_path / "device_physics.bin")
    n, npart = 32, 20000
    r = subprocess.run([exe, str(n), str(npart), out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    hdr, id0, pos0, vel0, Fv, id1, pos1, vel1 = _read(out)
    dtau = hdr[2]
    assert int(hdr[1]) == npart
    ctx = L.Context((n, n, n), box=1.0, mode=L.DEPOSIT_FIXED64)
    ctx.set_positions(pos0.reshape(-1, 3), vel0.reshape(-1, 3), global_mass=1.0 / npart,
                      ids=id0.astype(np.int64))
    Fi = torch.from_numpy(np.ascontiguousarray(
        Fv.reshape(n, n, n, 3).transpose(3, 0, 1, 2)).astype(np.float32)).cuda()
    F = ctx.field(3, Fi)
    ctx.gather_kick(F, dtau)
    ctx.drift_rebin(dtau)
    pos, vel, ids = ctx.get_positions(ids=True)
    k, k1 = np.argsort(ids), np.argsort(id1)
    np.testing.assert_array_equal(ids[k], id1[k1].astype(np.int64))
    v_user, p_user = vel1.reshape(-1, 3)[k1], pos1.reshape(-1, 3)[k1]
    assert np.max(np.abs(vel[k] - v_user)) <= 1e-6 * np.max(np.abs(vel))
    d = np.abs(pos[k] - p_user)
    d = np.minimum(d, 1.0 - d)  # periodic
    assert np.max(d) <= 1e-6 / n
    v2 = np.sum(v_user.astype(np.float64) ** 2, axis=1)
    assert hdr[4] == pytest.approx(v2.sum(), rel=1e-6)
    assert hdr[5] == pytest.approx(v2.max(), rel=1e-6)
    assert hdr[3] == pytest.approx(np.sqrt(v2.max()), rel=1e-6)
