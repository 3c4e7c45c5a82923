"""The CUDA path against the reference's own outputs (tests/golden/, written
by the reference compiled from its sources): deposits, kick and move on the
same particles.  Tolerances as in test_gpu_parity.py: fixed-point and FP32
(compensated) deposits 1e-6 of the field maximum; velocities 2e-6 of the
maximum; positions 1e-6 of a cell, cells identical except within 1e-4 cells
of a face."""
import glob
import os

import numpy as np
import pytest

from tests.helpers import normalized_error

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(glob.glob(os.path.join(HERE, "*_double.npz")))


def _ctx(g, mode):
    import latfield2_b200 as L
    n = int(g["n"])
    ctx = L.Context((n, n, n), box=1.0, mode=mode)
    ctx.set_positions(g["pos"], g["vel"], global_mass=float(g["gmass"]), ids=g["ids"].copy())
    return ctx


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p) for p in CASES])
@pytest.mark.parametrize("mode", [0, 1])
def test_deposits_match_reference(cuda, path, mode):
    g = dict(np.load(path))
    ctx = _ctx(g, mode)
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    got = rho.export(0, np.float64)
    assert normalized_error(got, g["rho"]) < 1e-6
    if "vec" in g:
        v, t = ctx.field(3), ctx.field(6)
        ctx.deposit_vector(v)
        ctx.deposit_symtensor(t)
        for c in range(3):
            assert normalized_error(v.export(0, np.float64)[..., c], g["vec"][..., c]) < 1e-6
        for c in range(6):
            assert normalized_error(t.export(0, np.float64)[..., c], g["ten"][..., c]) < 1e-6


@pytest.mark.parametrize("path", [p for p in CASES if "vcic" in np.load(p)],
                         ids=lambda p: os.path.basename(p))
@pytest.mark.parametrize("mode", [0, 1])
def test_full_cic_deposits_match_reference(cuda, path, mode):
    """vectorProjectionCIC and VecVecProjectionCIC of the reference on a 2x2
    process grid against the single-GPU deposits (FP32 and fixed point,
    1e-6)."""
    g = dict(np.load(path))
    ctx = _ctx(g, mode)
    v, t = ctx.field(3), ctx.field(6)
    ctx.deposit_vector_cic(v)
    ctx.deposit_vecvec_cic(t)
    for c in range(3):
        assert normalized_error(v.export(0, np.float64)[..., c], g["vcic"][..., c]) < 1e-6
    for c in range(6):
        assert normalized_error(t.export(0, np.float64)[..., c], g["vv"][..., c]) < 1e-6


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p) for p in CASES])
def test_kick_and_move_match_reference(cuda, path):
    import torch
    g = dict(np.load(path))
    if "kick_vel" not in g:
        pytest.skip("fixture holds deposits only")
    n = int(g["n"])
    ctx = _ctx(g, 1)
    F = torch.from_numpy(np.ascontiguousarray(g["F"].transpose(3, 0, 1, 2)).astype(np.float32)).cuda()
    Fh = ctx.field(3, F)
    maxv = ctx.gather_kick(Fh, float(g["dtau_kick"]), want_max_v=True)
    pos, vel, ids = ctx.get_positions(ids=True)
    k = np.argsort(ids)
    np.testing.assert_array_equal(ids[k], g["kick_id"])
    assert normalized_error(vel[k], g["kick_vel"]) < 2e-6
    assert maxv == pytest.approx(float(g["maxv"]), rel=2e-6)
    if "move_pos" in g:
        ctx.drift_rebin(float(g["dtau_move"]))
        pos, vel, ids = ctx.get_positions(ids=True)
        k = np.argsort(ids)
        d = np.abs(pos[k] - g["move_pos"])
        d = np.minimum(d, 1.0 - d)
        assert d.max() < 1e-6 / n
        ref_u = g["move_pos"] * n
        ref_xyz = np.floor(ref_u).astype(np.int64) % n
        ref_cell = ref_xyz[:, 0] + n * (ref_xyz[:, 1] + n * ref_xyz[:, 2])
        st = ctx.get_particles(ids=True)
        got_cell = st["cell"][np.argsort(st["id"])]
        near = np.any(np.abs(ref_u - np.round(ref_u)) < 1e-4, axis=1)
        assert np.all((ref_cell == got_cell) | near)
        counts = ctx.cell_counts()
        np.testing.assert_array_equal(counts, np.bincount(got_cell, minlength=n ** 3))
        if not near.any():
            np.testing.assert_array_equal(counts, np.bincount(ref_cell, minlength=n ** 3))
