"""The no-allocation scalar deposit (lf2_deposit_scalar_noalloc).

Callers that may not allocate device memory while running (an application
that hands out device memory from its own pool, a plugin allowed to allocate
only at load time, a loop that cannot afford cudaMalloc's synchronisation)
use this entry point: they pass their own device inputs and output, and the
deposit's scratch is a fixed array inside the library.  These tests call it
through the C ABI and check it against lf2_deposit_scalar, twice in a row on
the same inputs (the shared scratch keeps the previous call's contents).
The file is named so that pytest collects it after every other test.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import normalized_error, small_case

pytestmark = pytest.mark.gpu

BRICK = 16


def _bricked(n, cell, off):
    """Particles grouped by brick, and the brick start offsets."""
    nb = [-(-v // BRICK) for v in n]
    c = cell.astype(np.int64)
    x, y, z = c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1])
    b = x // BRICK + nb[0] * (y // BRICK + nb[1] * (z // BRICK))
    order = np.argsort(b, kind="stable")
    counts = np.bincount(b, minlength=nb[0] * nb[1] * nb[2])
    start = np.zeros(counts.size + 1, np.int64)
    start[1:] = np.cumsum(counts)
    return cell[order], off[order], start


def _noalloc(n, mode, mass, cell_t, off_t, start_t, rho_t, want_flags=True):
    from latfield2_b200 import _lib
    lib = _lib.load()
    na = (ctypes.c_int * 3)(*n)
    box = (ctypes.c_double * 3)(*[v / n[0] for v in n])
    flags = ctypes.c_uint32(0)
    st = lib.lf2_deposit_scalar_noalloc(
        na, box, mode, mass, int(cell_t.numel()), ctypes.c_void_p(cell_t.data_ptr()),
        ctypes.c_void_p(off_t.data_ptr()), ctypes.c_void_p(start_t.data_ptr()),
        ctypes.c_void_p(rho_t.data_ptr()), None, ctypes.byref(flags) if want_flags else None)
    return st, flags.value


def _reference(n, mode, mass, cell, off):
    import latfield2_b200 as L
    ctx = L.Context(n, box=tuple(v / n[0] for v in n), mode=mode)
    ctx.set_particles(cell, off, np.zeros_like(off), global_mass=mass)
    rho = ctx.field(1)
    ctx.deposit_scalar(rho)
    return rho.export_internal()[0]


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n", [(48, 40, 33), (64, 64, 64), (8, 8, 8)])
def test_noalloc_matches_deposit_scalar_twice(cuda, mode, n):
    import torch
    from latfield2_b200 import _lib
    cell, off, _ = small_case(n, 30000, seed=77, clustered=True)
    mass = 1.0 / 30000
    ref = _reference(n, mode, mass, cell, off)
    bc, bo, start = _bricked(n, cell, off)
    cell_t = torch.from_numpy(bc).cuda()
    off_t = torch.from_numpy(np.ascontiguousarray(bo)).cuda()
    start_t = torch.from_numpy(start).cuda()
    for call in range(2):
        rho_t = torch.full((n[2], n[1], n[0]), float("nan"), dtype=torch.float32, device="cuda")
        st, flags = _noalloc(n, mode, mass, cell_t, off_t, start_t, rho_t)
        assert st == _lib.LF2_OK and flags == 0, (call, st, flags)
        got = rho_t.cpu().numpy()
        if mode == 1:
            np.testing.assert_array_equal(got, ref)
        else:
            assert normalized_error(got, ref) < 1e-5, call


def test_noalloc_rejects_lattices_beyond_its_scratch(cuda):
    import torch
    from latfield2_b200 import _lib
    n = (256, 256, 256)  # 4096 bricks > LF2_NOALLOC_MAX_BRICKS
    empty_i = torch.zeros(1, dtype=torch.int32, device="cuda")
    empty_f = torch.zeros(3, dtype=torch.float32, device="cuda")
    start = torch.zeros(4097, dtype=torch.int64, device="cuda")
    rho = torch.zeros(1, dtype=torch.float32, device="cuda")
    st, _ = _noalloc(n, 1, 1.0, empty_i[:0], empty_f[:0], start, rho)
    assert st == _lib.LF2_ERR_UNSUPPORTED
    assert _lib.NOALLOC_MAX_BRICKS == 1363


def test_noalloc_reports_particles_outside_their_brick(cuda):
    import torch
    from latfield2_b200 import _lib
    n = (32, 32, 32)
    cell, off, _ = small_case(n, 2000, seed=5)
    bc, bo, start = _bricked(n, cell, off)
    start[1] = 0  # brick 0 now claims no particles; brick 1 gets brick 0's
    cell_t = torch.from_numpy(bc).cuda()
    off_t = torch.from_numpy(np.ascontiguousarray(bo)).cuda()
    start_t = torch.from_numpy(start).cuda()
    rho_t = torch.zeros(32 ** 3, dtype=torch.float32, device="cuda")
    st, flags = _noalloc(n, 1, 1.0 / 2000, cell_t, off_t, start_t, rho_t)
    assert st == _lib.LF2_ERR_STATE and flags & _lib.FLAG_BAD_CELL
    # the next good call clears the error word
    bc, bo, start = _bricked(n, cell, off)
    st, flags = _noalloc(n, 1, 1.0 / 2000, cell_t, off_t, torch.from_numpy(start).cuda(), rho_t)
    assert st == _lib.LF2_OK and flags == 0


def test_noalloc_clamps_and_reports_a_brick_range_past_the_particles(cuda):
    """A last brick offset beyond np is reported and never read past: the
    particle arrays are backed by longer buffers, so the test itself stays in
    bounds whatever the kernel does."""
    import torch
    from latfield2_b200 import _lib
    n = (32, 32, 32)
    cell, off, _ = small_case(n, 2000, seed=9)
    bc, bo, start = _bricked(n, cell, off)
    npart = bc.size
    pad = 4096
    cell_t = torch.zeros(npart + pad, dtype=torch.int32, device="cuda")
    off_t = torch.zeros((npart + pad, 3), dtype=torch.float32, device="cuda")
    cell_t[:npart] = torch.from_numpy(bc).cuda()
    off_t[:npart] = torch.from_numpy(np.ascontiguousarray(bo)).cuda()
    bad = start.copy()
    bad[-1] = npart + pad  # the last brick claims slots past np
    rho_t = torch.zeros(32 ** 3, dtype=torch.float32, device="cuda")
    from latfield2_b200 import _lib as L
    lib = L.load()
    na = (ctypes.c_int * 3)(*n)
    box = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    flags = ctypes.c_uint32(0)
    bad_t = torch.from_numpy(bad).cuda()
    st = lib.lf2_deposit_scalar_noalloc(
        na, box, 1, 1.0 / npart, npart, ctypes.c_void_p(cell_t.data_ptr()),
        ctypes.c_void_p(off_t.data_ptr()), ctypes.c_void_p(bad_t.data_ptr()),
        ctypes.c_void_p(rho_t.data_ptr()), None, ctypes.byref(flags))
    assert st == _lib.LF2_ERR_STATE and flags.value & _lib.FLAG_BAD_CELL
    # offsets that decrease are reported the same way
    bad = start.copy()
    bad[3] = bad[2] - 1 if bad[2] > 0 else -1
    bad_t = torch.from_numpy(bad).cuda()
    st = lib.lf2_deposit_scalar_noalloc(
        na, box, 1, 1.0 / npart, npart, ctypes.c_void_p(cell_t.data_ptr()),
        ctypes.c_void_p(off_t.data_ptr()), ctypes.c_void_p(bad_t.data_ptr()),
        ctypes.c_void_p(rho_t.data_ptr()), None, ctypes.byref(flags))
    assert st == _lib.LF2_ERR_STATE and flags.value & _lib.FLAG_BAD_CELL


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_without_flags_runs_asynchronously(cuda, mode):
    """flags == NULL: the call only queues the work; after a synchronize the
    result equals the context deposit's."""
    import torch
    from latfield2_b200 import _lib
    n = (48, 48, 48)
    cell, off, _ = small_case(n, 20000, seed=31, clustered=True)
    mass = 1.0 / 20000
    ref = _reference(n, mode, mass, cell, off)
    bc, bo, start = _bricked(n, cell, off)
    cell_t = torch.from_numpy(bc).cuda()
    off_t = torch.from_numpy(np.ascontiguousarray(bo)).cuda()
    start_t = torch.from_numpy(start).cuda()
    for call in range(2):
        rho_t = torch.full((n[2], n[1], n[0]), float("nan"), dtype=torch.float32, device="cuda")
        st, _ = _noalloc(n, mode, mass, cell_t, off_t, start_t, rho_t, want_flags=False)
        assert st == _lib.LF2_OK
        torch.cuda.synchronize()
        got = rho_t.cpu().numpy()
        if mode == 1:
            np.testing.assert_array_equal(got, ref)
        else:
            assert normalized_error(got, ref) < 1e-5, call
