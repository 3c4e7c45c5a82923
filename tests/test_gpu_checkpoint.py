"""lf2_checkpoint_save / lf2_checkpoint_load: a run saved after some steps and
restored into a fresh context continues bit for bit (particles by id, and
the fixed-point density), with global and with per-particle masses; a
checkpoint of another lattice is refused; the file header is the documented
80-byte layout."""
import struct

import numpy as np
import pytest
import torch

from tests.helpers import small_case

pytestmark = pytest.mark.gpu


def _ctx(n):
    import latfield2_b200 as L
    return L.Context(n, box=tuple(v / n[0] for v in n), mode=L.DEPOSIT_FIXED64)


@pytest.mark.parametrize("per_particle_mass", [False, True])
def test_restart_is_bit_exact(tmp_path, per_particle_mass):
    n = (48, 40, 32)
    cell, off, vel = small_case(n, 80000, seed=31, vel_sigma=0.05, clustered=True)
    ids = np.arange(cell.shape[0], dtype=np.int64)
    mass = None
    if per_particle_mass:
        mass = (1.0 + 0.3 * np.random.default_rng(32).uniform(-1, 1, cell.shape[0])).astype(
            np.float32) / cell.shape[0]
    F = torch.from_numpy(np.random.default_rng(33).standard_normal((3, n[2], n[1], n[0]))
                         .astype(np.float32) * 0.05).cuda()
    a = _ctx(n)
    a.set_particles(cell, off, vel, mass=mass, global_mass=0.0 if per_particle_mass else 1e-5,
                    ids=ids)
    Fa, rho_a = a.field(3, F), a.field(1)
    for _ in range(3):
        a.step(Fa, 0.05, 0.1, rho_a)
    path = tmp_path / "run.lf2c"
    a.checkpoint_save(path)
    head = open(path, "rb").read(80)
    magic, version, n0, n1, n2, mode, hm, hi = struct.unpack("<8i", head[:32])
    assert (magic, version, (n0, n1, n2), hm, hi) == (0x4332464C, 1, n, int(per_particle_mass), 1)
    assert struct.unpack("<q", head[72:80])[0] == cell.shape[0]

    b = _ctx(n)
    b.checkpoint_load(path)
    Fb, rho_b = b.field(3, F.clone()), b.field(1)
    for _ in range(4):
        a.step(Fa, 0.05, 0.1, rho_a)
        b.step(Fb, 0.05, 0.1, rho_b)
    pa = a.get_particles(mass=per_particle_mass, ids=True)
    pb = b.get_particles(mass=per_particle_mass, ids=True)
    oa, ob = np.argsort(pa["id"]), np.argsort(pb["id"])
    for k in pa:
        np.testing.assert_array_equal(pa[k][oa], pb[k][ob], err_msg=k)
    np.testing.assert_array_equal(rho_a.export_internal(), rho_b.export_internal())


def test_other_lattice_is_refused(tmp_path):
    import latfield2_b200 as L
    a = _ctx((32, 32, 32))
    cell, off, vel = small_case((32, 32, 32), 1000, seed=1)
    a.set_particles(cell, off, vel, global_mass=1e-3)
    p = tmp_path / "a.lf2c"
    a.checkpoint_save(p)
    b = _ctx((32, 32, 16))
    with pytest.raises(L.LF2Error, match="another lattice"):
        b.checkpoint_load(p)
    (tmp_path / "junk").write_bytes(b"not a checkpoint at all" * 10)
    with pytest.raises(L.LF2Error, match="not a checkpoint"):
        a.checkpoint_load(tmp_path / "junk")


def test_snapshot_in_the_reference_layout_round_trips(tmp_path):
    """latfield2_b200.snapshot: a Context's particles saved as part_simple
    records and loaded into a fresh Context (bit-exact by ID: res is a power
    of two), and a one-rank SlabDomain on the GPU saved and loaded the same
    way, after steps that moved particles across cells."""
    from latfield2_b200 import _lib
    from latfield2_b200 import snapshot as S
    from latfield2_b200.distributed import SlabDomain
    n = (32, 32, 32)
    cell, off, vel = small_case(n, 40000, seed=35, vel_sigma=0.05)
    ids = np.arange(cell.shape[0], dtype=np.int64)[::-1].copy()
    gm = 1.0 / cell.shape[0]
    F = torch.from_numpy(np.random.default_rng(36).standard_normal((3, n[2], n[1], n[0]))
                         .astype(np.float32) * 0.05).cuda()
    a = _ctx(n)
    a.set_particles(cell, off, vel, global_mass=gm, ids=ids)
    Fa = a.field(3, F)
    for _ in range(2):
        a.step(Fa, 0.05, 0.1, None)
    want = a.get_particles(ids=True)
    path = tmp_path / "parts.npz"
    S.save_context(path, a, gm)
    snap = S.read(path)
    assert snap["data"].shape[0] == cell.shape[0] and snap["part_info"]["mass"][0] == gm
    assert np.all(np.diff(S.positions_to_cells(S.columns(snap["data"])[1], n, 1.0 / 32)[0]) >= 0)
    b = _ctx(n)
    S.load_context(path, b)
    got = b.get_particles(ids=True)
    o1, o2 = np.argsort(want["id"]), np.argsort(got["id"])
    for k in ("id", "cell", "off", "vel"):
        np.testing.assert_array_equal(got[k][o2], want[k][o1], err_msg=k)
    d = SlabDomain(n, box=1.0, mode=_lib.DEPOSIT_FIXED64)
    d.set_particles(want["cell"], want["off"], want["vel"], gm, ids=want["id"])
    d.save_particles(tmp_path / "slab.npz", gm)
    c = _ctx(n)
    S.load_context(tmp_path / "slab.npz", c)
    got = c.get_particles(ids=True)
    o3 = np.argsort(got["id"])
    for k in ("id", "cell", "off", "vel"):
        np.testing.assert_array_equal(got[k][o3], want[k][o1], err_msg=k)


def test_field_snapshot_in_the_reference_layout(tmp_path):
    """snapshot.save_field / load_field: the dataset of Field::saveHDF5
    (dims [z][y][x], comps Reals per site) of a deposited density and of a
    3-component field, back into fresh fields bit for bit (FP32 values
    stored as double)."""
    from latfield2_b200 import snapshot as S
    n = (24, 20, 16)
    cell, off, vel = small_case(n, 20000, seed=37)
    a = _ctx(n)
    a.set_particles(cell, off, vel, global_mass=1e-4)
    rho = a.field(1)
    a.deposit_scalar(rho)
    v = a.field(3)
    a.deposit_vector(v)
    S.save_field(tmp_path / "rho.npz", rho)
    S.save_field(tmp_path / "v.npz", v, dataset_name="vel")
    with np.load(tmp_path / "rho.npz") as z:
        assert z["data"].shape == (16, 20, 24) and z["data"].dtype == np.float64
    with np.load(tmp_path / "v.npz") as z:
        assert z["vel"].shape == (16, 20, 24, 3)
    b = _ctx(n)
    r2, v2 = b.field(1), b.field(3)
    S.load_field(tmp_path / "rho.npz", r2)
    S.load_field(tmp_path / "v.npz", v2, dataset_name="vel")
    np.testing.assert_array_equal(r2.export_internal(), rho.export_internal())
    np.testing.assert_array_equal(v2.export_internal(), v.export_internal())
    with pytest.raises(ValueError, match="shape"):
        S.load_field(tmp_path / "rho.npz", v2)
