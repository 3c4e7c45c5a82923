"""Particle snapshots in the layout of the reference's HDF5 particle files
(latfield2_b200/snapshot.py): the record and part_info layouts against
part_simple_dataType (particles/LATfield2_particle_simple.hpp:99-112), the
file description against save_hdf5_particles and Particles::saveHDF5
(particles/LATfield2_particlesIO.h:290-560, LATfield2_Particles.hpp:2808-2905),
the position <-> (cell, offset) rules, and a save on 2 gloo ranks of the slab
decomposition restored on 1 and 4 ranks (particles bit-exact by ID)."""
import os
import socket

import numpy as np
import pytest

from latfield2_b200 import _lib
from latfield2_b200 import snapshot as S
from tests.helpers import small_case

N = (16, 12, 16)


def test_record_layouts_are_the_reference_file_types():
    # part_fileType: a long, then six Reals (double) at 8-byte steps
    assert S.PART_SIMPLE.itemsize == 8 + 6 * 8
    assert [S.PART_SIMPLE.fields[k][1] for k in S.PART_SIMPLE.names] == [0, 8, 16, 24, 32, 40, 48]
    assert S.PART_SIMPLE.names == ("ID", "positionX", "positionY", "positionZ", "velocityX",
                                   "velocityY", "velocityZ")
    # part_info_fileType: double mass, int relativistic, int type_name_size, char[64]
    assert S.PART_SIMPLE_INFO.itemsize == 8 + 2 * 4 + 64
    assert [S.PART_SIMPLE_INFO.fields[k][1] for k in S.PART_SIMPLE_INFO.names] == [0, 8, 12, 16]
    info = S.part_info(0.25, 1, "part_simple")
    assert info["type_name_size"][0] == 11 and info["type_name"][0] == b"part_simple"


def test_file_description_of_a_z_split():
    box = (1.0, 0.75, 1.0)
    attrs, num, offs, size = S.description(N, box, 4, [5, 6, 7, 8])
    res = 1.0 / 16
    np.testing.assert_array_equal(num, [5, 6, 7, 8])
    np.testing.assert_array_equal(offs, [[0, 0, r * 4 * res] for r in range(4)])
    np.testing.assert_array_equal(size, [[1.0, 0.75, 4 * res]] * 4)
    assert attrs["fileNumber"] == 1 and attrs["numProcPerFile"] == 4
    assert attrs["world_size"] == 4 and list(attrs["grid_size"]) == [4, 1]
    assert attrs["fileBoxSize"] == 0.75 and attrs["fileBoxOffset"] == 0.0
    assert list(attrs["latSize"]) == list(N) and list(attrs["boxSize"]) == list(box)


@pytest.mark.parametrize("n,res", [((16, 12, 16), 1.0 / 16), ((20, 12, 24), 1.0 / 20)])
def test_positions_and_cells_round_trip(n, res):
    """Exact when res is a power of two (the products and quotients are
    exact); otherwise x res / res may land an ulp from x, and an offset of 0
    comes back as about 1e-15 (or carries), as in the library."""
    cell, off, _ = small_case(n, 5000, seed=3)
    off[:7] = 0.0
    off[7:14] = np.nextafter(np.float32(1.0), np.float32(0.0))
    pos = S.cells_to_positions(cell, off, n, res)
    c2, o2 = S.positions_to_cells(pos, n, res)
    np.testing.assert_array_equal(c2, cell)
    if res == 1.0 / 16:
        np.testing.assert_array_equal(o2, off)
        # positions outside the box wrap periodically
        c3, o3 = S.positions_to_cells(pos + np.array(n) * res, n, res)
        np.testing.assert_array_equal(c3, cell)
        np.testing.assert_array_equal(o3, off)
    else:
        assert np.abs(o2 - off).max() <= 2.0 ** -40


def test_records_are_in_cell_then_id_order(tmp_path):
    cell = np.array([5, 2, 5, 2, 9], np.int32)
    ids = np.array([40, 30, 10, 20, 0], np.int64)
    pos = np.arange(15, dtype=np.float64).reshape(5, 3)
    rec = S.records(cell, pos, -pos, ids)
    np.testing.assert_array_equal(rec["ID"], [20, 30, 10, 40, 0])
    np.testing.assert_array_equal(rec["positionY"], pos[[3, 1, 2, 0, 4], 1])
    attrs, num, offs, size = S.description(N, (1.0, 0.75, 1.0), 1, [5])
    S.write(tmp_path / "p.npz", rec, S.part_info(0.5), attrs, num, offs, size)
    snap = S.read(tmp_path / "p.npz")
    assert snap["data"].dtype == S.PART_SIMPLE and snap["part_info"]["mass"][0] == 0.5
    assert sorted(k[1:] for k in snap if k.startswith("@")) == sorted(S.ATTRS)
    with pytest.raises(ValueError, match="boxSize"):
        S.check_box(snap, (1.0, 1.0, 1.0))


def _case():
    cell, off, vel = small_case(N, 3000, seed=41)
    return cell, off, vel, np.arange(cell.shape[0], dtype=np.int64) * 3 + 7


def _domain():
    from latfield2_b200.distributed import SlabDomain
    from tests.slab_oracle_engine import OracleEngine
    return SlabDomain(N, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=OracleEngine)


def _save(path):
    cell, off, vel, ids = _case()
    d = _domain()
    d.set_particles(cell, off, vel, 1.0 / cell.shape[0], ids=ids)
    d.save_particles(path, 1.0 / cell.shape[0])
    return d.rank


def _load(path):
    d = _domain()
    info = d.load_particles(path)
    return d.rank, d.particles_global(), float(info["mass"])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out, fn, path):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out.put(globals()[fn](path))
    finally:
        dist.destroy_process_group()


def _ranks(world, fn, path):
    if world == 1:
        return [globals()[fn](path)]
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fn, str(path)))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("load_world", [1, 4])
def test_slab_save_on_two_ranks_restores_on_any_number(tmp_path, load_world):
    path = tmp_path / "parts.npz"
    _ranks(2, "_save", path)
    cell, off, vel, ids = _case()
    snap = S.read(path)
    np.testing.assert_array_equal(snap["numParts"].sum(), cell.shape[0])
    z = cell // (N[0] * N[1])
    np.testing.assert_array_equal(snap["numParts"], [(z < 8).sum(), (z >= 8).sum()])
    assert list(snap["@grid_size"]) == [2, 1]
    got = _ranks(load_world, "_load", path)
    parts = {k: np.concatenate([g[1][k] for g in got]) for k in ("cell", "off", "vel", "id")}
    order = np.argsort(parts["id"])
    want = np.argsort(ids)
    np.testing.assert_array_equal(parts["id"][order], ids[want])
    np.testing.assert_array_equal(parts["cell"][order], cell[want])
    np.testing.assert_array_equal(parts["off"][order], off[want])
    np.testing.assert_array_equal(parts["vel"][order], vel[want])
    assert all(g[2] == 1.0 / cell.shape[0] for g in got)


class _FakeContext:
    """The Context methods the snapshot functions call, on host arrays."""

    def __init__(self, n, box):
        self.n, self.box, self.res = n, box, box[0] / n[0]
        self.parts = None
        self.loaded = None

    def get_particles(self, ids=False):
        return dict(self.parts)

    def set_positions(self, pos, vel, global_mass=0.0, ids=None):
        self.loaded = (pos, vel, global_mass, ids)


def test_context_snapshot_functions_on_host_arrays(tmp_path):
    cell, off, vel, ids = _case()
    a = _FakeContext(N, (1.0, 0.75, 1.0))
    a.parts = {"cell": cell, "off": off, "vel": vel, "id": ids}
    S.save_context(tmp_path / "c.npz", a, 0.125, type_name="part_simple")
    snap = S.read(tmp_path / "c.npz")
    assert list(snap["numParts"]) == [cell.shape[0]] and list(snap["@grid_size"]) == [1, 1]
    b = _FakeContext(N, (1.0, 0.75, 1.0))
    info = S.load_context(tmp_path / "c.npz", b)
    pos, v, gm, i = b.loaded
    assert gm == 0.125 and info["type_name"] == b"part_simple"
    c2, o2 = S.positions_to_cells(pos, N, 1.0 / 16)
    order = np.argsort(i)
    want = np.argsort(ids)
    np.testing.assert_array_equal(i[order], ids[want])
    np.testing.assert_array_equal(c2[order], cell[want])
    np.testing.assert_array_equal(o2[order], off[want])
    np.testing.assert_array_equal(v[order], vel[want].astype(np.float64))
    with pytest.raises(ValueError, match="boxSize"):
        S.load_context(tmp_path / "c.npz", _FakeContext(N, (1.0, 1.0, 1.0)))


def _fields(path):
    """A 3-component field set from a global array on every rank, saved in
    both layouts; then loaded into fresh fields."""
    d = _domain()
    g = np.arange(3 * N[0] * N[1] * N[2], dtype=np.float64).reshape(3, N[2], N[1], N[0]) / 7.0
    f = d.field(3)
    d.set_own_planes(f, g.astype(np.float32))
    d.save_field(path + ".npz", f, dataset_name="vel")
    d.save_field_binary(path + ".bin", f)
    a, b = d.field(3), d.field(3)
    d.load_field(path + ".npz", a, dataset_name="vel")
    d.load_field_binary(path + ".bin", b)
    return d.rank, d.own_planes(a), d.own_planes(b), a[0].numpy()[:, 0].copy(), d.z0


@pytest.mark.parametrize("world", [1, 2])
def test_slab_fields_in_the_reference_file_layouts(tmp_path, world):
    path = str(tmp_path / "f")
    res = _ranks(world, "_fields", path)
    g = (np.arange(3 * N[0] * N[1] * N[2], dtype=np.float64).reshape(3, N[2], N[1], N[0])
         / 7.0).astype(np.float32)
    with np.load(path + ".npz") as z:
        np.testing.assert_array_equal(z["vel"], g.transpose(1, 2, 3, 0).astype(np.float64))
    np.testing.assert_array_equal(np.fromfile(path + ".bin").reshape(N[2], N[1], N[0], 3),
                                  g.transpose(1, 2, 3, 0))
    for _, a, b, ghost0, z0 in res:
        nz = a.shape[1]
        np.testing.assert_array_equal(a, g[:, z0:z0 + nz])
        np.testing.assert_array_equal(b, g[:, z0:z0 + nz])
        np.testing.assert_array_equal(ghost0, g[:, (z0 - 1) % N[2]])  # plane 0 = plane below
