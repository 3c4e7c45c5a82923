"""Particle snapshots in the layout of the reference's HDF5 particle files.

Particles::saveHDF5 / loadHDF5 (particles/LATfield2_Particles.hpp:2808-3045,
written by save_hdf5_particles, particles/LATfield2_particlesIO.h:290-560)
store one file per group of ranks with
  - dataset "data": the part_simple records {ID, positionX..Z, velocityX..Z}
    (the packed file type of part_simple_dataType,
    particles/LATfield2_particle_simple.hpp:99-106: a long and six Reals),
    rank by rank, each rank's particles in site order;
  - dataset "numParts" (long [ranks]), "localBoxOffset" and "localBoxSize"
    (Real [ranks][3]): the particle count and local box of every rank;
  - dataset "part_info": one part_simple_info {mass, relativistic,
    type_name_size, type_name[64]};
  - attributes fileNumber, numProcPerFile, world_size, grid_size[2],
    boxSize[3], fileBoxSize, fileBoxOffset, latSize[3].

HDF5 is not available to this library, so a snapshot is a numpy archive
(.npz) whose members are those datasets under the same names and the
attributes under "@name"; each member is the array HDF5 would hold (double
Reals, little-endian), so a writer with HDF5 at hand copies them one to one.

Order: the reference writes a rank's particles cell by cell in site order
and, inside a cell, in its list order.  The library does not keep list
order, so particles inside a cell are written by increasing ID.

Fields: Field::saveHDF5(filename, dataset_name = "data")
(LATfield2_Field_decl.hpp:309-310, :1532-1544, written by save_hdf5,
LATfield2_save_hdf5.h:15-140) stores one dataset of the global lattice,
dims [z][y][x] and, with several components, an array type of comps Reals
per site; save_field writes that array (shape (n2, n1, n0) or
(n2, n1, n0, comps)) under the dataset name.  A build of the reference
without HDF5 writes filename + "BIN" with Field::write instead
(LATfield2_Field_decl.hpp:1179-1239): the same array as raw Reals, no
header; write_field_binary / read_field_binary produce and read that file.
"""
import numpy as np

PART_SIMPLE = np.dtype([("ID", "<i8"), ("positionX", "<f8"), ("positionY", "<f8"),
                        ("positionZ", "<f8"), ("velocityX", "<f8"), ("velocityY", "<f8"),
                        ("velocityZ", "<f8")])
PART_SIMPLE_INFO = np.dtype([("mass", "<f8"), ("relativistic", "<i4"),
                             ("type_name_size", "<i4"), ("type_name", "S64")])
ATTRS = ("fileNumber", "numProcPerFile", "world_size", "grid_size", "boxSize", "fileBoxSize",
         "fileBoxOffset", "latSize")


def records(cell, pos, vel, ids):
    """part_simple records of one rank, sorted by (cell, ID)."""
    cell = np.asarray(cell, np.int64)
    ids = np.asarray(ids, np.int64)
    order = np.lexsort((ids, cell))
    out = np.empty(cell.shape[0], PART_SIMPLE)
    out["ID"] = ids[order]
    pos = np.asarray(pos, np.float64)[order]
    vel = np.asarray(vel, np.float64)[order]
    for d, a in enumerate("XYZ"):
        out["position" + a] = pos[:, d]
        out["velocity" + a] = vel[:, d]
    return out


def part_info(mass, relativistic=0, type_name="part_simple"):
    info = np.zeros(1, PART_SIMPLE_INFO)
    name = type_name.encode()
    if len(name) > 63:
        raise ValueError("type_name longer than 63 bytes")
    info["mass"] = mass
    info["relativistic"] = relativistic
    info["type_name_size"] = len(name)
    info["type_name"] = name
    return info


def description(n, box, ranks_z, counts):
    """The file description of save_hdf5_particles for a lattice split in z
    over ranks_z ranks (one file, the reference's grid [ranks_z, 1]: dim 2 is
    split over grid dim 0, LATfield2_Lattice.hpp:88-94).  Returns
    (attributes, numParts, localBoxOffset, localBoxSize)."""
    n = tuple(int(v) for v in n)
    box = tuple(float(b) for b in box)
    res = box[0] / n[0]
    nz = n[2] // ranks_z
    offs = np.zeros((ranks_z, 3))
    size = np.empty((ranks_z, 3))
    for r in range(ranks_z):
        offs[r, 2] = res * (r * nz)  # localBoxOffset[2] = res coordSkip()[0]
        size[r] = (res * n[0], res * n[1], res * nz)
    attrs = {"fileNumber": np.int32(1), "numProcPerFile": np.int32(ranks_z),
             "world_size": np.int32(ranks_z), "grid_size": np.array([ranks_z, 1], np.int32),
             "boxSize": np.array(box), "fileBoxSize": np.float64(size[0, 1]),
             "fileBoxOffset": np.float64(0.0), "latSize": np.array(n, np.int32)}
    return attrs, np.asarray(counts, np.int64), offs, size


def write(path, data, info, attrs, num_parts, local_offset, local_size):
    members = {"data": data, "part_info": info, "numParts": num_parts,
               "localBoxOffset": local_offset, "localBoxSize": local_size}
    members.update({"@" + k: np.asarray(attrs[k]) for k in ATTRS})
    with open(path, "wb") as f:
        np.savez(f, **members)


def read(path):
    """{dataset or "@attribute": array} of a snapshot."""
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def check_box(snap, box):
    """Raises unless the snapshot's boxSize is `box`."""
    if not np.array_equal(np.asarray(snap["@boxSize"], np.float64), np.asarray(box, np.float64)):
        raise ValueError(f"wrong boxSize: the snapshot has {snap['@boxSize'].tolist()}, "
                         f"the lattice {list(box)} (as Particles::loadHDF5 refuses)")


def columns(data):
    """(ID, positions (n, 3), velocities (n, 3)) of part_simple records."""
    pos = np.stack([data["position" + a] for a in "XYZ"], axis=1)
    vel = np.stack([data["velocity" + a] for a in "XYZ"], axis=1)
    return np.ascontiguousarray(data["ID"]), pos, vel


def positions_to_cells(pos, n, res):
    """Box-unit positions -> (cell, FP32 offset) by the rule of
    lf2_particles_set_pos: u = pos (1/res), cell = floor(u) mod n, offset
    = u - floor(u) rounded to FP32 (an offset that rounds to 1 carries into
    the next cell), as getPartCoord (LATfield2_Particles.hpp:463-467)."""
    u = np.asarray(pos, np.float64) * (1.0 / res)
    fl = np.floor(u)
    off = (u - fl).astype(np.float32)
    carry = off >= np.float32(1.0)
    off[carry] = 0.0
    fl[carry] += 1.0
    ci = np.mod(fl.astype(np.int64), np.asarray(n, np.int64))
    cell = ci[:, 0] + n[0] * (ci[:, 1] + n[1] * ci[:, 2])
    return cell.astype(np.int32), np.ascontiguousarray(off)


def cells_to_positions(cell, off, n, res):
    """(cell, offset) -> box-unit positions, ((double)x + off) res as
    lf2_particles_get_pos computes them."""
    c = np.asarray(cell, np.int64)
    xyz = np.stack([c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1])], axis=1)
    return (xyz.astype(np.float64) + np.asarray(off, np.float64)) * res


def save_context(path, ctx, global_mass, relativistic=0, type_name="part_simple"):
    """Particles of one Context (which must carry IDs) as a one-rank snapshot.
    part_simple has no per-particle mass: a store with per-particle masses
    keeps them only in lf2_checkpoint_save's format."""
    p = ctx.get_particles(ids=True)
    pos = cells_to_positions(p["cell"], p["off"], ctx.n, ctx.res)
    data = records(p["cell"], pos, p["vel"], p["id"])
    attrs, num, offs, size = description(ctx.n, ctx.box, 1, [data.shape[0]])
    write(path, data, part_info(global_mass, relativistic, type_name), attrs, num, offs, size)


def load_context(path, ctx):
    """Particles of a snapshot (any number of ranks) into ctx, with their IDs
    and the part_info mass as global mass (Particles::loadHDF5 adds every
    record with addParticle_global).  Returns the part_info record."""
    snap = read(path)
    check_box(snap, ctx.box)
    ids, pos, vel = columns(snap["data"])
    info = snap["part_info"][0]
    ctx.set_positions(pos, vel, global_mass=float(info["mass"]), ids=ids)
    return info


def save_field(path, field, dataset_name="data", dtype=np.float64):
    """A field (FieldHandle) as the dataset of Field::saveHDF5, halo excluded."""
    a = field.export(halo=0, dtype=dtype)
    if a.shape[3] == 1:
        a = a[..., 0]
    with open(path, "wb") as f:
        np.savez(f, **{dataset_name: np.ascontiguousarray(a)})


def load_field(path, field, dataset_name="data"):
    """Field::loadHDF5: the dataset into `field` (same lattice and components)."""
    with np.load(path, allow_pickle=False) as z:
        a = z[dataset_name]
    n = field.ctx.n
    want = (n[2], n[1], n[0]) + (() if field.comps == 1 else (field.comps,))
    if tuple(a.shape) != want:
        raise ValueError(f"dataset {dataset_name!r} has shape {a.shape}, the field {want}")
    field.import_(np.ascontiguousarray(a.reshape(n[2], n[1], n[0], field.comps)), halo=0)


def write_field_binary(path, field, real_bytes=8):
    """Field::write's file: the lattice without halo, [z][y][x][comps], raw
    Reals of real_bytes (8 double, 4 SINGLE), no header."""
    a = field.export(halo=0, dtype=np.float64 if real_bytes == 8 else np.float32)
    with open(path, "wb") as f:
        f.write(np.ascontiguousarray(a).tobytes())


def read_field_binary(path, field, real_bytes=8):
    """Field::read: a file of write_field_binary's layout into `field`."""
    n = field.ctx.n
    a = np.fromfile(path, dtype=np.float64 if real_bytes == 8 else np.float32)
    if a.size != n[0] * n[1] * n[2] * field.comps:
        raise ValueError(f"{path}: {a.size} values, the field has "
                         f"{n[0] * n[1] * n[2] * field.comps}")
    field.import_(a.reshape(n[2], n[1], n[0], field.comps), halo=0)
