"""z-slab decomposition of the particle-mesh step over the ranks of a
torch.distributed process group, one rank per GPU: the multi-GPU form of the
path (LATfield2's Lattice splits z and y over a 2-D process grid,
LATfield2_Lattice.hpp:88-94; here z alone is split).

Rank r of R owns the cell planes [z0, z0 + nz) with nz = n2 / R and z0 = r nz.
Its local lattice is (n0, n1, nz + 2): local plane p is global plane
z0 + p - 1, so planes 1..nz are its own and planes 0 and nz+1 are ghost
planes shared with the rank below and the rank above (periodic over the
ranks).  x and y are not split.  One step does what lf2_step does on one GPU:

  1. ghost planes of the force field: plane nz+1 <- plane 1 of the rank above,
     plane 0 <- plane nz of the rank below (Field::updateHalo across ranks,
     LATfield2_Field_decl.hpp:889-935);
  2. kick, drift and rebin of the local particles in one pass.  A particle
     moves less than one cell per step, so it ends on an own plane or on a
     ghost plane.  The check after the pass is max |v| dtau < res (the whole
     velocity, as the library reports max |v|); a larger move raises, since a
     particle that left by more than one plane cannot be routed;
  3. migration: particles on plane 0 go to the rank below (its plane nz),
     particles on plane nz+1 to the rank above (its plane 1), as
     moveParticles' exchange (LATfield2_Particles.hpp:2176-2799);
  4. deposit of the own particles.  Their CIC weights reach vertex planes
     1..nz+1, and plane nz+1 is added into plane 1 of the rank above: the
     upper-halo fold of scalarProjectionCIC_comm (projections.hpp:194-300).

`project` deposits the other projections of the own particles with the same
folds: the vector and symtensor CIC-NGP projections reach planes 1..nz+1 and
fold upward as the scalar does (vectorProjectionCICNGP_comm,
symtensorProjectionCICNGP_comm, projections.hpp:548-681, :845-976); the
full-CIC projections reach planes 0..nz+1, so plane 0 is also added into
plane nz of the rank below (the Up+Down fold of vectorProjectionCIC_comm and
VecVecProjectionCIC_comm, projections.hpp:1192-1349, :1624-1814).

`pm_force` is the PM operator of lf2_pm_force on the split lattice (cubic,
n a multiple of R), in the manner of the distributed PlanFFT
(LATfield2_PlanFFT_decl.hpp:83-230) with a 1-D split: every rank transforms
its nz planes in 2-D, an all-to-all transpose gives rank r all n planes of
k_y in [r nky, (r+1) nky) (nky = n / R), the 1-D transforms along z, the
Green's function and the inverse 1-D transforms run there, the transpose
goes back, the inverse 2-D transforms give phi on the own planes, and the
central-difference gradient reads phi's ghost planes after fill_ghosts.

`deposit(rho, exact=True)` replaces the FP32 fold by ghost-particle copies
(the top plane of the rank below), so that the fixed-point density is the
single-domain one bit for bit.  `pm_step` chains deposit, pm_force and step.
Checks that can fail on one rank (the speed limit, a lost particle) are
reduced over all ranks first, so that every rank raises together.  Particle
and field files in the reference's layouts are gathered on rank 0
(save_particles, save_field, save_field_binary) and read back by every rank.

Exchanges are point-to-point messages between neighbours (NCCL between GPUs,
gloo between CPU processes), all-to-all for the FFT's transposes and
all-reduce for the checks and conservation sums.  A single rank exchanges with itself, which
gives the periodic single-domain result.  The local work is done by an
engine: CudaEngine (the library's Context) by default; any object with the
same methods can stand in (the tests run the exchange logic on CPU processes
with one).
"""
import numpy as np

from . import _lib
from .core import Context


class CudaEngine:
    """Local work on the GPU through the library's Context."""

    def __init__(self, n_local, res, mode, device=0):
        import torch
        self.torch = torch
        self.n = n_local
        self.dev = torch.device("cuda", device)
        box = tuple(res * v for v in n_local)
        self.ctx = Context(n_local, box=box, mode=mode, device=device)
        self.res = res
        self.has_mass = self.has_id = False

    def set_particles(self, cell, off, vel, mass, gmass, ids):
        self.has_mass, self.has_id = mass is not None, ids is not None
        self._words = None
        self.ctx.set_particles(cell, off, vel, mass=mass, global_mass=gmass, ids=ids)

    def new_field(self, comps):
        t = self.torch.zeros((comps, self.n[2], self.n[1], self.n[0]), dtype=self.torch.float32,
                             device=self.dev)
        return t, self.ctx.field(comps, t)

    def kick_drift(self, F, dtk, dtd):
        """Kick, drift and rebin (max |v| stays on the device, for the
        migration's speed check)."""
        self.ctx.step(F[1], dtk, dtd, None)

    def deposit(self, rho):
        self.ctx.deposit_scalar(rho[1])

    def project(self, kind, f):
        getattr(self.ctx, "deposit_" + kind)(f[1])

    def extract_outside(self, zlo, zhi):
        return self.ctx.extract_z(zlo, zhi, mass=self.has_mass, ids=self.has_id)

    # migration in stream order (SlabDomain.migrate)
    def migration_counts(self, zlo, zhi):
        """CUDA int64 tensor of 6: counts below, above and beyond one plane,
        max |v|^2 after the last kick as float bits, and two words for the
        caller (the neighbours' counts)."""
        if getattr(self, "_counts", None) is None:
            self._counts = self.torch.zeros(6, dtype=self.torch.int64, device=self.dev)
        return self.ctx.slab_count(zlo, zhi, self._counts)

    def extract_records(self, zlo, zhi, n_below, n_above):
        if getattr(self, "_words", None) is None:
            self._words = self.ctx.slab_record_words()
        return self.ctx.slab_extract(zlo, zhi, n_below, n_above, self._words)

    def insert_records(self, a, b):
        self.ctx.slab_insert(a, b)

    # the PM operator's pieces (SlabDomain.pm_force)
    def fft_prepare(self, n, nz, nky):
        from .core import SlabFFT
        key = (n, nz, nky)
        if getattr(self, "_fft_key", None) != key:
            self._fft = SlabFFT(self.ctx, n, nz, nky)
            self._fft_key = key

    def complex_buffer(self, shape):
        return self.torch.empty(shape, dtype=self.torch.complex64, device=self.dev)

    def planes_r2c(self, planes, A):
        self._fft.planes_r2c(planes, A)

    def planes_c2r(self, A, planes):
        self._fft.planes_c2r(A, planes)

    def lines(self, B, direction):
        self._fft.lines(B, direction)

    def green(self, B, ky0, coupling):
        self._fft.green(B, ky0, coupling)

    def gradient(self, phi, F):
        self.ctx.pm_gradient(phi[1], F[1])

    def add(self, parts):
        if int(parts["cell"].shape[0]) == 0:
            return
        self.ctx.add_particles(parts["cell"], parts["off"], parts["vel"], parts.get("mass"),
                               parts.get("id"))

    def particles(self):
        return self.ctx.get_particles(mass=self.has_mass, ids=self.has_id)

    def count(self):
        return self.ctx.count()

    @property
    def device(self):
        return self.dev

    def conservation(self):
        return self.ctx.conservation()

    def synchronize(self):
        self.ctx.synchronize()


class SlabDomain:
    """The global lattice n = (n0, n1, n2) split in z over the ranks of
    `group` (the default torch.distributed group when it is initialised,
    else one rank).  n2 must be a multiple of the number of ranks."""

    def __init__(self, n, box=1.0, mode=_lib.DEPOSIT_FIXED64, engine=None, device=0,
                 group=None):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.size = self.dist.get_world_size(group) if self.dist else 1
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.n = tuple(int(v) for v in n)
        if self.n[2] % self.size:
            raise ValueError(f"n2 = {self.n[2]} is not a multiple of {self.size} ranks")
        self.nz = self.n[2] // self.size
        self.z0 = self.rank * self.nz
        self.res = float(box) / self.n[0]
        self.local_n = (self.n[0], self.n[1], self.nz + 2)
        self.plane = self.n[0] * self.n[1]
        self.mode = mode
        cls = CudaEngine if engine is None else engine
        self.engine = cls(self.local_n, self.res, mode, device)
        self.up = (self.rank + 1) % self.size
        self.down = (self.rank - 1) % self.size

    # ------------------------------------------------------------ messages
    def _shift(self, send, dst, recv, src):
        """send -> rank dst while recv <- rank src (one batch; every rank
        calls it with the same direction)."""
        if self.size == 1:
            recv.copy_(send)
            return
        ops = [self.dist.P2POp(self.dist.isend, send.contiguous(), dst, self.group),
               self.dist.P2POp(self.dist.irecv, recv, src, self.group)]
        for r in self.dist.batch_isend_irecv(ops):
            r.wait()

    def _shift_parts(self, parts, dst, src):
        """A particle set (dict of tensors) to rank dst, one from rank src:
        the counts first, then each array.  An empty array is neither sent
        nor received (both ends know the count)."""
        t = self.engine.torch
        n = int(parts["cell"].shape[0])
        n_send = t.tensor([n], dtype=t.int64, device=parts["cell"].device)
        n_recv = t.zeros_like(n_send)
        self._shift(n_send, dst, n_recv, src)
        k = int(n_recv.item())
        out = {}
        for name in sorted(parts):
            a = parts[name]
            recv = t.empty((k,) + tuple(a.shape[1:]), dtype=a.dtype, device=a.device)
            if self.size == 1:
                recv.copy_(a)
            else:
                ops = []
                if n:
                    ops.append(self.dist.P2POp(self.dist.isend, a.contiguous(), dst, self.group))
                if k:
                    ops.append(self.dist.P2POp(self.dist.irecv, recv, src, self.group))
                if ops:
                    for r in self.dist.batch_isend_irecv(ops):
                        r.wait()
            out[name] = recv
        return out

    def _plane_buf(self, a):
        t = self.engine.torch
        return t.empty(tuple(a[:, 0].shape), dtype=a.dtype, device=a.device)

    # ---------------------------------------------------------------- API
    def set_particles(self, cell, off, vel, global_mass, ids=None):
        """Global particles (numpy, cell indices of the global lattice); each
        rank keeps those of its own planes."""
        cell = np.asarray(cell, np.int64)
        z = cell // self.plane
        mine = (z >= self.z0) & (z < self.z0 + self.nz)
        local = (cell[mine] + (1 - self.z0) * self.plane).astype(np.int32)
        self.engine.set_particles(local, np.ascontiguousarray(np.asarray(off, np.float32)[mine]),
                                  np.ascontiguousarray(np.asarray(vel, np.float32)[mine]), None,
                                  float(global_mass),
                                  None if ids is None else np.asarray(ids, np.int64)[mine])

    def field(self, comps):
        """A local field (comps, nz + 2, n1, n0): (array, engine handle)."""
        return self.engine.new_field(comps)

    def set_own_planes(self, f, global_array):
        """f's own planes from a global array (comps, n2, n1, n0)."""
        src = np.asarray(global_array, np.float32)[:, self.z0:self.z0 + self.nz]
        f[0][:, 1:self.nz + 1] = self.engine.torch.from_numpy(np.ascontiguousarray(src)).to(
            f[0].device)

    def own_planes(self, f):
        """f's own planes as numpy (comps, nz, n1, n0)."""
        return f[0][:, 1:self.nz + 1].cpu().numpy()

    def _from_neighbour(self, a, plane, dst, src):
        """Plane `plane` of a (comps, planes, n1, n0) goes to rank dst; the
        same plane of rank src is returned (the plane itself on one rank)."""
        if self.size == 1:
            return a[:, plane]
        buf = self._plane_buf(a)
        self._shift(a[:, plane], dst, buf, src)
        return buf

    def fill_ghosts(self, f):
        a = f[0]
        a[:, self.nz + 1] = self._from_neighbour(a, 1, self.down, self.up)  # above's plane 1
        a[:, 0] = self._from_neighbour(a, self.nz, self.up, self.down)      # below's plane nz

    def deposit(self, rho, exact=False):
        """Scalar CIC deposit of the own particles with the upper-plane fold;
        the ghost planes of rho end at zero.

        The fold adds two FP32 values at every vertex of plane 1.  With
        exact=True (fixed-point mode, nz >= 2) there is no fold: the rank
        receives copies of the particles on the top plane of the rank below,
        deposits them on its plane 0 together with its own particles, and
        drops them again, so every own vertex converts its one exact integer
        sum, as on a single domain (the density is then bit-identical to the
        single-domain deposit whatever the number of ranks)."""
        a = rho[0]
        if exact:
            if self.mode != _lib.DEPOSIT_FIXED64 or self.nz < 2:
                raise ValueError("exact deposits need the fixed-point mode and 2 or more planes "
                                 "per rank")
            top = self.engine.extract_outside(1, self.nz - 1)  # the own plane nz
            self.engine.add(top)
            ghost = {k: v.clone() for k, v in top.items()}
            ghost["cell"] = ghost["cell"] - self.nz * self.plane  # -> plane 0 of the rank above
            self.engine.add(self._shift_parts(ghost, self.up, self.down))
            self.engine.deposit(rho)
            self.engine.extract_outside(1, self.nz)  # the copies leave again
        else:
            self.engine.deposit(rho)
            a[:, 1] += self._from_neighbour(a, self.nz + 1, self.up, self.down)
        a[:, 0] = 0
        a[:, self.nz + 1] = 0

    # projection -> (components, writes the plane below its particles)
    PROJECTIONS = {"vector": (3, False), "symtensor": (6, False),
                   "vector_cic": (3, True), "vecvec_cic": (6, True)}

    def project(self, kind, f):
        """Projection `kind` (vector, symtensor: CIC-NGP; vector_cic,
        vecvec_cic: full CIC) of the own particles into f, a field of this
        domain with the projection's components, with the slab folds; the
        ghost planes of f end at zero."""
        if kind not in self.PROJECTIONS:
            raise ValueError(f"unknown projection {kind!r}")
        comps, lower = self.PROJECTIONS[kind]
        a = f[0]
        if int(a.shape[0]) != comps:
            raise ValueError(f"{kind} needs a field of {comps} components, got {int(a.shape[0])}")
        self.engine.project(kind, f)
        a[:, 1] += self._from_neighbour(a, self.nz + 1, self.up, self.down)  # rank above's
        if lower:
            a[:, self.nz] += self._from_neighbour(a, 0, self.down, self.up)  # rank below's
        a[:, 0] = 0
        a[:, self.nz + 1] = 0

    def _all_to_all(self, send, recv):
        """Block r of send (split along dim 0) to rank r, block s of recv
        from rank s."""
        if self.size == 1:
            recv.copy_(send)
            return
        t = self.engine.torch
        a, b = t.view_as_real(send), t.view_as_real(recv)
        self.dist.all_to_all_single(b, a, group=self.group)

    def pm_force(self, rho, F, coupling, phi=None):
        """F (3 components) = -grad phi with lap7(phi) = coupling (rho - mean
        rho) on the global lattice, from rho's own planes (after deposit);
        phi (1 component), when given, receives the potential.  F's and
        phi's ghost planes are filled."""
        n = self.n[0]
        if self.n[1] != n or self.n[2] != n:
            raise ValueError("the PM operator needs a cubic lattice")
        R, nz = self.size, self.nz
        nky, nkx = n // R, n // 2 + 1
        e = self.engine
        e.fft_prepare(n, nz, nky)
        A = e.complex_buffer((nz, n, nkx))
        e.planes_r2c(rho[0][0, 1:nz + 1], A)
        send = A.view(nz, R, nky, nkx).permute(1, 0, 2, 3).contiguous()  # [to rank][z][ky][kx]
        B = e.complex_buffer((n, nky, nkx))                              # [z from all][ky][kx]
        self._all_to_all(send, B.view(R, nz, nky, nkx))
        e.lines(B, _lib.FFT_FORWARD)
        e.green(B, self.rank * nky, coupling)
        e.lines(B, _lib.FFT_BACKWARD)
        back = e.complex_buffer((R, nz, nky, nkx))                       # [from rank][z][ky][kx]
        self._all_to_all(B.view(R, nz, nky, nkx), back)
        A = back.permute(1, 0, 2, 3).reshape(nz, n, nkx).contiguous()
        if phi is None:
            if getattr(self, "_phi", None) is None:
                self._phi = self.field(1)  # scratch potential, kept for later calls
            phi = self._phi
        p = phi
        e.planes_c2r(A, p[0][0, 1:nz + 1])
        self.fill_ghosts(p)
        e.gradient(p, F)
        self.fill_ghosts(F)

    def _shift_records(self, send, dst, k_recv, src):
        """Migration records (k, words) to rank dst while k_recv records come
        from rank src, in one message each way; an empty set is neither sent
        nor received (both ends know the counts)."""
        t = self.engine.torch
        recv = t.empty((int(k_recv), int(send.shape[1])), dtype=send.dtype, device=send.device)
        ops = []
        if int(send.shape[0]):
            ops.append(self.dist.P2POp(self.dist.isend, send.contiguous(), dst, self.group))
        if int(k_recv):
            ops.append(self.dist.P2POp(self.dist.irecv, recv, src, self.group))
        if ops:
            for r in self.dist.batch_isend_irecv(ops):
                r.wait()
        return recv

    def migrate(self, move_scale=0.0):
        """Particles on a ghost plane go to the neighbour that owns it.  The
        counts and checks stay on the device until one read per call (the
        host's only wait): this rank's counts below and above, the counts
        its neighbours will send (exchanged first), and two checks reduced
        over the ranks, so that every rank raises together and none is left
        waiting in the exchange: a particle more than one plane outside, and
        (move_scale > 0: dtau / cell size of the last drift) max |v| after
        the last kick times move_scale reaching 1.  The records then travel
        in one message per direction, sized from the counts."""
        buf = self.engine.migration_counts(1, self.nz)
        # buf: below, above, beyond, max |v|^2 bits | from below, from above
        if self.size > 1:
            self.dist.all_reduce(buf[2:4], op=self.dist.ReduceOp.MAX, group=self.group)
            self._shift(buf[1:2], self.up, buf[4:5], self.down)
            self._shift(buf[0:1], self.down, buf[5:6], self.up)
        host = buf.tolist()
        vmax = float(np.sqrt(np.array([host[3]], np.uint32).view(np.float32)[0]))
        if move_scale > 0 and vmax * move_scale >= 1.0:
            raise RuntimeError(f"max |v| dtau = {vmax * move_scale:.3f} cells: the slab "
                               "decomposition moves particles by less than one cell per step")
        if host[2]:
            raise RuntimeError("a particle left the slab by more than one plane")
        n_below, n_above = host[0], host[1]
        below, above = self.engine.extract_records(1, self.nz, n_below, n_above)
        if self.size == 1:
            from_below, from_above = above, below
        else:
            from_below = self._shift_records(above, self.up, host[4], self.down)
            from_above = self._shift_records(below, self.down, host[5], self.up)
        self.engine.insert_records(from_below, from_above)

    def _all_reduce(self, values, op):
        """FP64 values reduced over the ranks (op "sum" or "max"); every rank
        takes part, so that all of them act on the same result."""
        if self.size == 1:
            return np.asarray(values, np.float64)
        t = self.engine.torch
        x = t.tensor(np.asarray(values, np.float64), device=self.engine.device)
        red = self.dist.ReduceOp.SUM if op == "sum" else self.dist.ReduceOp.MAX
        self.dist.all_reduce(x, op=red, group=self.group)
        return x.cpu().numpy()

    def conservation(self):
        """FP64 total mass, momentum sum and max |v| over all ranks (the
        reductions of cout_particle_velocity_stats and updateVel's SUM/MAX
        outputs, LATfield2_Particles.hpp:543-583, :645-743)."""
        m, mom, vmax = self.engine.conservation()
        s = self._all_reduce([m, mom[0], mom[1], mom[2]], "sum")
        return float(s[0]), s[1:4], float(self._all_reduce([vmax], "max")[0])

    def step(self, F, dtau_kick, dtau_drift, rho=None):
        """fill_ghosts(F), kick + drift + rebin, migrate, and (rho given)
        deposit.  The speed check (max |v| dtau below one cell, max |v| over
        all ranks) travels with the migration's counts, so the host waits
        once per step."""
        self.fill_ghosts(F)
        self.engine.kick_drift(F, dtau_kick, dtau_drift)
        self.migrate(abs(float(dtau_drift)) / self.res)
        if rho is not None:
            self.deposit(rho)

    def pm_step(self, rho, F, dtau_kick, dtau_drift, coupling, exact=False):
        """One self-consistent particle-mesh step over the slabs: deposit
        rho from the particles (exact: see deposit), the PM force F from rho
        (pm_force), then kick + drift + rebin and migration (step)."""
        self.deposit(rho, exact)
        self.pm_force(rho, F, coupling)
        self.step(F, dtau_kick, dtau_drift)

    def count(self):
        return self.engine.count()

    def save_particles(self, path, global_mass, relativistic=0, type_name="part_simple"):
        """All ranks' particles (which must carry IDs) as one snapshot in the
        layout of Particles::saveHDF5 (latfield2_b200.snapshot): rank 0
        gathers every rank's records, in rank order, and writes `path`."""
        from . import snapshot as S
        p = self.particles_global()
        if "id" not in p:
            raise ValueError("a snapshot needs particle IDs")
        pos = S.cells_to_positions(p["cell"], p["off"], self.n, self.res)
        data = S.records(p["cell"], pos, p["vel"], p["id"])
        parts = [data]
        if self.size > 1:
            parts = [None] * self.size if self.rank == 0 else None
            self.dist.gather_object(data, parts, dst=0, group=self.group)
        if self.rank == 0:
            box = tuple(self.res * v for v in self.n)
            attrs, num, offs, size = S.description(self.n, box, self.size,
                                                   [d.shape[0] for d in parts])
            S.write(path, np.concatenate(parts), S.part_info(global_mass, relativistic, type_name),
                    attrs, num, offs, size)
        if self.size > 1:
            self.dist.barrier(group=self.group)

    def load_particles(self, path):
        """Particles of a snapshot (saved from any number of ranks): every
        rank reads it and keeps the particles of its own planes, as
        Particles::loadHDF5 adds the records of the blocks that overlap its
        box.  Returns the part_info record."""
        from . import snapshot as S
        snap = S.read(path)
        S.check_box(snap, tuple(self.res * v for v in self.n))
        ids, pos, vel = S.columns(snap["data"])
        cell, off = S.positions_to_cells(pos, self.n, self.res)
        info = snap["part_info"][0]
        self.set_particles(cell, off, vel.astype(np.float32), float(info["mass"]), ids=ids)
        return info

    def _field_global(self, f, dtype):
        """f's own planes of every rank as one global array (n2, n1, n0,
        comps) on rank 0 (None elsewhere)."""
        a = np.ascontiguousarray(self.own_planes(f).astype(dtype))  # (comps, nz, n1, n0)
        parts = [a]
        if self.size > 1:
            parts = [None] * self.size if self.rank == 0 else None
            self.dist.gather_object(a, parts, dst=0, group=self.group)
        if self.rank != 0:
            return None
        return np.ascontiguousarray(np.concatenate(parts, axis=1).transpose(1, 2, 3, 0))

    def _barrier(self):
        if self.size > 1:
            self.dist.barrier(group=self.group)

    def save_field(self, path, f, dataset_name="data", dtype=np.float64):
        """The field as the dataset of Field::saveHDF5 (latfield2_b200.
        snapshot.save_field), written by rank 0 from every rank's planes."""
        g = self._field_global(f, dtype)
        if g is not None:
            with open(path, "wb") as fp:
                np.savez(fp, **{dataset_name: g[..., 0] if g.shape[3] == 1 else g})
        self._barrier()

    def save_field_binary(self, path, f, real_bytes=8):
        """The file of Field::write (latfield2_b200.snapshot.write_field_binary)
        for the whole lattice, written by rank 0."""
        g = self._field_global(f, np.float64 if real_bytes == 8 else np.float32)
        if g is not None:
            with open(path, "wb") as fp:
                fp.write(g.tobytes())
        self._barrier()

    def _load_global(self, f, g):
        comps = int(f[0].shape[0])
        want = self.n[::-1] + (comps,)
        g = g.reshape(self.n[2], self.n[1], self.n[0], -1)
        if tuple(g.shape) != want:
            raise ValueError(f"the file holds {g.shape}, the field {want}")
        self.set_own_planes(f, g.transpose(3, 0, 1, 2))

    def load_field(self, path, f, dataset_name="data"):
        """Every rank reads its own planes of a save_field dataset, then the
        ghost planes are filled (Field::loadHDF5 and updateHalo)."""
        with np.load(path, allow_pickle=False) as z:
            self._load_global(f, z[dataset_name])
        self.fill_ghosts(f)

    def load_field_binary(self, path, f, real_bytes=8):
        """Field::read of a save_field_binary file, then the ghost planes."""
        self._load_global(f, np.fromfile(path, dtype=np.float64 if real_bytes == 8 else
                                         np.float32))
        self.fill_ghosts(f)

    def particles_global(self):
        """The local particles with global cell indices (numpy dict)."""
        p = self.engine.particles()
        p["cell"] = (np.asarray(p["cell"], np.int64) + (self.z0 - 1) * self.plane).astype(np.int32)
        return p
