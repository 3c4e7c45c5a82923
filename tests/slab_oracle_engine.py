"""A CPU engine for latfield2_b200.distributed.SlabDomain: the local work of
a rank done by the oracle's restatement of the device arithmetic (FP32 kick
and drift with the device's fmaf order, int64 fixed-point deposit), bit-exact
with the CUDA engine.  TEST INFRASTRUCTURE: it lets the exchange logic of the
slab decomposition run as gloo ranks on CPU processes."""
import numpy as np

from latfield2_b200 import _lib


class OracleEngine:
    """Local work on the CPU with the oracle's restatement of the device
    arithmetic (FP32 kick and drift, int64 fixed-point deposit), bit-exact
    with CudaEngine, and the oracle's FP64 projections; global particle mass
    and the fixed-point mode only."""

    def __init__(self, n_local, res, mode, device=None):
        import torch
        from oracle import oracle as O
        if mode != _lib.DEPOSIT_FIXED64:
            raise ValueError("OracleEngine restates the fixed-point deposit only")
        self.torch = torch
        self.O = O
        self.n = n_local
        self.res = res
        self.cell = np.zeros(0, np.int32)
        self.off = np.zeros((0, 3), np.float32)
        self.vel = np.zeros((0, 3), np.float32)
        self.ids = None
        self.vmax = 0.0

    def set_particles(self, cell, off, vel, mass, gmass, ids):
        if mass is not None:
            raise ValueError("OracleEngine takes a global particle mass")
        self.cell = np.array(cell, np.int32)
        self.off = np.array(off, np.float32)
        self.vel = np.array(vel, np.float32)
        self.ids = None if ids is None else np.array(ids, np.int64)
        self.gmass = gmass

    def new_field(self, comps):
        return self.torch.zeros((comps, self.n[2], self.n[1], self.n[0]), dtype=self.torch.float32), None

    def kick_drift(self, F, dtk, dtd):
        v = self.O.state_kick(self.n, self.cell, self.off, self.vel, F[0].numpy(), np.float32(dtk))
        c, o, bad = self.O.state_drift(self.n, self.cell, self.off, v, np.float32(dtd / self.res))
        if bad:
            raise RuntimeError("non-finite particle state")
        self.cell, self.off, self.vel = c, o, v
        v64 = v.astype(np.float64)
        self.vmax = float(np.sqrt((v64 * v64).sum(axis=1).max())) if v.shape[0] else 0.0

    def deposit(self, rho):
        acc = self.O.state_deposit_fixed(self.n, self.cell, self.off)
        scale = np.float32(2.0 ** -32 * self.gmass / (self.res ** 3))
        rho[0][0] = self.torch.from_numpy(self.O.fixed_to_f32(acc, scale).reshape(rho[0].shape[1:]))

    def project(self, kind, f):
        """The oracle's FP64 projection on the local periodic lattice (halo 1,
        with its _comm fold), stored in FP32 as the device stores it."""
        cs, order = self.O.lists_from_insertion(self.n, self.cell)
        pos = self.O.state_to_pos(self.n, self.res, self.cell, self.off)[order]
        vel = self.vel.astype(np.float64)[order]
        fn = {"vector": self.O.vector_cicngp, "symtensor": self.O.symtensor_cicngp,
              "vector_cic": self.O.vector_cic, "vecvec_cic": self.O.vecvec_cic}[kind]
        g = self.O.interior(fn(self.n, 1, self.res, cs, pos, vel, gmass=self.gmass), self.n, 1)
        f[0][:] = self.torch.from_numpy(g.astype(np.float32))

    # the PM operator's pieces in FP64 numpy, stored in complex64 / FP32
    def fft_prepare(self, n, nz, nky):
        self.fft_n = n

    def complex_buffer(self, shape):
        return self.torch.empty(shape, dtype=self.torch.complex64)

    def planes_r2c(self, planes, A):
        a = np.fft.rfft2(planes.numpy().astype(np.float64), axes=(1, 2))
        A.copy_(self.torch.from_numpy(a.astype(np.complex64)))

    def planes_c2r(self, A, planes):
        n = self.fft_n
        r = np.fft.irfft2(A.numpy().astype(np.complex128), s=(n, n), axes=(1, 2)) * float(n * n)
        planes.copy_(self.torch.from_numpy(r.astype(np.float32)))

    def lines(self, B, direction):
        b = B.numpy().astype(np.complex128)
        b = np.fft.fft(b, axis=0) if direction == 1 else np.fft.ifft(b, axis=0) * b.shape[0]
        B.copy_(self.torch.from_numpy(b.astype(np.complex64)))

    def green(self, B, ky0, coupling):
        from oracle import fft_oracle as FO
        n = self.fft_n
        nky = int(B.shape[1])
        lam = FO.laplacian_eigenvalues(n, self.res)[:, ky0:ky0 + nky, :]
        g = np.where(lam == 0.0, 0.0, coupling / np.where(lam == 0.0, 1.0, lam)) / float(n) ** 3
        B.copy_(self.torch.from_numpy((B.numpy().astype(np.complex128) * g).astype(np.complex64)))

    def gradient(self, phi, F):
        p = phi[0][0].numpy().astype(np.float64)
        for c, axis in enumerate((2, 1, 0)):
            g = -(np.roll(p, -1, axis) - np.roll(p, 1, axis)) / (2.0 * self.res)
            F[0][c] = self.torch.from_numpy(g.astype(np.float32))

    def extract_outside(self, zlo, zhi):
        z = self.cell // (self.n[0] * self.n[1])
        out = (z < zlo) | (z > zhi)
        parts = {"cell": self.torch.from_numpy(self.cell[out].copy()),
                 "off": self.torch.from_numpy(self.off[out].copy()),
                 "vel": self.torch.from_numpy(self.vel[out].copy())}
        if self.ids is not None:
            parts["id"] = self.torch.from_numpy(self.ids[out].copy())
            self.ids = self.ids[~out]
        self.cell, self.off, self.vel = self.cell[~out], self.off[~out], self.vel[~out]
        return parts

    # migration records: int32 words (cell, offset and velocity bits, id
    # low and high words), the library's record layout
    def migration_counts(self, zlo, zhi):
        z = self.cell // (self.n[0] * self.n[1])
        far = (z < zlo - 1) | (z > zhi + 1)
        v2 = int(np.array([self.vmax * self.vmax], np.float32).view(np.uint32)[0])
        return self.torch.tensor([int((z < zlo).sum()), int((z > zhi).sum()), int(far.sum()),
                                  v2, 0, 0], dtype=self.torch.int64)

    def extract_records(self, zlo, zhi, n_below, n_above):
        plane = self.n[0] * self.n[1]
        z = self.cell // plane
        lo, hi = z < zlo, z > zhi
        if int(lo.sum()) != n_below or int(hi.sum()) != n_above:
            raise RuntimeError("extract_records: counts differ from migration_counts")
        nz = zhi - zlo + 1

        def records(sel, dz):
            cols = [(self.cell[sel] + dz * plane).astype(np.int32)[:, None],
                    self.off[sel].view(np.int32), self.vel[sel].view(np.int32)]
            if self.ids is not None:
                cols.append(self.ids[sel].view(np.int32).reshape(-1, 2))
            return self.torch.from_numpy(np.ascontiguousarray(np.concatenate(cols, axis=1)))

        below, above = records(lo, nz), records(hi, -nz)
        keep = ~(lo | hi)
        self.cell, self.off, self.vel = self.cell[keep], self.off[keep], self.vel[keep]
        if self.ids is not None:
            self.ids = self.ids[keep]
        return below, above

    def insert_records(self, a, b):
        r = np.concatenate([a.numpy(), b.numpy()])
        self.cell = np.concatenate([self.cell, r[:, 0]])
        self.off = np.concatenate([self.off, np.ascontiguousarray(r[:, 1:4]).view(np.float32)])
        self.vel = np.concatenate([self.vel, np.ascontiguousarray(r[:, 4:7]).view(np.float32)])
        if self.ids is not None:
            self.ids = np.concatenate([self.ids, np.ascontiguousarray(r[:, 7:9]).view(np.int64)[:, 0]])

    def add(self, parts):
        self.cell = np.concatenate([self.cell, parts["cell"].numpy()])
        self.off = np.concatenate([self.off, parts["off"].numpy()])
        self.vel = np.concatenate([self.vel, parts["vel"].numpy()])
        if self.ids is not None:
            self.ids = np.concatenate([self.ids, parts["id"].numpy()])

    def particles(self):
        out = {"cell": self.cell.copy(), "off": self.off.copy(), "vel": self.vel.copy()}
        if self.ids is not None:
            out["id"] = self.ids.copy()
        return out

    def count(self):
        return int(self.cell.shape[0])

    @property
    def device(self):
        return self.torch.device("cpu")

    def conservation(self):
        """FP64 mass, momentum sum and max |v| of the local particles."""
        v = self.vel.astype(np.float64)
        npart = v.shape[0]
        vmax = float(np.sqrt((v * v).sum(axis=1).max())) if npart else 0.0
        return self.gmass * npart, self.gmass * v.sum(axis=0), vmax

    def synchronize(self):
        pass
