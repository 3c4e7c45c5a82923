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
    with CudaEngine; global particle mass and the fixed-point mode only."""

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
        return float(np.sqrt((v64 * v64).sum(axis=1).max())) if v.shape[0] else 0.0

    def deposit(self, rho):
        acc = self.O.state_deposit_fixed(self.n, self.cell, self.off)
        scale = np.float32(2.0 ** -32 * self.gmass / (self.res ** 3))
        rho[0][0] = self.torch.from_numpy(self.O.fixed_to_f32(acc, scale).reshape(rho[0].shape[1:]))

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

    def synchronize(self):
        pass
