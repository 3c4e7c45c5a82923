"""Thin object wrapper over the C ABI (include/lf2gpu.h).

`Context` owns one lf2_ctx: the lattice geometry, the device particle store
and the deposit mode.  Arrays are numpy (host) or torch CUDA tensors
(device); the pointer kind is chosen from the argument type.
"""
import ctypes

import numpy as np

from . import _lib

_c = ctypes


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _ptr(x):
    if x is None:
        return None, _lib.PTR_HOST
    if _is_torch(x):
        if not x.is_cuda:
            raise ValueError("torch tensors passed to lf2 must be CUDA tensors")
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return _c.c_void_p(x.data_ptr()), _lib.PTR_DEVICE
    if not x.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return _c.c_void_p(x.ctypes.data), _lib.PTR_HOST


def _same_kind(*arrs):
    kinds = {(_is_torch(a)) for a in arrs if a is not None}
    if len(kinds) > 1:
        raise ValueError("mix of host and device arrays in one call")
    return _lib.PTR_DEVICE if kinds == {True} else _lib.PTR_HOST


class FieldHandle:
    """A device field (FP32, component-major, no halo) owned by the context or
    wrapping a caller's CUDA tensor."""

    def __init__(self, ctx, comps, tensor=None):
        self.ctx = ctx
        self.comps = comps
        self.tensor = tensor
        h = _c.c_void_p()
        lib = _lib.load()
        if tensor is None:
            _lib.check(ctx.h, lib.lf2_field_create(ctx.h, comps, _c.byref(h)), "field_create")
        else:
            if tensor.dtype.itemsize != 4 or tensor.numel() != comps * ctx.nsites:
                raise ValueError("tensor must hold comps * nsites float32 values")
            _lib.check(ctx.h, lib.lf2_field_wrap(ctx.h, comps, _c.c_void_p(tensor.data_ptr()),
                                                 _c.byref(h)), "field_wrap")
        self.h = h

    def close(self):
        if self.h:
            _lib.load().lf2_field_destroy(self.ctx.h, self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self, halo=0, dtype=np.float32, fill_halo=False):
        """Reference layout: shape (n2+2h, n1+2h, n0+2h, comps)."""
        n = self.ctx.n
        out = np.empty((n[2] + 2 * halo, n[1] + 2 * halo, n[0] + 2 * halo, self.comps), dtype=dtype)
        p, kind = _ptr(out)
        _lib.check(self.ctx.h, _lib.load().lf2_field_export(
            self.ctx.h, self.h, p, halo, out.itemsize, 1 if fill_halo else 0, kind), "export")
        return out

    def export_internal(self):
        """Internal layout copy: shape (comps, n2, n1, n0), float32."""
        return self.export(0, np.float32).transpose(3, 0, 1, 2).copy()

    def import_(self, arr, halo=0):
        p, kind = _ptr(arr)
        _lib.check(self.ctx.h, _lib.load().lf2_field_import(
            self.ctx.h, self.h, p, halo, arr.dtype.itemsize, kind), "import")

    def zero(self):
        _lib.check(self.ctx.h, _lib.load().lf2_field_zero(self.ctx.h, self.h), "zero")


class KFieldHandle:
    """A device k-field: the Fourier transform of a `comps`-component real
    field (PlanFFT's Field<Imag>), complex64 on the device."""

    def __init__(self, ctx, comps):
        self.ctx = ctx
        self.comps = comps
        h = _c.c_void_p()
        _lib.check(ctx.h, _lib.load().lf2_kfield_create(ctx.h, comps, _c.byref(h)), "kfield_create")
        self.h = h

    def close(self):
        if self.h:
            _lib.load().lf2_kfield_destroy(self.ctx.h, self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _shape(self):
        n = self.ctx.n
        return (n[1], n[2], n[0] // 2 + 1, self.comps)

    def export(self, dtype=np.complex128):
        """Reference layout: shape (n, n, n/2+1, comps) indexed
        [k_y][k_z][k_x][c], complex."""
        out = np.empty(self._shape(), dtype=dtype)
        p, kind = _ptr(out)
        _lib.check(self.ctx.h, _lib.load().lf2_kfield_export(
            self.ctx.h, self.h, p, out.itemsize // 2, kind), "kfield_export")
        return out

    def import_(self, arr):
        arr = np.ascontiguousarray(arr)
        if arr.shape != self._shape() or arr.dtype not in (np.complex64, np.complex128):
            raise ValueError(f"k-field array must be complex with shape {self._shape()}")
        p, kind = _ptr(arr)
        _lib.check(self.ctx.h, _lib.load().lf2_kfield_import(
            self.ctx.h, self.h, p, arr.itemsize // 2, kind), "kfield_import")


class SlabFFT:
    """The transforms of the PM operator over z slabs (lf2_slab_fft_*): 2-D
    transforms of a rank's nz planes of an n^3 lattice, 1-D transforms along
    the outer axis of a [n][nky][n/2+1] block, and the Green's function on
    it.  Complex arrays are torch complex64 tensors on the context's device."""

    def __init__(self, ctx, n, nz, nky):
        self.ctx = ctx
        h = _c.c_void_p()
        ctx._check(_lib.load().lf2_slab_fft_create(ctx.h, int(n), int(nz), int(nky), _c.byref(h)),
                   "slab_fft_create")
        self.h = h
        self.n, self.nz, self.nky = int(n), int(nz), int(nky)

    def close(self):
        if getattr(self, "h", None):
            _lib.load().lf2_slab_fft_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptr(t, shape, dtype):
        if tuple(t.shape) != tuple(shape) or t.dtype != dtype or not t.is_contiguous():
            raise ValueError(f"expected a contiguous {dtype} tensor of shape {shape}")
        return _c.c_void_p(t.data_ptr())

    def planes_r2c(self, planes, A):
        import torch
        n, nz = self.n, self.nz
        self.ctx._check(_lib.load().lf2_slab_fft_planes_r2c(
            self.h, self._ptr(planes, (nz, n, n), torch.float32),
            self._ptr(A, (nz, n, n // 2 + 1), torch.complex64)), "slab_fft_planes_r2c")

    def planes_c2r(self, A, planes):
        import torch
        n, nz = self.n, self.nz
        self.ctx._check(_lib.load().lf2_slab_fft_planes_c2r(
            self.h, self._ptr(A, (nz, n, n // 2 + 1), torch.complex64),
            self._ptr(planes, (nz, n, n), torch.float32)), "slab_fft_planes_c2r")

    def lines(self, B, direction):
        import torch
        n = self.n
        self.ctx._check(_lib.load().lf2_slab_fft_lines(
            self.h, self._ptr(B, (n, self.nky, n // 2 + 1), torch.complex64), int(direction)),
            "slab_fft_lines")

    def green(self, B, ky0, coupling):
        import torch
        n = self.n
        self.ctx._check(_lib.load().lf2_slab_green(
            self.h, self._ptr(B, (n, self.nky, n // 2 + 1), torch.complex64), int(ky0),
            float(coupling)), "slab_green")


class Context:
    def __init__(self, n, box=1.0, mode=_lib.DEPOSIT_FP32, device=0, stream=None):
        if np.isscalar(n):
            n = (int(n),) * 3
        if np.isscalar(box):
            box = tuple(float(box) * ni / n[0] for ni in n)
        self.n = tuple(int(v) for v in n)
        self.box = tuple(float(b) for b in box)
        self.nsites = self.n[0] * self.n[1] * self.n[2]
        self.nbricks = 1
        for v in self.n:
            self.nbricks *= -(-v // 16)  # bricks of 16^3 cells
        self.res = self.box[0] / self.n[0]
        self.mode = mode
        self.device = int(device)
        lib = _lib.load()
        h = _c.c_void_p()
        na = (_c.c_int * 3)(*self.n)
        ba = (_c.c_double * 3)(*self.box)
        st = _c.c_void_p(stream) if stream is not None else None
        s = lib.lf2_create(_c.byref(h), device, na, ba, mode, st)
        if s != _lib.LF2_OK:
            raise _lib.LF2Error(s, f"lf2_create(n={self.n}, box={self.box}, mode={mode})")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib.load().lf2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status, what):
        _lib.check(self.h, status, what)

    def set_stream(self, stream):
        self._check(_lib.load().lf2_set_stream(self.h, _c.c_void_p(stream)), "set_stream")

    # ---------------------------------------------------------------- particles
    def set_particles(self, cell, off, vel, mass=None, global_mass=0.0, ids=None):
        kind = _same_kind(cell, off, vel, mass, ids)
        n = int(cell.shape[0])
        args = [_ptr(a)[0] for a in (cell, off, vel, mass)]
        self._check(_lib.load().lf2_particles_set(
            self.h, n, args[0], args[1], args[2], args[3], float(global_mass),
            _ptr(ids)[0], kind), "particles_set")

    def set_positions(self, pos, vel, mass=None, global_mass=0.0, ids=None):
        pos = np.ascontiguousarray(pos)
        vel = np.ascontiguousarray(vel, dtype=pos.dtype)
        self._check(_lib.load().lf2_particles_set_pos(
            self.h, int(pos.shape[0]), _ptr(pos)[0], _ptr(vel)[0], pos.itemsize,
            _ptr(mass)[0], float(global_mass), _ptr(ids)[0]), "particles_set_pos")

    def count(self):
        n = _c.c_int64()
        self._check(_lib.load().lf2_particles_count(self.h, _c.byref(n)), "count")
        return n.value

    def get_particles(self, mass=False, ids=False):
        n = self.count()
        cell = np.empty(n, np.int32)
        off = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        m = np.empty(n, np.float32) if mass else None
        i = np.empty(n, np.int64) if ids else None
        self._check(_lib.load().lf2_particles_get(
            self.h, _ptr(cell)[0], _ptr(off)[0], _ptr(vel)[0], _ptr(m)[0], _ptr(i)[0],
            _lib.PTR_HOST), "particles_get")
        out = {"cell": cell, "off": off, "vel": vel}
        if mass:
            out["mass"] = m
        if ids:
            out["id"] = i
        return out

    def get_positions(self, dtype=np.float64, ids=False):
        n = self.count()
        pos = np.empty((n, 3), dtype)
        vel = np.empty((n, 3), dtype)
        i = np.empty(n, np.int64) if ids else None
        self._check(_lib.load().lf2_particles_get_pos(
            self.h, _ptr(pos)[0], _ptr(vel)[0], pos.itemsize, _ptr(i)[0]), "particles_get_pos")
        return (pos, vel, i) if ids else (pos, vel)

    def extract_z(self, z_lo, z_hi, mass=False, ids=False):
        """Removes every particle whose cell z lies outside [z_lo, z_hi] and
        returns them as CUDA tensors {cell, off, vel[, mass][, id]} (the
        migration step of a slab decomposition)."""
        import torch
        lib = _lib.load()
        dev = torch.device("cuda", self.device)
        n = _c.c_int64()
        st = lib.lf2_particles_extract_z(self.h, int(z_lo), int(z_hi), 0, None, None, None, None,
                                         None, _c.byref(n))
        if st != 0 and n.value == 0:
            self._check(st, "extract_z")
        cap = n.value
        out = {"cell": torch.empty(cap, dtype=torch.int32, device=dev),
               "off": torch.empty((cap, 3), dtype=torch.float32, device=dev),
               "vel": torch.empty((cap, 3), dtype=torch.float32, device=dev)}
        if mass:
            out["mass"] = torch.empty(cap, dtype=torch.float32, device=dev)
        if ids:
            out["id"] = torch.empty(cap, dtype=torch.int64, device=dev)
        if cap == 0:
            return out

        def p(k):
            return _c.c_void_p(out[k].data_ptr()) if k in out else None
        self._check(lib.lf2_particles_extract_z(self.h, int(z_lo), int(z_hi), cap, p("cell"),
                                                p("off"), p("vel"), p("mass"), p("id"),
                                                _c.byref(n)), "extract_z")
        return out

    def slab_record_words(self):
        """32-bit words of one migration record of this store."""
        w = _c.c_int()
        self._check(_lib.load().lf2_slab_record_words(self.h, _c.byref(w)), "slab_record_words")
        return w.value

    def slab_count(self, z_lo, z_hi, out):
        """out[:4] (CUDA int64 tensor) <- the particles below z_lo, above
        z_hi and more than one plane outside [z_lo, z_hi], and max |v|^2
        after the last kick as float bits; in stream order (no wait)."""
        self._check(_lib.load().lf2_slab_count(self.h, int(z_lo), int(z_hi),
                                               _c.c_void_p(out.data_ptr())), "slab_count")
        return out

    def slab_extract(self, z_lo, z_hi, n_below, n_above, words=0):
        """The particles outside [z_lo, z_hi] leave the store as migration
        records (CUDA int32 tensors of (n, record_words)): those below z_lo
        and those above z_hi, with the cell index of the neighbouring slab.
        n_below / n_above are slab_count's counts; words, when given, is
        slab_record_words().  No wait."""
        import torch
        dev = torch.device("cuda", self.device)
        w = words if words else self.slab_record_words()
        below = torch.empty((int(n_below), w), dtype=torch.int32, device=dev)
        above = torch.empty((int(n_above), w), dtype=torch.int32, device=dev)
        self._check(_lib.load().lf2_slab_extract(
            self.h, int(z_lo), int(z_hi), int(n_below), _c.c_void_p(below.data_ptr()),
            int(n_above), _c.c_void_p(above.data_ptr())), "slab_extract")
        return below, above

    def slab_insert(self, a, b):
        """Migration records a and b (CUDA int32 tensors of (n, record_words))
        join the store; no wait unless the store must grow."""
        self._check(_lib.load().lf2_slab_insert(
            self.h, int(a.shape[0]), _c.c_void_p(a.data_ptr()), int(b.shape[0]),
            _c.c_void_p(b.data_ptr())), "slab_insert")

    def add_particles(self, cell, off, vel, mass=None, ids=None):
        """New particles (cell, offsets, velocities[, mass][, ids]) join the
        store (numpy arrays or CUDA tensors)."""
        kind = _same_kind(cell, off, vel, mass, ids)
        self._check(_lib.load().lf2_particles_add(
            self.h, int(cell.shape[0]), _ptr(cell)[0], _ptr(off)[0], _ptr(vel)[0], _ptr(mass)[0],
            _ptr(ids)[0], kind), "particles_add")

    def checkpoint_save(self, path):
        """The particle store to `path` (exact restart)."""
        self._check(_lib.load().lf2_checkpoint_save(self.h, str(path).encode()), "checkpoint_save")

    def checkpoint_load(self, path):
        """A store saved by checkpoint_save (same lattice, box and mode)."""
        self._check(_lib.load().lf2_checkpoint_load(self.h, str(path).encode()), "checkpoint_load")

    def cell_counts(self):
        out = np.empty(self.nsites, np.int32)
        self._check(_lib.load().lf2_cell_counts(self.h, _ptr(out)[0], _lib.PTR_HOST), "cell_counts")
        return out

    # ------------------------------------------------------------------- fields
    def field(self, comps, tensor=None):
        return FieldHandle(self, comps, tensor)

    def kfield(self, comps=1):
        return KFieldHandle(self, comps)

    def fft_forward(self, r, k):
        """PlanFFT::execute(FFT_FORWARD): k = unnormalised transform of r."""
        self._check(_lib.load().lf2_fft_forward(self.h, r.h, k.h), "fft_forward")

    def fft_backward(self, k, r):
        """PlanFFT::execute(FFT_BACKWARD): r = unnormalised inverse of k."""
        self._check(_lib.load().lf2_fft_backward(self.h, k.h, r.h), "fft_backward")

    def pm_force(self, rho, F, coupling=1.0, phi=None):
        """F = -grad phi (central differences), lap7(phi) = coupling (rho - mean)."""
        self._check(_lib.load().lf2_pm_force(self.h, rho.h, None if phi is None else phi.h, F.h,
                                             float(coupling)), "pm_force")

    def pm_gradient(self, phi, F):
        """F = -grad phi by central differences on this lattice (periodic)."""
        self._check(_lib.load().lf2_pm_gradient(self.h, phi.h, F.h), "pm_gradient")

    def halo_fill(self, tensor, comps, halo):
        self._check(_lib.load().lf2_halo_fill(self.h, _c.c_void_p(tensor.data_ptr()), comps, halo,
                                              tensor.element_size()), "halo_fill")

    # --------------------------------------------------------------- operations
    def deposit_scalar(self, f):
        self._check(_lib.load().lf2_deposit_scalar(self.h, f.h), "deposit_scalar")

    def deposit_vector(self, f):
        self._check(_lib.load().lf2_deposit_vector_cicngp(self.h, f.h), "deposit_vector")

    def deposit_symtensor(self, f):
        self._check(_lib.load().lf2_deposit_symtensor_cicngp(self.h, f.h), "deposit_symtensor")

    def deposit_vector_cic(self, f):
        """vectorProjectionCIC: m v / res^3 on the links, 3 components."""
        self._check(_lib.load().lf2_deposit_vector_cic(self.h, f.h), "deposit_vector_cic")

    def deposit_vecvec_cic(self, f):
        """VecVecProjectionCIC: symmetric m v_i v_j / res^3, 6 components."""
        self._check(_lib.load().lf2_deposit_vecvec_cic(self.h, f.h), "deposit_vecvec_cic")

    def gather_kick(self, F, dtau, want_max_v=False):
        mv = _c.c_double()
        self._check(_lib.load().lf2_gather_kick(self.h, F.h, float(dtau),
                                                _c.byref(mv) if want_max_v else None),
                    "gather_kick")
        return mv.value if want_max_v else None

    def drift_rebin(self, dtau):
        self._check(_lib.load().lf2_drift_rebin(self.h, float(dtau)), "drift_rebin")

    def step(self, F, dtau_kick, dtau_drift, rho=None):
        self._check(_lib.load().lf2_step(self.h, F.h, float(dtau_kick), float(dtau_drift),
                                         rho.h if rho is not None else None), "step")

    def set_move_kernel(self, which):
        """Kernel of step()'s kick-drift-rebin pass: 0 automatic, 1 per-brick,
        2 persistent TMA-pipelined."""
        self._check(_lib.load().lf2_set_move_kernel(self.h, int(which)), "set_move_kernel")

    def set_wait_limit(self, cycles=0, stall=False):
        """Limit of the pipelined move's bounded waits in SM cycles (0: the
        default, about 2 s); stall=True makes its consumers wait on a barrier
        nothing completes (tests of the timeout path)."""
        self._check(_lib.load().lf2_set_wait_limit(self.h, int(cycles), 1 if stall else 0),
                    "set_wait_limit")

    def last_max_velocity(self, out=None):
        """max |v| after the last kick.  With a CUDA float64 tensor `out` the
        value is written there in stream order (no wait); otherwise it is
        returned."""
        if out is not None:
            self._check(_lib.load().lf2_last_max_velocity(self.h, _c.c_void_p(out.data_ptr()),
                                                          _lib.PTR_DEVICE), "last_max_velocity")
            return out
        v = _c.c_double()
        self._check(_lib.load().lf2_last_max_velocity(self.h, _c.byref(v), _lib.PTR_HOST),
                    "last_max_velocity")
        return v.value

    def last_move_kernel(self):
        """Kernel of the last step's kick-drift-rebin pass: 1 per-brick,
        2 pipelined, 0 before the first step."""
        w = _c.c_int()
        self._check(_lib.load().lf2_last_move_kernel(self.h, _c.byref(w)), "last_move_kernel")
        return w.value

    def conservation(self):
        m = _c.c_double()
        mom = (_c.c_double * 3)()
        mv = _c.c_double()
        self._check(_lib.load().lf2_conservation(self.h, _c.byref(m), mom, _c.byref(mv)),
                    "conservation")
        return m.value, np.array(list(mom)), mv.value

    def flags(self, clear=False):
        f = _c.c_uint32()
        self._check(_lib.load().lf2_get_flags(self.h, _c.byref(f), 1 if clear else 0), "flags")
        return f.value

    def synchronize(self):
        self._check(_lib.load().lf2_synchronize(self.h), "synchronize")

    # ------------------------------------------------------------- measurement
    def profile(self, on=True):
        self._check(_lib.load().lf2_profile_enable(self.h, 1 if on else 0), "profile_enable")

    def profile_read(self):
        """{phase: (milliseconds, launches)} since the previous read."""
        ms = (_c.c_double * _lib.NPHASE)()
        ln = (_c.c_int64 * _lib.NPHASE)()
        self._check(_lib.load().lf2_profile_read(self.h, ms, ln), "profile_read")
        return {p: (ms[i], ln[i]) for i, p in enumerate(_lib.PHASES)}

    def rebin_stats(self):
        """(full repacks, single-brick relocations, particles that changed brick
        in the last drift)."""
        r, q, m = _c.c_int64(), _c.c_int64(), _c.c_int64()
        self._check(_lib.load().lf2_rebin_stats(self.h, _c.byref(r), _c.byref(q), _c.byref(m)),
                    "rebin_stats")
        return r.value, q.value, m.value

    def kernel_launches(self):
        n = _c.c_int64()
        self._check(_lib.load().lf2_kernel_launches(self.h, _c.byref(n)), "kernel_launches")
        return n.value
