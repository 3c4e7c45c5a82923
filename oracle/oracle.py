"""Python access to the CPU oracle (liblf2oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
CPU-baseline leg of bench.py, always as the checker of the CUDA path.

Layer (A) restates the reference (particles/projections.hpp,
particles/LATfield2_Particles.hpp, LATfield2_Field_decl.hpp) in its own data
layout; layer (B) restates the device arithmetic of this library.  See
lf2_oracle.h for the per-function citations.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblf2oracle.so")
_LIB = None

_d = ctypes.c_double
_f = ctypes.c_float
_i = ctypes.c_int
_i64 = ctypes.c_int64
_vp = ctypes.c_void_p


def _sources_newer():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t
               for f in ("lf2_oracle.c", "lf2_oracle_ref.inc", "lf2_oracle.h"))


def build():
    if _sources_newer():
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _LIB
    if _LIB is None:
        build()
        _LIB = ctypes.CDLL(LIB_PATH)
        for s in ("d", "f"):
            getattr(_LIB, f"lf2o_update_vel_cic_{s}").restype = _d
        _LIB.lf2o_state_drift.restype = _i64
        _LIB.lf2o_fixed_weight.restype = ctypes.c_uint64
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _n3(n):
    return (_i * 3)(*[int(v) for v in n])


def _real(prec):
    return (np.float64, _d, "d") if prec == "d" else (np.float32, _f, "f")


def gross_shape(n, halo, comps):
    return (n[2] + 2 * halo, n[1] + 2 * halo, n[0] + 2 * halo, comps)


# ------------------------------------------------------------------ layer (A)
def lists_from_insertion(n, cell):
    """CSR lists in reverse insertion order (addParticle_global push_front)."""
    ncells = int(n[0]) * int(n[1]) * int(n[2])
    cell = np.ascontiguousarray(cell, np.int32)
    cs = np.empty(ncells + 1, np.int64)
    order = np.empty(cell.shape[0], np.int64)
    lib().lf2o_lists_from_insertion(_i64(ncells), _i64(cell.shape[0]), _p(cell), _p(cs), _p(order))
    return cs, order


def rebin_lists(n, cs, order, new_cell):
    ncells = int(n[0]) * int(n[1]) * int(n[2])
    new_cell = np.ascontiguousarray(new_cell, np.int32)
    cs2 = np.empty(ncells + 1, np.int64)
    order2 = np.empty(order.shape[0], np.int64)
    lib().lf2o_rebin_lists(_i64(ncells), _i64(order.shape[0]), _p(cs), _p(order), _p(new_cell),
                           _p(cs2), _p(order2))
    return cs2, order2


def projection_init(n, halo, comps, prec="d"):
    dt, _, _ = _real(prec)
    return np.zeros(gross_shape(n, halo, comps), dt)


def scalar_cic(n, halo, res, cs, pos, pmass=None, gmass=0.0, prec="d", comm=True):
    """projection_init + scalarProjectionCIC_project (+ _comm)."""
    dt, ct, s = _real(prec)
    rho = projection_init(n, halo, 1, prec)
    pos = np.ascontiguousarray(pos, dt)
    pm = None if pmass is None else np.ascontiguousarray(pmass, np.float64)
    L = lib()
    getattr(L, f"lf2o_scalar_cic_project_{s}")(_n3(n), _i(halo), ct(res), _p(cs), _p(pos), _p(pm),
                                               _d(gmass), _p(rho))
    if comm:
        getattr(L, f"lf2o_scalar_cic_comm_{s}")(_p(rho), _n3(n), _i(halo))
    return rho


def vector_cicngp(n, halo, res, cs, pos, vel, pmass=None, gmass=0.0, prec="d", comm=True):
    dt, ct, s = _real(prec)
    v = projection_init(n, halo, 3, prec)
    pos = np.ascontiguousarray(pos, dt)
    vel = np.ascontiguousarray(vel, dt)
    pm = None if pmass is None else np.ascontiguousarray(pmass, np.float64)
    L = lib()
    getattr(L, f"lf2o_vector_cicngp_project_{s}")(_n3(n), _i(halo), ct(res), _p(cs), _p(pos),
                                                  _p(vel), _p(pm), _d(gmass), _p(v))
    if comm:
        getattr(L, f"lf2o_vector_cicngp_comm_{s}")(_p(v), _n3(n), _i(halo))
    return v


def symtensor_cicngp(n, halo, res, cs, pos, vel, pmass=None, gmass=0.0, prec="d", comm=True):
    dt, ct, s = _real(prec)
    t = projection_init(n, halo, 6, prec)
    pos = np.ascontiguousarray(pos, dt)
    vel = np.ascontiguousarray(vel, dt)
    pm = None if pmass is None else np.ascontiguousarray(pmass, np.float64)
    L = lib()
    getattr(L, f"lf2o_symtensor_cicngp_project_{s}")(_n3(n), _i(halo), ct(res), _p(cs), _p(pos),
                                                     _p(vel), _p(pm), _d(gmass), _p(t))
    if comm:
        getattr(L, f"lf2o_symtensor_cicngp_comm_{s}")(_p(t), _n3(n), _i(halo))
    return t


def _full_cic(name, comps, n, halo, res, cs, pos, vel, pmass, gmass, prec, comm):
    dt, ct, s = _real(prec)
    f = projection_init(n, halo, comps, prec)
    pos = np.ascontiguousarray(pos, dt)
    vel = np.ascontiguousarray(vel, dt)
    pm = None if pmass is None else np.ascontiguousarray(pmass, np.float64)
    L = lib()
    getattr(L, f"lf2o_{name}_project_{s}")(_n3(n), _i(halo), ct(res), _p(cs), _p(pos), _p(vel),
                                           _p(pm), _d(gmass), _p(f))
    if comm:
        getattr(L, f"lf2o_{name}_comm_{s}")(_p(f), _n3(n), _i(halo))
    return f


def vector_cic(n, halo, res, cs, pos, vel, pmass=None, gmass=0.0, prec="d", comm=True):
    """projection_init + vectorProjectionCIC_project (+ _comm): m v / res^3 on
    the links, staggered CIC along each component's own dim."""
    return _full_cic("vector_cic", 3, n, halo, res, cs, pos, vel, pmass, gmass, prec, comm)


def vecvec_cic(n, halo, res, cs, pos, vel, pmass=None, gmass=0.0, prec="d", comm=True):
    """projection_init + VecVecProjectionCIC_project (+ _comm): symmetric
    m v_i v_j / res^3, components 00,01,02,11,12,22."""
    return _full_cic("vecvec_cic", 6, n, halo, res, cs, pos, vel, pmass, gmass, prec, comm)


def update_halo(f, n, halo, prec="d"):
    """Field::updateHalo on a reference-layout array (in place)."""
    _, _, s = _real(prec)
    getattr(lib(), f"lf2o_update_halo_{s}")(_p(f), _n3(n), _i(halo), _i(f.shape[-1]))
    return f


def update_vel_cic(n, halo, cs, pos, vel, F, dtau, prec="d"):
    """updateVel with the CIC gather-kick; vel updated in place.  Returns
    (max |v|, sum |v|^2)."""
    _, _, s = _real(prec)
    sv = _d()
    mv = getattr(lib(), f"lf2o_update_vel_cic_{s}")(_n3(n), _i(halo), _p(cs), _p(pos), _p(vel),
                                                    _p(F), _d(dtau), ctypes.byref(sv))
    return mv, sv.value


def move_simple(n, box, pos, vel, dtau, prec="d"):
    """Drift + wrap + new cell (pos updated in place).  Returns new cells."""
    _, ct, s = _real(prec)
    cell = np.empty(pos.shape[0], np.int32)
    getattr(lib(), f"lf2o_move_simple_{s}")(_n3(n), ct(box), _i64(pos.shape[0]), _p(pos), _p(vel),
                                            _d(dtau), _p(cell))
    return cell


# ------------------------------------------------------------------ layer (B)
def state_kick(n, cell, off, vel, F, dtk):
    """F: internal layout (3, n2, n1, n0) float32.  Returns the new velocities."""
    cell = np.ascontiguousarray(cell, np.int32)
    off = np.ascontiguousarray(off, np.float32)
    v = np.array(vel, np.float32, copy=True, order="C")
    F = np.ascontiguousarray(F, np.float32)
    lib().lf2o_state_kick(_n3(n), _i64(cell.shape[0]), _p(cell), _p(off), _p(v), _p(F), _f(dtk))
    return v


def state_drift(n, cell, off, vel, dtn):
    c = np.array(cell, np.int32, copy=True, order="C")
    o = np.array(off, np.float32, copy=True, order="C")
    vel = np.ascontiguousarray(vel, np.float32)
    bad = lib().lf2o_state_drift(_n3(n), _i64(c.shape[0]), _p(c), _p(o), _p(vel), _f(dtn))
    return c, o, bad


def state_deposit_fixed(n, cell, off, mrel=None):
    cell = np.ascontiguousarray(cell, np.int32)
    off = np.ascontiguousarray(off, np.float32)
    mr = None if mrel is None else np.ascontiguousarray(mrel, np.float32)
    acc = np.zeros(int(n[0]) * int(n[1]) * int(n[2]), np.int64)
    lib().lf2o_state_deposit_fixed(_n3(n), _i64(cell.shape[0]), _p(cell), _p(off), _p(mr), _p(acc))
    return acc


def vexp(vel):
    """Exponent e of the fixed-point velocity unit V = 2^e of a deposit."""
    v = np.ascontiguousarray(vel, np.float32)
    return int(lib().lf2o_vexp(_i64(v.shape[0]), _p(v)))


def state_deposit_fixed_kind(kind, n, cell, off, vel, mrel=None, e=None):
    """Fixed-point momentum (kinds 1, 3) or stress (2, 4) deposit: int64
    accumulator (comps, n2, n1, n0) and the exponent of V used."""
    cell = np.ascontiguousarray(cell, np.int32)
    off = np.ascontiguousarray(off, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    mr = None if mrel is None else np.ascontiguousarray(mrel, np.float32)
    if e is None:
        e = vexp(vel)
    comps = 3 if kind in (1, 3) else 6
    acc = np.zeros(comps * int(n[0]) * int(n[1]) * int(n[2]), np.int64)
    lib().lf2o_state_deposit_fixed_kind(_i(kind), _n3(n), _i64(cell.shape[0]), _p(cell), _p(off),
                                        _p(vel), _p(mr), _i(e), _p(acc))
    return acc.reshape(comps, int(n[2]), int(n[1]), int(n[0])), e


def fixed_kind_to_f32(acc, kind, e, gmass, res):
    """Converts a momentum / stress accumulator as the device does:
    (float)q * (2^-32 m_unit / res^3 as FP32) * 2^-16 V^p, the accumulator
    being in units of 2^-48 of a unit mass times V^p (an exact power of 2)."""
    p = 1 if kind in (1, 3) else 2
    scale = np.float32(2.0 ** -32 * gmass / (res * res * res))
    scale = np.float32(np.ldexp(scale, p * e - 16))
    return (acc.astype(np.float32) * scale).astype(np.float32)


def fixed_to_f32(acc, scale):
    out = np.empty(acc.shape[0], np.float32)
    lib().lf2o_state_fixed_to_f32(_i64(acc.shape[0]), _p(acc), _f(scale), _p(out))
    return out


def state_deposit_f64(n, cell, off, res, mass=None, gmass=0.0):
    cell = np.ascontiguousarray(cell, np.int32)
    off = np.ascontiguousarray(off, np.float32)
    m = None if mass is None else np.ascontiguousarray(mass, np.float32)
    rho = np.zeros(int(n[0]) * int(n[1]) * int(n[2]), np.float64)
    lib().lf2o_state_deposit_f64(_n3(n), _i64(cell.shape[0]), _p(cell), _p(off), _p(m), _d(gmass),
                                 _d(res), _p(rho))
    return rho


def fixed_weight(fx, fy, fz, bx, by, bz):
    return lib().lf2o_fixed_weight(_f(fx), _f(fy), _f(fz), _i(bx), _i(by), _i(bz))


# ---------------------------------------------------------------- conversions
def interior(f, n, halo):
    """Reference layout (z, y, x, c) with halo -> internal (c, z, y, x)."""
    h = halo
    return np.ascontiguousarray(f[h:h + n[2], h:h + n[1], h:h + n[0], :].transpose(3, 0, 1, 2))


def state_to_pos(n, res, cell, off, dtype=np.float64):
    n0, n1 = int(n[0]), int(n[1])
    c = np.asarray(cell, np.int64)
    xyz = np.stack([c % n0, (c // n0) % n1, c // (n0 * n1)], axis=1).astype(np.float64)
    return ((xyz + np.asarray(off, np.float64)) * res).astype(dtype)
