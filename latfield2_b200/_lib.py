"""ctypes binding of liblf2gpu.so (the C ABI in include/lf2gpu.h).

The library is loaded from this package directory.  If it is missing it is
built with nvcc (latfield2_b200/build.py); if that is impossible the import
fails loudly.  There is no CPU fallback: every call runs the CUDA kernels.
"""
import ctypes
import os

from . import build as _build

LF2_OK = 0
LF2_ERR_ARG = -1
LF2_ERR_CUDA = -2
LF2_ERR_STATE = -3
LF2_ERR_NOMEM = -4
LF2_ERR_UNSUPPORTED = -5

DEPOSIT_FP32 = 0        # FP32 atomics with compensated (TwoSum) rounding errors
DEPOSIT_FIXED64 = 1     # int64 fixed point, bit-exact run to run
DEPOSIT_FP32_PLAIN = 2  # FP32 atomics without compensation (the speed reference)
FFT_FORWARD = 1
FFT_BACKWARD = -1
PTR_HOST = 0
PTR_DEVICE = 1

FLAG_NONFINITE = 0x1
FLAG_BAD_CELL = 0x2
FLAG_MASS_RANGE = 0x4
FLAG_REPACK = 0x8
FLAG_CAPACITY = 0x10
FLAG_FIXED_OVERFLOW = 0x20
FLAG_TIMEOUT = 0x40
NOALLOC_MAX_BRICKS = 1363

c_void_p = ctypes.c_void_p
c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_double = ctypes.c_double
P = ctypes.POINTER

# name -> argtypes (restype is always lf2_status / int unless listed below)
SIGNATURES = {
    "lf2_create": [P(c_void_p), c_int, P(c_int), P(c_double), c_int, c_void_p],
    "lf2_destroy": [c_void_p],
    "lf2_last_error": [c_void_p],
    "lf2_set_stream": [c_void_p, c_void_p],
    "lf2_synchronize": [c_void_p],
    "lf2_get_flags": [c_void_p, P(ctypes.c_uint32), c_int],
    "lf2_particles_set": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                          c_void_p, c_int],
    "lf2_particles_set_pos": [c_void_p, c_i64, c_void_p, c_void_p, c_int, c_void_p, c_double,
                              c_void_p],
    "lf2_particles_count": [c_void_p, P(c_i64)],
    "lf2_particles_get": [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int],
    "lf2_particles_get_pos": [c_void_p, c_void_p, c_void_p, c_int, c_void_p],
    "lf2_cell_counts": [c_void_p, c_void_p, c_int],
    "lf2_field_create": [c_void_p, c_int, P(c_void_p)],
    "lf2_field_wrap": [c_void_p, c_int, c_void_p, P(c_void_p)],
    "lf2_field_destroy": [c_void_p, c_void_p],
    "lf2_field_device_ptr": [c_void_p, c_void_p, P(c_void_p)],
    "lf2_field_components": [c_void_p, c_void_p, P(c_int)],
    "lf2_field_zero": [c_void_p, c_void_p],
    "lf2_field_export": [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int],
    "lf2_field_import": [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int],
    "lf2_halo_fill": [c_void_p, c_void_p, c_int, c_int, c_int],
    "lf2_deposit_scalar": [c_void_p, c_void_p],
    "lf2_deposit_vector_cicngp": [c_void_p, c_void_p],
    "lf2_deposit_symtensor_cicngp": [c_void_p, c_void_p],
    "lf2_deposit_vector_cic": [c_void_p, c_void_p],
    "lf2_deposit_vecvec_cic": [c_void_p, c_void_p],
    "lf2_particles_extract_z": [c_void_p, c_int, c_int, c_i64, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p, P(c_i64)],
    "lf2_particles_add": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                          c_int],
    "lf2_slab_record_words": [c_void_p, P(c_int)],
    "lf2_slab_count": [c_void_p, c_int, c_int, c_void_p],
    "lf2_slab_extract": [c_void_p, c_int, c_int, c_i64, c_void_p, c_i64, c_void_p],
    "lf2_slab_insert": [c_void_p, c_i64, c_void_p, c_i64, c_void_p],
    "lf2_checkpoint_save": [c_void_p, ctypes.c_char_p],
    "lf2_checkpoint_load": [c_void_p, ctypes.c_char_p],
    "lf2_kfield_create": [c_void_p, c_int, P(c_void_p)],
    "lf2_kfield_destroy": [c_void_p, c_void_p],
    "lf2_kfield_export": [c_void_p, c_void_p, c_void_p, c_int, c_int],
    "lf2_kfield_import": [c_void_p, c_void_p, c_void_p, c_int, c_int],
    "lf2_fft_forward": [c_void_p, c_void_p, c_void_p],
    "lf2_fft_backward": [c_void_p, c_void_p, c_void_p],
    "lf2_pm_force": [c_void_p, c_void_p, c_void_p, c_void_p, c_double],
    "lf2_gather_kick": [c_void_p, c_void_p, c_double, P(c_double)],
    "lf2_drift_rebin": [c_void_p, c_double],
    "lf2_step": [c_void_p, c_void_p, c_double, c_double, c_void_p],
    "lf2_set_move_kernel": [c_void_p, c_int],
    "lf2_set_wait_limit": [c_void_p, c_i64, c_int],
    "lf2_set_global_mass": [c_void_p, c_double],
    "lf2_last_move_kernel": [c_void_p, P(c_int)],
    "lf2_last_max_velocity": [c_void_p, c_void_p, c_int],
    "lf2_conservation": [c_void_p, P(c_double), P(c_double), P(c_double)],
    "lf2_velocity_reductions": [c_void_p, P(c_double), P(c_double), P(c_double)],
    "lf2_pm_state_pack": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_double, c_void_p,
                          c_void_p],
    "lf2_pm_state_unpack": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                            c_void_p],
    "lf2_pm_brick_start": [c_void_p, c_i64, c_void_p, c_void_p],
    "lf2_pm_grads_unorder": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                             c_void_p, c_void_p, c_void_p, c_void_p],
    "lf2_pm_deposit_bricks": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_double, c_void_p,
                              c_void_p],
    "lf2_pm_step": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_double],
    "lf2_pm_deposit": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_double, c_void_p],
    "lf2_pm_gather": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p],
    "lf2_pm_kick_drift": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                          c_double],
    "lf2_pm_deposit_adjoint": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_double, c_void_p,
                               c_void_p, c_void_p],
    "lf2_pm_gather_adjoint": [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p],
    "lf2_stencil27": [c_void_p, c_void_p, c_void_p, c_void_p],
    "lf2_stencil27_adjoint": [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    "lf2_pm_force4": [c_void_p, c_void_p, c_void_p, c_double],
    "lf2_slab_fft_create": [c_void_p, c_int, c_int, c_int, P(c_void_p)],
    "lf2_slab_fft_destroy": [c_void_p],
    "lf2_slab_fft_planes_r2c": [c_void_p, c_void_p, c_void_p],
    "lf2_slab_fft_planes_c2r": [c_void_p, c_void_p, c_void_p],
    "lf2_slab_fft_lines": [c_void_p, c_void_p, c_int],
    "lf2_slab_green": [c_void_p, c_void_p, c_int, c_double],
    "lf2_pm_gradient": [c_void_p, c_void_p, c_void_p],
    "lf2_pm_force4_adjoint": [c_void_p, c_void_p, c_void_p, c_double],
    "lf2_profile_enable": [c_void_p, c_int],
    "lf2_profile_read": [c_void_p, P(c_double), P(c_i64)],
    "lf2_kernel_launches": [c_void_p, P(c_i64)],
    "lf2_rebin_stats": [c_void_p, P(c_i64), P(c_i64), P(c_i64)],
    "lf2_deposit_scalar_noalloc": [P(c_int), P(c_double), c_int, c_double, c_i64, c_void_p,
                                   c_void_p, c_void_p, c_void_p, c_void_p, P(ctypes.c_uint32)],
}
NPHASE = 5
PHASES = ("move", "insert_repack", "deposit_tile", "deposit_fixup", "other")
RESTYPES = {"lf2_last_error": ctypes.c_char_p}

_LIB = None


def library_path():
    return _build.LIB


def load():
    """Returns the loaded CDLL, building it first when it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB
    if not os.path.exists(path):
        _build.build()
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = RESTYPES.get(name, c_int)
    _LIB = lib
    return lib


class LF2Error(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"lf2 status {status}: {message}")
        self.status = status


def check(ctx, status, what=""):
    if status != LF2_OK:
        msg = load().lf2_last_error(ctx) if ctx else b""
        raise LF2Error(status, (what + ": " if what else "") + (msg or b"").decode())
