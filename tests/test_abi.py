"""CPU checks of the C ABI boundary: the built library loads without a GPU and
exports every function that include/*.h declares; argument validation that
happens before any device work."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(lf2_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("lf2_create", "lf2_particles_set", "lf2_deposit_scalar", "lf2_gather_kick",
                 "lf2_drift_rebin", "lf2_step", "lf2_field_export", "lf2_conservation"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from latfield2_b200 import _lib
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    for name in _lib.SIGNATURES:
        assert name in declared_functions(), f"binding for undeclared {name}"


def test_create_rejects_bad_geometry_without_touching_the_device():
    from latfield2_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    n = (ctypes.c_int * 3)(8, 8, 8)
    bad_box = (ctypes.c_double * 3)(1.0, 2.0, 1.0)  # unequal resolution
    assert lib.lf2_create(ctypes.byref(h), 0, n, bad_box, 0, None) == _lib.LF2_ERR_ARG
    box = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    assert lib.lf2_create(ctypes.byref(h), 0, n, box, 7, None) == _lib.LF2_ERR_ARG
    zero = (ctypes.c_int * 3)(0, 8, 8)
    assert lib.lf2_create(ctypes.byref(h), 0, zero, box, 0, None) == _lib.LF2_ERR_ARG
    big = (ctypes.c_int * 3)(2048, 2048, 2048)
    assert lib.lf2_create(ctypes.byref(h), 0, big, (ctypes.c_double * 3)(1, 1, 1), 0,
                          None) == _lib.LF2_ERR_UNSUPPORTED


def test_null_context_is_an_argument_error():
    from latfield2_b200 import _lib
    lib = _lib.load()
    assert lib.lf2_deposit_scalar(None, None) == _lib.LF2_ERR_ARG
    assert lib.lf2_drift_rebin(None, ctypes.c_double(0.1)) == _lib.LF2_ERR_ARG
    assert lib.lf2_particles_count(None, None) == _lib.LF2_ERR_ARG
    assert lib.lf2_last_error(None) == b"null context"


def test_next_row_entry_points_reject_null_arguments():
    """The full-CIC, migration, checkpoint and PM-operator entry points
    return LF2_ERR_ARG on a null context or handle before any device work."""
    from latfield2_b200 import _lib
    lib = _lib.load()
    E = _lib.LF2_ERR_ARG
    n = ctypes.c_int64()
    assert lib.lf2_deposit_vector_cic(None, None) == E
    assert lib.lf2_deposit_vecvec_cic(None, None) == E
    assert lib.lf2_particles_extract_z(None, 0, 1, 0, None, None, None, None, None,
                                       ctypes.byref(n)) == E
    assert lib.lf2_particles_add(None, 0, None, None, None, None, None, 0) == E
    assert lib.lf2_checkpoint_save(None, b"x") == E
    assert lib.lf2_checkpoint_load(None, b"x") == E
    assert lib.lf2_kfield_create(None, 1, None) == E
    assert lib.lf2_fft_forward(None, None, None) == E
    assert lib.lf2_pm_force(None, None, None, None, 1.0) == E
    assert lib.lf2_pm_force4(None, None, None, 1.0) == E
    assert lib.lf2_pm_force4_adjoint(None, None, None, 1.0) == E
    assert lib.lf2_pm_gradient(None, None, None) == E
    h = ctypes.c_void_p()
    assert lib.lf2_slab_fft_create(None, 16, 4, 4, ctypes.byref(h)) == E
    assert lib.lf2_slab_fft_planes_r2c(None, None, None) == E
    assert lib.lf2_slab_fft_planes_c2r(None, None, None) == E
    assert lib.lf2_slab_fft_lines(None, None, _lib.FFT_FORWARD) == E
    assert lib.lf2_slab_green(None, None, 0, 1.0) == E
    assert lib.lf2_slab_fft_destroy(None) == _lib.LF2_OK


def test_sources_target_sm100a_only():
    from latfield2_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_the_package_never_imports_the_oracle():
    """The product (latfield2_b200/) runs on the CUDA library alone: no
    module imports, loads or calls the oracle, which is test infrastructure."""
    import ast
    root = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "latfield2_b200")
    for path in glob.glob(os.path.join(root, "**", "*.py"), recursive=True):
        with open(path) as f:
            tree = ast.parse(f.read(), path)
        for node in ast.walk(tree):
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            else:
                continue
            assert not any(n.split(".")[0] == "oracle" for n in names), path
        with open(path) as f:
            src = f.read()
        assert "liblf2oracle" not in src and "lf2_ref_driver" not in src, path
