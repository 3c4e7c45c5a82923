"""The binary field file of the reference (Field::write / Field::read,
LATfield2_Field_decl.hpp:1179-1345; Field::saveHDF5 of a build without HDF5
writes it as filename + "BIN"): pinned against the reference itself, whose
Field::write runs here in oracle/_ref's driver on a 2x2 process grid, and
produced identically by the C++ layer (tests/compat/field_io_demo.cpp) and
by latfield2_b200.snapshot.write_field_binary."""
import os
import subprocess
import sys

import numpy as np
import pytest

from latfield2_b200 import snapshot as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "lf2_ref_driver_double")


class _Field:
    """export / import_ of a FieldHandle over a host array (c, z, y, x)."""

    class _Ctx:
        def __init__(self, n):
            self.n = n

    def __init__(self, values):
        self.values = values
        self.comps = values.shape[0]
        self.ctx = self._Ctx((values.shape[3], values.shape[2], values.shape[1]))

    def export(self, halo=0, dtype=np.float32):
        return np.ascontiguousarray(self.values.transpose(1, 2, 3, 0)).astype(dtype)

    def import_(self, arr, halo=0):
        self.values = np.ascontiguousarray(np.asarray(arr).transpose(3, 0, 1, 2))


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref is not built")
def test_reference_field_write_is_the_interior_array(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as G
    n, grid = 8, (2, 2)
    ids, pos, vel, F = G.make_inputs(n, 600, False, 0.01, 5)
    inp = str(tmp_path / "in.bin")
    G.write_input(inp, n, 1, grid, 1.0 / 600, G.OP_VECTOR, 0.0, 0.0, ids, pos, vel, F)
    out = str(tmp_path / "field.bin")
    env = dict(os.environ, LF2_MINIMPI_NP="4", LF2_REF_FIELD_WRITE=out)
    subprocess.run([DRIVER, inp, str(tmp_path / "out")], env=env, check=True, timeout=120,
                   stdin=subprocess.DEVNULL, stdout=subprocess.DEVNULL)
    ranks = [G.read_rank(str(tmp_path / f"out.{r}"), n, G.OP_VECTOR, None) for r in range(4)]
    B = G.assemble(ranks, n, G.OP_VECTOR, 3)  # [z][y][x][c], the ranks' own values
    got = np.fromfile(out, dtype=np.float64)
    assert got.size == n ** 3 * 3
    np.testing.assert_array_equal(got.reshape(n, n, n, 3), B)
    # the library's writer gives the same bytes for the same values
    mine = str(tmp_path / "mine.bin")
    S.write_field_binary(mine, _Field(np.ascontiguousarray(B.transpose(3, 0, 1, 2))))
    with open(out, "rb") as a, open(mine, "rb") as b:
        assert a.read() == b.read()
    f = _Field(np.zeros((3, n, n, n)))
    S.read_field_binary(out, f)
    np.testing.assert_array_equal(f.values, B.transpose(3, 0, 1, 2))


def test_cpp_layer_writes_and_reads_the_reference_file(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "tests", "compat"))
    import build_demo
    exe = build_demo.build(str(tmp_path / "field_io_demo"), source="field_io_demo.cpp")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
    a = np.fromfile(tmp_path / "field.bin", dtype=np.float64).reshape(4, 5, 6, 3)
    z, y, x = np.meshgrid(np.arange(4), np.arange(5), np.arange(6), indexing="ij")
    for c in range(3):
        np.testing.assert_array_equal(a[..., c], x + 10 * y + 100 * z + c / 4)
    with open(tmp_path / "field.bin", "rb") as f1, open(tmp_path / "outBIN", "rb") as f2:
        assert f1.read() == f2.read()
