"""Checkpoint file format, host side (no GPU): the PETSc binary Vec layout
(big-endian int32 class id 1211214, int32 length, big-endian doubles) and
the natural interior order [k][j][i][var] that grid::dump writes
(grid.cpp:367-381; the DMDA global vector), checked byte by byte against
numpy."""
import ctypes

import numpy as np
import pytest

from grim_b200 import _lib
from grim_b200 import config as C


EINVAL = -1
ENOTSUP = -5


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_vec_file_bytes(tmp_path):
    rng = np.random.default_rng(0)
    v = rng.standard_normal(37)
    f = tmp_path / "v.bin"
    assert _lib.lib().grim_petsc_vec_write(str(f).encode(), _ptr(v), v.size) == 0
    raw = f.read_bytes()
    assert len(raw) == 8 + 8 * v.size
    assert np.frombuffer(raw[:8], dtype=">i4").tolist() == [1211214, v.size]
    assert np.array_equal(np.frombuffer(raw[8:], dtype=">f8"), v)
    back = np.zeros_like(v)
    assert _lib.lib().grim_petsc_vec_read(str(f).encode(), _ptr(back), v.size) == 0
    assert np.array_equal(back, v)


def test_vec_file_rejects_wrong_class_or_size(tmp_path):
    v = np.arange(5.)
    f = tmp_path / "v.bin"
    assert _lib.lib().grim_petsc_vec_write(str(f).encode(), _ptr(v), 5) == 0
    out = np.zeros(6)
    assert _lib.lib().grim_petsc_vec_read(str(f).encode(), _ptr(out), 6) == EINVAL
    bad = tmp_path / "bad.bin"
    bad.write_bytes(np.array([1, 5], dtype=">i4").tobytes() + v.astype(">f8").tobytes())
    assert _lib.lib().grim_petsc_vec_read(str(bad).encode(), _ptr(out), 5) == EINVAL
    assert _lib.lib().grim_petsc_vec_read(str(tmp_path / "missing").encode(), _ptr(out), 5) == EINVAL


@pytest.mark.parametrize("dim,emhd", [(1, 0), (2, 1), (3, 0)])
def test_natural_order(dim, emhd):
    cfg = C.make_config(N1=6, N2=5, N3=4, dim=dim, conduction=emhd, viscosity=emhd)
    gc = C.to_struct(cfg)
    X1, _, _ = C.cell_centers(cfg)
    dof = C.var_counts(cfg)[0]
    P = np.random.default_rng(1).standard_normal((dof,) + X1.shape)
    nat = np.zeros(dof * cfg["N1"] * cfg["N2"] * cfg["N3"])
    assert _lib.lib().grim_natural_from_prims(ctypes.byref(gc), _ptr(P), _ptr(nat)) == 0
    s3, s2, s1 = C.interior_slices(cfg)
    expect = np.moveaxis(P[:, s3, s2, s1], 0, -1).ravel()  # [k][j][i][var]
    assert np.array_equal(nat, expect)
    Q = np.full_like(P, 7.)
    assert _lib.lib().grim_prims_from_natural(ctypes.byref(gc), _ptr(nat), _ptr(Q)) == 0
    assert np.array_equal(Q[:, s3, s2, s1], P[:, s3, s2, s1])
    ghost = np.ones(Q.shape[1:], bool)
    ghost[s3, s2, s1] = False
    assert np.all(Q[:, ghost] == 7.)


def test_vec_read_rejects_hdf5_restart_files(tmp_path):
    """A restart file of the reference (PETSc's HDF5 viewer, grid.cpp:367-381)
    starts with the HDF5 signature; it is refused with GRIM_ENOTSUP and a
    message saying that HDF5 restart files are not supported."""
    f = tmp_path / "restartFile.h5"
    f.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(8) + np.arange(8.).tobytes())
    out = np.zeros(5)
    assert _lib.lib().grim_petsc_vec_read(str(f).encode(), _ptr(out), 5) == ENOTSUP
    msg = _lib.lib().grim_last_error().decode()
    assert "HDF5" in msg and "not supported" in msg
