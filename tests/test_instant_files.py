"""Instantaneous-field files in the reference's layout (no GPU): the file
name, the 40-byte header and the Fortran-order interior, checked against an
independent numpy reading/writing of the same layout."""
import ctypes
import os

import numpy as np
import pytest

from chapsim1ww_b200 import _lib


def lib():
    return _lib.load()


def test_file_name_matches_fortran_es15_9():
    buf = ctypes.create_string_buffer(512)
    assert lib().chapsim_instant_file_name(buf, 512, b"run/", 2655.004202, b"U", 0) == 0
    assert buf.value == b"run/DNS_perixz_INSTANT_T2.655004202E+03_U.D"
    assert lib().chapsim_instant_file_name(buf, 512, b"", 0.0, b"E", 0) == 0
    assert buf.value == b"DNS_perixz_INSTANT_T0.000000000E+00_E.D"


def test_file_name_of_io_beside_tg_section():
    """An IO section that runs beside a TG section names its files
    DNS_perioz_... (src/processing/WRT_VARS_IO.f90:24-28), so a TG + IO run
    writing both sections into one directory overwrites nothing."""
    buf = ctypes.create_string_buffer(512)
    assert lib().chapsim_instant_file_name(buf, 512, b"run/", 0.5, b"U", 1) == 0
    assert buf.value == b"run/DNS_perioz_INSTANT_T5.000000000E-01_U.D"


def test_write_layout_and_round_trip(tmp_path):
    nx, ny, nz = 6, 5, 4
    rng = np.random.default_rng(0)
    field = rng.standard_normal((nz, ny + 2, nx))  # F(1:nx, 0:ny+1, 1:nz)
    path = str(tmp_path / "f.D").encode()
    assert lib().chapsim_instant_file_write(path, nx, ny, nz, 17, 1.25, 2800.0, 1e-3, field.ctypes.data) == 0
    raw = open(path, "rb").read()
    assert len(raw) == 16 + 24 + 8 * nx * ny * nz
    assert np.frombuffer(raw[:16], dtype=np.int32).tolist() == [nx, ny, nz, 17]
    assert np.frombuffer(raw[16:40], dtype=np.float64).tolist() == [1.25, 2800.0, 1e-3]
    body = np.frombuffer(raw[40:], dtype=np.float64).reshape((nz, ny, nx))  # Fortran order (i fastest)
    assert np.array_equal(body, field[:, 1:ny + 1, :])
    back = np.full_like(field, -7.0)
    it, tm, re, dt = ctypes.c_int(), ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    assert lib().chapsim_instant_file_read(path, nx, ny, nz, ctypes.byref(it), ctypes.byref(tm), ctypes.byref(re),
                                           ctypes.byref(dt), back.ctypes.data) == 0
    assert (it.value, tm.value, re.value, dt.value) == (17, 1.25, 2800.0, 1e-3)
    assert np.array_equal(back[:, 1:ny + 1, :], field[:, 1:ny + 1, :])
    assert np.all(back[:, 0, :] == -7.0) and np.all(back[:, ny + 1, :] == -7.0)


def test_numpy_written_file_is_read_and_mesh_mismatch_refused(tmp_path):
    nx, ny, nz = 4, 3, 2
    body = np.arange(nx * ny * nz, dtype=np.float64).reshape((nz, ny, nx))
    p = tmp_path / "g.D"
    with open(p, "wb") as f:
        f.write(np.array([nx, ny, nz, 5], dtype=np.int32).tobytes())
        f.write(np.array([0.5, 100.0, 2e-3], dtype=np.float64).tobytes())
        f.write(body.tobytes())
    out = np.zeros((nz, ny + 2, nx))
    it = ctypes.c_int()
    assert lib().chapsim_instant_file_read(str(p).encode(), nx, ny, nz, ctypes.byref(it), None, None, None,
                                           out.ctypes.data) == 0
    assert it.value == 5 and np.array_equal(out[:, 1:ny + 1, :], body)
    assert lib().chapsim_instant_file_read(str(p).encode(), nx + 2, ny, nz, None, None, None, None,
                                           np.zeros((nz, ny + 2, nx + 2)).ctypes.data) != 0
    assert lib().chapsim_instant_file_read(str(tmp_path / "missing.D").encode(), nx, ny, nz, None, None, None, None,
                                           out.ctypes.data) != 0
