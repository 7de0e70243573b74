"""ctypes wrapper of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product package never
imports it.  Parity of this oracle with the reference is unpinned (the Fortran
reference cannot be built here); it is pinned by the reference's self-checks
and by the independent numpy restatement in tests/golden/.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
FIELDS = {"u": 0, "v": 1, "w": 2, "p": 3, "phi": 4, "rhsphi": 5, "h0u": 6, "h0v": 7, "h0w": 8}
_lib = None


def load(build=True):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB) and build:
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    L = ctypes.CDLL(LIB)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.oracle_tg_create.restype = P
    L.oracle_tg_create.argtypes = [I, I, I, D, D, D, I, D, D, I, D]
    L.oracle_tg_destroy.argtypes = [P]
    L.oracle_tg_field_len.restype = ctypes.c_int64
    L.oracle_tg_field_len.argtypes = [P]
    L.oracle_tg_get_field.argtypes = [P, I, P]
    L.oracle_tg_set_field.argtypes = [P, I, P]
    L.oracle_tg_get_coef.argtypes = [P, I, P]
    L.oracle_tg_volm.restype = D
    L.oracle_tg_volm.argtypes = [P]
    L.oracle_tg_init_random.argtypes = [P, ctypes.c_uint64, D]
    L.oracle_tg_init_poiseuille.argtypes = [P]
    for f in ("oracle_tg_substep", "oracle_tg_divg", "oracle_tg_velo_correction", "oracle_tg_prcalc"):
        getattr(L, f).argtypes = [P, I]
    for f in ("oracle_tg_step", "oracle_tg_pois3d"):
        getattr(L, f).argtypes = [P]
    for f in ("oracle_tg_divmax", "oracle_tg_bulk", "oracle_tg_pois_residual"):
        getattr(L, f).restype = D
        getattr(L, f).argtypes = [P]
    L.oracle_set_threads.argtypes = [I]
    L.oracle_get_threads.restype = I
    _lib = L
    return L


class OracleTG:
    def __init__(self, nx, ny, nz, lx=4 * math.pi, lz=4 * math.pi / 3, str2=2.0, istr2=1, ren=2800.0,
                 dt=1e-3, flowdrvtp=1, cfgv=0.0):
        self.L = load()
        self.h = self.L.oracle_tg_create(nx, ny, nz, lx, lz, str2, istr2, ren, dt, flowdrvtp, cfgv)
        if not self.h:
            raise ValueError("oracle_tg_create rejected the configuration")
        self.nx, self.ny, self.nz = nx, ny, nz

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_tg_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.nz, self.ny + 2, self.nx)

    def get(self, name):
        a = np.empty(self.shape)
        self.L.oracle_tg_get_field(self.h, FIELDS[name], a.ctypes.data)
        return a

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == self.nx * (self.ny + 2) * self.nz
        self.L.oracle_tg_set_field(self.h, FIELDS[name], a.ctypes.data)

    def coef(self, what):
        out = np.empty(self.ny + 2)
        n = self.L.oracle_tg_get_coef(self.h, what, out.ctypes.data)
        return out[:n]

    def init_random(self, seed, amp=0.1):
        self.L.oracle_tg_init_random(self.h, seed, amp)

    def init_poiseuille(self):
        self.L.oracle_tg_init_poiseuille(self.h)

    def substep(self, ns):
        assert self.L.oracle_tg_substep(self.h, ns) == 0

    def step(self, n=1):
        for _ in range(n):
            assert self.L.oracle_tg_step(self.h) == 0

    def divg(self, ns):
        self.L.oracle_tg_divg(self.h, ns)

    def pois3d(self):
        self.L.oracle_tg_pois3d(self.h)

    def velo_correction(self, ns):
        self.L.oracle_tg_velo_correction(self.h, ns)
        self.L.oracle_tg_prcalc(self.h, ns)

    def divmax(self):
        return self.L.oracle_tg_divmax(self.h)

    def bulk(self):
        return self.L.oracle_tg_bulk(self.h)

    def pois_residual(self):
        return self.L.oracle_tg_pois_residual(self.h)


def set_threads(n):
    load().oracle_set_threads(n)


def get_threads():
    return load().oracle_get_threads()
