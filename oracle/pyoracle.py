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
    L.oracle_io_create.restype = P
    L.oracle_io_create.argtypes = [I, I, I, D, D, D, I, D, D, I, D, I, D, D, D, I, D]
    L.oracle_io_destroy.argtypes = [P]
    L.oracle_io_set_table.argtypes = [P, P, P, P, P, P, I, I]
    L.oracle_io_init_random.argtypes = [P, ctypes.c_uint64, D]
    L.oracle_io_init_random.restype = I
    L.oracle_io_set_inlet.argtypes = [P, I, P, P, P, P]
    L.oracle_io_set_inlet.restype = I
    for f in ("oracle_io_eng", "oracle_io_mom", "oracle_io_substep"):
        getattr(L, f).argtypes = [P, I]
    L.oracle_io_step.argtypes = [P]
    L.oracle_io_get_field.argtypes = [P, I, P]
    L.oracle_io_set_field.argtypes = [P, I, P]
    for f in ("oracle_io_divmax", "oracle_io_divmax_q", "oracle_io_rhohmax"):
        getattr(L, f).restype = D
        getattr(L, f).argtypes = [P]
    L.oracle_io_bulk.restype = D
    L.oracle_io_bulk.argtypes = [P, I]
    L.oracle_io_bad_cells.restype = ctypes.c_int64
    L.oracle_io_bad_cells.argtypes = [P]
    L.oracle_synth_table.argtypes = [I, P, P, P, P, P, P, P]
    for f in ("oracle_tg_cfl", "oracle_io_cfl"):
        getattr(L, f).restype = D
        getattr(L, f).argtypes = [P]
    for f in ("oracle_tg_set_dt", "oracle_io_set_dt"):
        getattr(L, f).argtypes = [P, D]
    L.oracle_io_set_scheme.argtypes = [P, I]
    L.oracle_io_bc_inlet.argtypes = [P, I, P, P, P, P]
    for f in ("oracle_io_bc_outlet_mom", "oracle_io_bc_outlet_eng"):
        getattr(L, f).argtypes = [P, I]
    L.oracle_io_get_plane.argtypes = [P, I, P]
    L.oracle_io_set_plane.argtypes = [P, I, P]
    L.oracle_io_bc_scalars.argtypes = [P, P]
    L.oracle_io_stats.argtypes = [P, P]
    L.oracle_io_set_walls.argtypes = [P, I]
    L.oracle_io_set_walls.restype = I
    L.oracle_io_set_bcx.argtypes = [P, I, I]
    L.oracle_io_set_bcx.restype = I
    L.oracle_io_pois3d.argtypes = [P]
    L.oracle_fftpack_real.argtypes = [I, I, I, P, I]
    L.oracle_fftpack_real.restype = I
    L.oracle_tg_stats.argtypes = [P, P]
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

    def cfl(self):
        return self.L.oracle_tg_cfl(self.h)

    def set_dt(self, dt):
        self.L.oracle_tg_set_dt(self.h, dt)

    def stats(self):
        """PP_MEAN_ZX_FLOW_TG: array (ny, 122)."""
        a = np.empty((self.ny, 122))
        self.L.oracle_tg_stats(self.h, a.ctypes.data)
        return a


def set_threads(n):
    load().oracle_set_threads(n)


def get_threads():
    return load().oracle_get_threads()


IO_FIELDS = {"u": 0, "v": 1, "w": 2, "p": 3, "phi": 4, "rhsphi": 5, "gx": 20, "gy": 21, "gz": 22, "g0x": 23,
             "g0y": 24, "g0z": 25, "h": 26, "t": 27, "rho": 28, "mu": 29, "k": 30, "rhoh": 31, "rho0": 32,
             "mu0": 33, "drho": 34, "ex0x": 35, "ex0y": 36, "ex0z": 37, "rhse0": 38}


def synth_table(n=4096):
    """The synthetic property table (columns H, T, D, M, K, CP, B) of the
    heated IO configuration, from the oracle's restatement."""
    L = load()
    cols = [np.empty(n) for _ in range(7)]
    L.oracle_synth_table(n, *[c.ctypes.data for c in cols])
    return cols


# coupled inflow/outflow ghost planes (i = 0 and i = NCL1_io + 1), each
# (nz, ny + 2); the same ids as the library's CHAPSIM_P_*
IO_PLANES = {n: q for q, n in enumerate((
    "in_u", "in_v", "in_w", "in_gx", "in_gy", "in_gz", "in_p", "in_rho",
    "out_u", "out_v", "out_w", "out_gx", "out_gy", "out_gz", "out_rho", "out_rhoh", "out_h", "out_t", "out_mu",
    "out_k", "conv0_x", "conv0_y", "conv0_z", "conv0_eng"))}
IO_BC_SCALARS = ("u_outlet", "scaling", "balance", "inflow", "outflow", "mass_rate", "u_outlet_eng")


class OracleIO:
    """x-periodic IO channel: SOLVERRK3_ENG_IO + SOLVERRK3_MOM_IO (explicit
    viscous terms, or with visc_scheme=1 the semi-implicit MOMFA_io scheme;
    FISHPACK Poisson), optionally with the energy equation."""

    def __init__(self, nx, ny, nz, lx=8 * math.pi, lz=4 * math.pi / 3, str2=2.0, istr2=1, ren=2800.0, dt=1e-3,
                 flowdrvtp=1, cfgv=0.0, thermal=1, prt=0.71, qw=(1.0, 1.0), gravdir=0, f_a=0.0, table=None,
                 shortcuts=0, visc_scheme=0, isothermal=0):
        self.L = load()
        self.h = self.L.oracle_io_create(nx, ny, nz, lx, lz, str2, istr2, ren, dt, flowdrvtp, cfgv, thermal, prt,
                                         qw[0], qw[1], gravdir, f_a)
        if not self.h:
            raise ValueError("oracle_io_create rejected the configuration")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.sx = nx  # x extent of the arrays (nx + 2 with the coupled section's ghost columns)
        assert self.L.oracle_io_set_scheme(self.h, int(visc_scheme)) == 0
        if thermal:
            if table is None:
                table = synth_table()
            self._table = [np.ascontiguousarray(c, dtype=np.float64) for c in table[:5]]
            assert self.L.oracle_io_set_table(self.h, *[c.ctypes.data for c in self._table], len(self._table[0]),
                                              shortcuts) == 0
        if isothermal:
            assert self.L.oracle_io_set_walls(self.h, int(isothermal)) == 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_io_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.nz, self.ny + 2, self.sx)

    def get(self, name):
        a = np.empty(self.shape)
        assert self.L.oracle_io_get_field(self.h, IO_FIELDS[name], a.ctypes.data) == 0
        return a

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == self.sx * (self.ny + 2) * self.nz
        assert self.L.oracle_io_set_field(self.h, IO_FIELDS[name], a.ctypes.data) == 0

    # ---- coupled inflow/outflow boundary planes
    def get_plane(self, name):
        a = np.empty((self.nz, self.ny + 2))
        assert self.L.oracle_io_get_plane(self.h, IO_PLANES[name], a.ctypes.data) == 0
        return a

    def set_plane(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == self.nz * (self.ny + 2)
        assert self.L.oracle_io_set_plane(self.h, IO_PLANES[name], a.ctypes.data) == 0

    def bc_tinlet_flow(self, tu, tv, tw, tp):
        """BC_TINLET_FLOW + BC_TINLET_THERML from TG fields (nz, ny+2, nx_tg)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (tu, tv, tw, tp)]
        self.L.oracle_io_bc_inlet(self.h, arrs[0].shape[-1], *[a.ctypes.data for a in arrs])

    def bc_coutlet_mom_rk3(self, ns):
        assert self.L.oracle_io_bc_outlet_mom(self.h, ns) == 0

    def bc_coutlet_eneg_rk3(self, ns):
        assert self.L.oracle_io_bc_outlet_eng(self.h, ns) == 0

    def bc_scalars(self):
        a = np.empty(7)
        self.L.oracle_io_bc_scalars(self.h, a.ctypes.data)
        return dict(zip(IO_BC_SCALARS, a.tolist()))

    def init_random(self, seed, amp=0.1):
        assert self.L.oracle_io_init_random(self.h, seed, amp) == 0

    def eng(self, ns):
        assert self.L.oracle_io_eng(self.h, ns) == 0

    def mom(self, ns):
        assert self.L.oracle_io_mom(self.h, ns) == 0

    def substep(self, ns):
        assert self.L.oracle_io_substep(self.h, ns) == 0

    def step(self, n=1):
        for _ in range(n):
            assert self.L.oracle_io_step(self.h) == 0

    def divmax(self):
        return self.L.oracle_io_divmax(self.h)

    def divmax_q(self):
        return self.L.oracle_io_divmax_q(self.h)

    def bulk(self, what=0):
        return self.L.oracle_io_bulk(self.h, what)

    def rhohmax(self):
        return self.L.oracle_io_rhohmax(self.h)

    def bad_cells(self):
        return self.L.oracle_io_bad_cells(self.h)

    def cfl(self):
        return self.L.oracle_io_cfl(self.h)

    def set_bcx(self, inlet, outlet):
        """BCX_io of the Poisson solve: 1 Dirichlet, 2 Neumann, 3 periodic.
        Non-periodic codes make this the coupled inflow / outflow section
        (TGFLOWFLG): arrays with the x ghost columns, (nz, ny + 2, nx + 2);
        set them before the initial field."""
        assert self.L.oracle_io_set_bcx(self.h, int(inlet), int(outlet)) == 0
        self.sx = self.nx + 2 if (inlet, outlet) != (3, 3) else self.nx

    def set_inlet(self, tu, tv, tw, tp):
        """The TG section's u, v, w, p (nz, ny + 2, nx_tg) that BC_TINLET_FLOW
        reads in the coupled substeps that follow (held until replaced)."""
        self._inlet = [np.ascontiguousarray(a, dtype=np.float64) for a in (tu, tv, tw, tp)]
        assert self.L.oracle_io_set_inlet(self.h, self._inlet[0].shape[-1],
                                          *[a.ctypes.data for a in self._inlet]) == 0

    def pois3d(self):
        """FISHPACK_POIS3D_SIMPLE alone: phi from rhsphi."""
        self.L.oracle_io_pois3d(self.h)

    def stats(self):
        """PP_MEAN_ZX_FLOW_Xperiodic_IO: (ny, 360) xz-plane averages."""
        a = np.empty((self.ny, 360))
        self.L.oracle_io_stats(self.h, a.ctypes.data)
        return a

    def set_dt(self, dt):
        self.L.oracle_io_set_dt(self.h, dt)

    def set_scheme(self, visc_scheme):
        assert self.L.oracle_io_set_scheme(self.h, int(visc_scheme)) == 0
