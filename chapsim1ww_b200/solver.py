"""Host-side mirror of the reference's TG-channel entry points over libchapsim.

Method names follow the Fortran subroutines they replace (CHAPSim1WW,
paths relative to the project root):

=========================  ==================================================
``solverrk3_mom_tg(ns)``   SOLVERRK3_MOM_tg(NS), src/SOLVERRK3_MOM_tg.f90:18-61
``divg_tg(ns)``            DIVG_tg(NS), src/DIVG.f90:21-57
``fft99_pois3d()``         FFT99_POIS3D_periodicxz(ITG), src/possion3d_FFT99.f90:254-488
``veloupdt_tg(ns)``        VELOUPDT_tg + PRCALC_tg with wall BCs,
                           src/VELO_CORRECTION.f90:19-105, src/PRESSURE_CORRECTION.f90:1-24
``divgck_tg()``            DIVGCK_tg, src/DIVGCK.f90:16-58
``bulk_velocity_tg()``     BULK_VELOCITY_TG, src/INITIAL_FL_FLD_TG.f90:122-149
``random_fl_fld_tg()``     RANDOM_FL_FLD_TG + CALC_INITIALIZATION_tg,
                           src/INITIAL_FL_FLD_TG.f90:2-119
=========================  ==================================================

Fields are numpy views of the Fortran layout F(1:nx, 0:ny+1, 1:nz): arrays of
shape (nz, ny+2, nx) in C order, so ``a[k-1, j, i-1]`` is F(i, j, k).
Errors raise ``ChapsimError`` (the reference prints and STOPs in ERRHDL).
"""
import ctypes
import math

import numpy as np

from . import _lib

FIELD_IDS = {"u": _lib.F_U, "v": _lib.F_V, "w": _lib.F_W, "p": _lib.F_P, "phi": _lib.F_PHI,
             "rhsphi": _lib.F_RHSPHI, "h0u": _lib.F_H0U, "h0v": _lib.F_H0V, "h0w": _lib.F_H0W}


class ChapsimError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_lib.ERRORS.get(code, code)}: {msg}")
        self.code = code


def default_config(**kw):
    cfg = _lib.ChapsimConfig()
    _lib.load().chapsim_config_default(ctypes.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


class TGChannel:
    """One TG (periodic) channel domain resident on a GPU."""

    DOMAIN = _lib.ITG
    FIELDS = FIELD_IDS

    def __init__(self, nx=64, ny=64, nz=64, lx=4 * math.pi, lz=4 * math.pi / 3, str2=2.0, istr2=1,
                 ren=2800.0, dt=1e-3, flowdrvtp=1, cfgv=0.0, precision=_lib.FP64, device=0):
        self.lib = _lib.load()
        self.cfg = default_config(nx=nx, ny=ny, nz=nz, lx=lx, lz=lz, str2=str2, istr2=istr2, ren=ren, dt=dt,
                                  flowdrvtp=flowdrvtp, cfgv=cfgv, precision=precision, device=device)
        h = ctypes.c_void_p()
        rc = self.lib.chapsim_create(ctypes.byref(self.cfg), ctypes.byref(h))
        if rc != _lib.CHAPSIM_OK:
            raise ChapsimError(rc, "chapsim_create failed")
        self.h = h
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = self.lib.chapsim_field_len(self.h)

    # ---------------------------------------------------------------- basics
    def _chk(self, rc):
        if rc != _lib.CHAPSIM_OK:
            raise ChapsimError(rc, self.lib.chapsim_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.chapsim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.nz, self.ny + 2, self.nx)

    def set_field(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.size != self.n:
            raise ValueError(f"field {name}: expected {self.n} values, got {a.size}")
        self._chk(self.lib.chapsim_set_field(self.h, self.DOMAIN, self.FIELDS[name], a.ctypes.data, self.n))

    def get_field(self, name, out=None):
        a = np.empty(self.shape, dtype=np.float64) if out is None else out
        self._chk(self.lib.chapsim_get_field(self.h, self.DOMAIN, self.FIELDS[name], a.ctypes.data, self.n))
        return a

    def set_field_async(self, name, arr):
        """Stream-ordered upload: arr (C-contiguous float64, page-locked for
        overlap) must stay alive until sync()."""
        if not (isinstance(arr, np.ndarray) and arr.dtype == np.float64 and arr.flags.c_contiguous):
            raise ValueError("set_field_async needs a C-contiguous float64 array")
        if arr.size != self.n:
            raise ValueError(f"field {name}: expected {self.n} values, got {arr.size}")
        self._chk(self.lib.chapsim_set_field_async(self.h, self.DOMAIN, self.FIELDS[name], arr.ctypes.data, self.n))

    def get_field_async(self, name, out):
        """Stream-ordered download into out (complete after sync())."""
        if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                and out.size == self.n):
            raise ValueError("get_field_async needs a C-contiguous float64 array of the field's size")
        self._chk(self.lib.chapsim_get_field_async(self.h, self.DOMAIN, self.FIELDS[name], out.ctypes.data, self.n))
        return out

    def set_field_device(self, name, ptr):
        self._chk(self.lib.chapsim_set_field_device(self.h, self.DOMAIN, self.FIELDS[name], ptr, self.n))

    def get_field_device(self, name, ptr):
        self._chk(self.lib.chapsim_get_field_device(self.h, self.DOMAIN, self.FIELDS[name], ptr, self.n))

    def mesh(self, what):
        n = self.ny + 1 if what in (0, 3) else self.ny
        out = np.empty(n)
        self._chk(self.lib.chapsim_get_mesh(self.h, what, out.ctypes.data, n))
        return out

    def sync(self):
        self._chk(self.lib.chapsim_sync(self.h))

    def set_refinement(self, sweeps):
        """Refinement sweeps (0 or 1) of the mixed form's Poisson solve."""
        self._chk(self.lib.chapsim_set_refinement(self.h, sweeps))

    def stream(self):
        s = ctypes.c_void_p()
        self._chk(self.lib.chapsim_get_stream(self.h, ctypes.byref(s)))
        return s.value

    # ------------------------------------------------------ reference entries
    def random_fl_fld_tg(self, seed=0, amp=0.1, project=True):
        self._chk(self.lib.chapsim_init_random(self.h, seed, amp, 1 if project else 0))

    def solverrk3_mom_tg(self, ns):
        self._chk(self.lib.chapsim_rk3_mom_tg(self.h, ns))

    def step(self, nsteps=1):
        """NS = 1, 2, 3 for each of nsteps time steps (graph-replayed)."""
        self._chk(self.lib.chapsim_step_tg(self.h, nsteps))

    def divg_tg(self, ns):
        self._chk(self.lib.chapsim_divg(self.h, _lib.ITG, ns))

    def fft99_pois3d(self):
        self._chk(self.lib.chapsim_pois3d(self.h, _lib.ITG))

    def veloupdt_tg(self, ns):
        self._chk(self.lib.chapsim_velo_correction(self.h, _lib.ITG, ns))

    def _reduce(self, what):
        v = ctypes.c_double()
        self._chk(self.lib.chapsim_reduce(self.h, self.DOMAIN, what, ctypes.byref(v)))
        return v.value

    def divgck_tg(self):
        return self._reduce(_lib.R_DIVMAX)

    def bulk_velocity_tg(self):
        return self._reduce(_lib.R_BULK)

    def nan_count(self):
        return int(self._reduce(_lib.R_NANCOUNT))

    def cfl(self):
        """CFLMM: CFL_tg (CFL_io + CFL_VISCOUS on an IO context), src/CFL.f90."""
        return self._reduce(_lib.R_CFL)

    def set_dt(self, dt):
        """Change DT; the dt-dependent coefficient tables are rebuilt."""
        self._chk(self.lib.chapsim_set_dt(self.h, dt))

    # ------------------------------------------------------- instant files
    def write_instant(self, directory, iteration, time):
        """WRT_INSTANT_VARS_* into directory (a path prefix ending in '/')."""
        self._chk(self.lib.chapsim_write_instant(self.h, directory.encode(), iteration, time))

    def read_instant(self, directory, time):
        """RESTART_INSTANT_VARS_* from directory; returns (iteration, time)."""
        it, tm = ctypes.c_int(), ctypes.c_double()
        self._chk(self.lib.chapsim_read_instant(self.h, directory.encode(), time, ctypes.byref(it), ctypes.byref(tm)))
        return it.value, tm.value

    # ------------------------------------------------------- statistics
    STATS_LAYOUT = (("U1", 4), ("UP", 3), ("U2", 6), ("U3", 10), ("DVDL1", 9), ("DVDLP", 9), ("DVDL2", 81))

    def pp_mean_zx(self, accumulate=False):
        """PP_MEAN_ZX_FLOW_TG on the device (and PP_MEAN_T_TG when accumulate)."""
        self._chk(self.lib.chapsim_stats(self.h, 1 if accumulate else 0))

    def stats(self, which=0):
        """(ny, 122) array of the xz (which=0) or time (which=1) averages and the sample count."""
        a = np.empty((self.ny, _lib.STATS_NV))
        n = ctypes.c_int64()
        self._chk(self.lib.chapsim_get_stats(self.h, which, a.ctypes.data, a.size, ctypes.byref(n)))
        return a, n.value

    def stats_reset(self):
        self._chk(self.lib.chapsim_stats_reset(self.h))

    def monitor(self):
        """The numbers of the PP_MONITOR_TG line (src/processing/PP_SCN_MONITOR.f90:138-242)
        from the device statistics: U1 at the channel centre (xz, xzt), the normal
        stresses and uv there, the skin friction on both walls, bulk and max of U1."""
        xz, _ = self.stats(0)
        xzt, _ = self.stats(1)
        dyfi = self.mesh(2)
        ren = self.cfg.ren
        jc = self.ny // 2 - 1
        mon = {"cflmm_dt": self.cfl() * self.cfg.dt, "dt": self.cfg.dt, "maxdiv": self.divgck_tg()}
        for tag, s in (("xz", xz), ("xzt", xzt)):
            mon[f"u_{tag}"], mon[f"v_{tag}"], mon[f"w_{tag}"] = s[jc, 0], s[jc, 1], s[jc, 2]
            mon[f"uu_{tag}"] = s[jc, 7] - s[jc, 0] * s[jc, 0]
            mon[f"uv_{tag}"] = s[jc, 8] - s[jc, 0] * s[jc, 1]
            mon[f"vv_{tag}"] = s[jc, 10] - s[jc, 1] * s[jc, 1]
            mon[f"ww_{tag}"] = s[jc, 12] - s[jc, 2] * s[jc, 2]
            mon[f"cf_bottom_{tag}"] = s[0, 0] * dyfi[0] * 2.0 * 2.0 / ren
            mon[f"cf_top_{tag}"] = s[-1, 0] * dyfi[-1] * 2.0 * 2.0 / ren
        lz = self.cfg.lz
        area = (1.0 / dyfi).sum() * lz
        mon["u1mean"] = (xz[:, 0] / dyfi).sum() * lz / area
        mon["u1maxx"] = np.abs(xz[:, 0]).max()
        return mon

    # ------------------------------------------------------------- timing
    def phase_timing(self, enable):
        self._chk(self.lib.chapsim_phase_timing(self.h, 1 if enable else 0))

    def phase_times(self):
        ms = (ctypes.c_double * len(_lib.PHASES))()
        n = ctypes.c_int64()
        self._chk(self.lib.chapsim_phase_times(self.h, ms, len(_lib.PHASES), ctypes.byref(n)))
        return dict(zip(_lib.PHASES, list(ms))), n.value

    def phase_reset(self):
        self._chk(self.lib.chapsim_phase_reset(self.h))

    def set_tuning(self, rhs_nzc=16, fft_lb=0):
        self._chk(self.lib.chapsim_set_tuning(self.h, rhs_nzc, fft_lb))

    def set_line_tuning(self, ysolve_bx=128):
        self._chk(self.lib.chapsim_set_line_tuning(self.h, ysolve_bx))

    def get_line_tuning(self):
        a = ctypes.c_int()
        self._chk(self.lib.chapsim_get_line_tuning(self.h, ctypes.byref(a)))
        return a.value

    def get_tuning(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        self._chk(self.lib.chapsim_get_tuning(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def launch_count(self):
        n = ctypes.c_int64()
        self._chk(self.lib.chapsim_launch_count(self.h, ctypes.byref(n)))
        return n.value
