"""Host-side mirror of the reference's IO-section entry points over libchapsim.

An ``IOChannel`` is the inflow/outflow channel section, run x-periodic
(BCX_io = 3, the default) with the explicit viscous scheme
(``visc_scheme=0``) or the semi-implicit one (``visc_scheme=1``:
VISCOUS_PAR_EXPLT_*_io and MOMFA_io, src/SOLVERRK3_MOM_IO.f90:73-87), or as
the coupled section (``bcx`` Dirichlet / Neumann, e.g. ``(2, 1)``: TGFLOWFLG)
whose inlet a ``TGChannel`` feeds (``set_inlet``) and whose outlet is
convective; its fields carry the x ghost columns, shape (nz, ny + 2, nx + 2).
With thermal on, the energy equation runs with table properties and iso-flux
(or, x-periodic, iso-thermal) walls.  Method names follow
the Fortran subroutines they replace (CHAPSim1WW, paths relative to the
project root):

=========================  ==================================================
``solverrk3_eng_io(ns)``   SOLVERRK3_ENG_IO(NS), src/SOLVERRK3_ENG_IO.f90:1-77
``solverrk3_mom_io(ns)``   DENSITY_TIME_DERIVATION, DENSITY_/MU_Staggered,
                           VELOCITY_CALC_io (ns >= 1), then SOLVERRK3_MOM_IO(NS),
                           src/SOLVE.f90:121-132, src/SOLVERRK3_MOM_IO.f90:1-168
``divg_io(ns)``            DIVG_io(NS), src/DIVG.f90:60-150
``fishpack_pois3d()``      FISHPACK_POIS3D_SIMPLE, src/possion3d_fishpack_reform.f90:431-547
``massflux_update_io(ns)`` MASSFLUX_UPDATE_IO + PRCALC_io,
                           src/VELO_CORRECTION.f90:107-185, src/PRESSURE_CORRECTION.f90:86-122
``divgck_io()``            DIVGCK_io, src/DIVGCK.f90:60-190
``random_fl_theml_fld_io`` RANDOM_FL_THEML_FLD_io + CALC_INITIALIZATION_io,
                           src/INITIAL_FL_THEML_FLD_io.f90:2-172
``step_coupled(tg, n)``    SOLVE's substep loop over both sections,
                           src/SOLVE.f90:119-134
=========================  ==================================================

Every compute call goes to libchapsim.so; there is no CPU fallback.
"""
import ctypes
import math

import numpy as np

from . import _lib
from .solver import FIELD_IDS, ChapsimError, TGChannel, default_config

IO_FIELD_IDS = dict(FIELD_IDS)
IO_FIELD_IDS.update({
    "ex0x": _lib.F_H0U, "ex0y": _lib.F_H0V, "ex0z": _lib.F_H0W,
    "gx": _lib.F_GX, "gy": _lib.F_GY, "gz": _lib.F_GZ, "g0x": _lib.F_G0X, "g0y": _lib.F_G0Y, "g0z": _lib.F_G0Z,
    "h": _lib.F_H, "t": _lib.F_T, "rho": _lib.F_RHO, "mu": _lib.F_MU, "k": _lib.F_K, "rhoh": _lib.F_RHOH,
    "rho0": _lib.F_RHO0, "mu0": _lib.F_MU0, "drho": _lib.F_DRHO, "rhse0": _lib.F_RHSE0,
})


def io_config(**kw):
    io = _lib.ChapsimIOConfig()
    _lib.load().chapsim_io_config_default(ctypes.byref(io))
    for k, v in kw.items():
        if not hasattr(io, k):
            raise KeyError(k)
        setattr(io, k, v)
    return io


class IOChannel(TGChannel):
    """One x-periodic IO channel section resident on a GPU (FP64, or the
    mixed form with FP32 Poisson spectra)."""

    DOMAIN = _lib.IIO
    FIELDS = IO_FIELD_IDS

    def __init__(self, nx=64, ny=64, nz=64, lx=8 * math.pi, lz=4 * math.pi / 3, str2=2.0, istr2=1, ren=2800.0,
                 dt=1e-3, flowdrvtp=1, cfgv=0.0, thermal=1, prt=0.71, qw=(1.0, 1.0), gravdir=0, f_a=0.0,
                 table=None, shortcuts=0, device=0, visc_scheme=0, coupled=0, precision=_lib.FP64, isothermal=0,
                 bcx=(3, 3)):
        self.lib = _lib.load()
        self.cfg = default_config(nx=nx, ny=ny, nz=nz, lx=lx, lz=lz, str2=str2, istr2=istr2, ren=ren, dt=dt,
                                  flowdrvtp=flowdrvtp, cfgv=cfgv, precision=precision, device=device)
        self.iocfg = io_config(thermal=thermal, prt=prt, qw_bot=qw[0], qw_top=qw[1], gravdir=gravdir, f_a=f_a,
                               visc_scheme=visc_scheme, coupled=coupled, isothermal=isothermal,
                               bcx_in=bcx[0], bcx_out=bcx[1])
        h = ctypes.c_void_p()
        rc = self.lib.chapsim_create_io(ctypes.byref(self.cfg), ctypes.byref(self.iocfg), ctypes.byref(h))
        if rc != _lib.CHAPSIM_OK:
            raise ChapsimError(rc, "chapsim_create_io failed")
        self.h = h
        self.nx, self.ny, self.nz = nx, ny, nz
        # x extent of the fields: the coupled section adds the ghost columns IC = 0, NCL1_io + 1
        self.sx = nx if tuple(bcx) == (3, 3) else nx + 2
        self.n = self.lib.chapsim_field_len(self.h)
        self._inlet = None
        if thermal:
            if table is None:
                from .props import synthetic_table
                table = synthetic_table()
            self.set_table(table, shortcuts)

    @property
    def shape(self):
        return (self.nz, self.ny + 2, self.sx)

    def set_table(self, table, shortcuts=0):
        """Columns H, T, D, M, K (extra columns ignored)."""
        cols = [np.ascontiguousarray(c, dtype=np.float64) for c in list(table)[:5]]
        self._chk(self.lib.chapsim_set_table(self.h, *[c.ctypes.data for c in cols], len(cols[0]),
                                             1 if shortcuts else 0))

    def set_props_mode(self, mode, engine=None):
        """Property evaluation of the energy substep: _lib.PROPS_TABLE (table
        splines) or _lib.PROPS_MLP with a trained, gated PropertyEngine on the
        same table (its model is copied into the context)."""
        self._chk(self.lib.chapsim_set_props_mode(self.h, mode, engine.h if engine is not None else None))

    def therm_prop_update(self, mode=0, iregion=0):
        """THERM_PROP_UPDATE(IREGION) on the interior: h -> T, mu, k, rho."""
        self._chk(self.lib.chapsim_therm_prop_update(self.h, iregion, mode))

    # ------------------------------------------------------ reference entries
    def random_fl_theml_fld_io(self, seed=0, amp=0.1, project=True):
        self._chk(self.lib.chapsim_init_random(self.h, seed, amp, 1 if project else 0))

    def solverrk3_eng_io(self, ns):
        self._chk(self.lib.chapsim_rk3_eng_io(self.h, ns))

    def solverrk3_mom_io(self, ns):
        self._chk(self.lib.chapsim_rk3_mom_io(self.h, ns))

    def step(self, nsteps=1):
        """NS = 1, 2, 3 (energy then momentum) for each of nsteps steps (graph-replayed)."""
        self._chk(self.lib.chapsim_step_io(self.h, nsteps))

    # ---- the coupled section (non-periodic bcx)
    def set_inlet(self, tg):
        """The TG section whose fields BC_TINLET_FLOW reads (same device, ny,
        nz); None detaches.  Set it before the initial field."""
        self._chk(self.lib.chapsim_io_set_inlet(self.h, tg.h if tg is not None else None))
        self._inlet = tg

    def step_coupled(self, tg, nsteps=1):
        """nsteps steps of the TG section and this one in SOLVE's order: per
        substep SOLVERRK3_MOM_tg, then SOLVERRK3_ENG_IO and SOLVERRK3_MOM_IO."""
        self._chk(self.lib.chapsim_step_coupled(tg.h, self.h, nsteps))

    def divg_io(self, ns):
        self._chk(self.lib.chapsim_divg(self.h, _lib.IIO, ns))

    def fishpack_pois3d(self):
        self._chk(self.lib.chapsim_pois3d(self.h, _lib.IIO))

    def massflux_update_io(self, ns):
        self._chk(self.lib.chapsim_velo_correction(self.h, _lib.IIO, ns))

    def divgck_io(self):
        return self._reduce(_lib.R_DIVMAX)

    def divgck_q_io(self):
        return self._reduce(_lib.R_DIVMAX_Q)

    def bulk_velocity_io(self):
        return self._reduce(_lib.R_BULK)

    def bulk_massflux_io(self):
        return self._reduce(_lib.R_BULK_G)

    def bulk_h_io(self):
        return self._reduce(_lib.R_BULK_H)

    def model_again_tiles(self):
        """Learned-property tiles whose second enthalpy took a second model
        evaluation (a step beyond the first-order expansion's range)."""
        return int(self._reduce(8))

    # ------------------------------------------------------- statistics
    STATS_LAYOUT = (("U1", 4), ("G1", 3), ("UP", 3), ("U2", 6), ("UG", 6), ("U3", 10), ("UGU", 10), ("DVDL1", 9),
                    ("DVDLP", 9), ("DVDL2", 81), ("T1", 1), ("D1", 1), ("H1", 1), ("M1", 1), ("T2", 1), ("D2", 1),
                    ("H2", 1), ("DH", 1), ("PH", 1), ("DVDL1M", 9), ("DVDL1MH", 9), ("DVDL1MU", 27), ("DVDL2M", 81),
                    ("UH", 3), ("GH", 3), ("U2DH", 6), ("DhDL1", 3), ("DhDLP", 3), ("DTDLK", 3), ("DTDLKU", 9),
                    ("DTDLKDVDL", 27), ("DHDLMDVDL", 27))

    def pp_mean_zx(self, accumulate=False):
        """PP_MEAN_ZX_FLOW_Xperiodic_IO on the device (and PP_MEAN_T_Xperiodic_IO
        when accumulate)."""
        self._chk(self.lib.chapsim_stats(self.h, 1 if accumulate else 0))

    def stats(self, which=0):
        """(ny, 360) array of the xz (which=0) or time (which=1) averages, in
        STATS_LAYOUT order, and the sample count."""
        a = np.empty((self.ny, _lib.STATS_IO_NV))
        n = ctypes.c_int64()
        self._chk(self.lib.chapsim_get_stats(self.h, which, a.ctypes.data, a.size, ctypes.byref(n)))
        return a, n.value

    def stats_groups(self, which=0):
        """The statistics as {name: (ny, width) array} in STATS_LAYOUT order."""
        a, _ = self.stats(which)
        out, lo = {}, 0
        for name, width in self.STATS_LAYOUT:
            out[name] = a[:, lo:lo + width]
            lo += width
        return out

    def monitor(self):
        """The bulk numbers that close PP_MEAN_ZX_FLOW_Xperiodic_IO
        (src/processing/PP_MEAN_ZX.f90:814-869) from the device xz averages:
        G1BULK (bulk x mass flux), G1MAXX, and with the energy equation
        H1bulk (mass-flux-weighted enthalpy) and T1MAXX."""
        g = self.stats_groups(0)
        dyfi = self.mesh(2)
        area = (1.0 / dyfi).sum() * self.cfg.lz  # AREA_INLET of the channel
        g1rate = (g["G1"][:, 0] / dyfi).sum()
        mon = {"g1bulk": g1rate * self.cfg.lz / area, "g1maxx": np.abs(g["G1"][:, 0]).max(),
               "maxdiv": self.divgck_io(), "cflmm_dt": self.cfl() * self.cfg.dt}
        if self.iocfg.thermal:
            mon["h1bulk"] = (g["GH"][:, 0] / dyfi).sum() / g1rate
            mon["t1maxx"] = np.abs(g["T1"][:, 0]).max()
        return mon

    def wall_values(self):
        """(2, 5) array: T, h, rho, mu, k of the bottom and top walls when
        iso-thermal (WALL_ISOTHERMAL_GIVEN), zero for an iso-flux wall."""
        a = np.zeros(10)
        self._chk(self.lib.chapsim_io_wall_values(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 10))
        return a.reshape(2, 5)

    def driven_force(self):
        """PP_DRIVEN_FORCE (src/processing/PP_MEAN_ZX.f90:969-1056) from the
        device xz averages of the last pp_mean_zx: the constant-mass-flux
        driving force FcDrv = (|wall friction 1| + |wall friction 2| -
        buoyancy) / 2 per unit wall area, and FUxzL_IO = FcDrv (U1, 1) per
        row.  Defined for FLOWDRVTP = 1; with the energy equation the wall
        viscosity is M_WAL_GV, which the reference holds for iso-thermal walls
        only (zero on an iso-flux wall beside an iso-thermal one), so a heated
        channel with two iso-flux walls raises ValueError."""
        if self.cfg.flowdrvtp != 1:
            raise ValueError("PP_DRIVEN_FORCE applies to FLOWDRVTP = 1 only")
        mu_w = np.ones(2)
        if self.iocfg.thermal:
            if not self.iocfg.isothermal:
                raise ValueError("M_WAL_GV is undefined with two iso-flux walls (the reference never allocates it)")
            mu_w = self.wall_values()[:, 3]
        g = self.stats_groups(0)
        u1 = g["U1"][:, 0]
        ynd, ycc, dyfi = self.mesh(0), self.mesh(1), self.mesh(2)
        cv = 1.0 / self.cfg.ren
        f1 = mu_w[0] * u1[0] / (ycc[0] - ynd[0]) * cv
        f2 = mu_w[1] * u1[-1] / (ycc[-1] - ynd[-1]) * cv
        buo = 0.0
        if self.iocfg.gravdir == 1:
            buo = float((g["D1"][:, 0] * self.iocfg.f_a / dyfi).sum())
        fc = (abs(f1) + abs(f2) - buo) / 2.0
        fu = np.concatenate([fc * g["U1"][:, :3], np.full((self.ny, 1), fc)], axis=1)
        return fc, fu

    def bad_cells(self):
        return int(self._reduce(_lib.R_BADCELLS))

    # ---- coupled inflow/outflow boundary planes (ghost columns i = 0 and NCL1_io + 1)
    def get_plane(self, name):
        """A ghost plane of the coupled inflow/outflow conditions, (nz, ny+2)."""
        a = np.empty((self.nz, self.ny + 2))
        self._chk(self.lib.chapsim_io_get_plane(self.h, _lib.IO_PLANES[name], a.ctypes.data, a.size))
        return a

    def set_plane(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.size != self.nz * (self.ny + 2):
            raise ValueError(f"plane {name}: expected {self.nz * (self.ny + 2)} values, got {a.size}")
        self._chk(self.lib.chapsim_io_set_plane(self.h, _lib.IO_PLANES[name], a.ctypes.data, a.size))

    def bc_tinlet_flow(self, tg):
        """BC_TINLET_FLOW + BC_TINLET_THERML (src/BC_INLET.f90:2-76) from a TG
        context of the same ny, nz on the same device."""
        self._chk(self.lib.chapsim_io_bc_inlet(self.h, tg.h))

    def bc_coutlet_mom_rk3(self, ns):
        """BC_COUTLET_MOM_RK3(NS) with CHK_MassConsv_io (src/BC_COUTLET_MOM_RK3.f90:2-174)."""
        self._chk(self.lib.chapsim_io_bc_outlet_mom(self.h, ns))

    def bc_coutlet_eneg_rk3(self, ns):
        """BC_COUTLET_ENEG_RK3(NS) (src/BC_COUTLET_ENEG_RK3.f90:2-41)."""
        self._chk(self.lib.chapsim_io_bc_outlet_eng(self.h, ns))

    def bc_scalars(self):
        """U_OUTLET (momentum and energy calls), CHK_Mass_CONSV0_SCALING, the
        balance inflow - mass rate - outflow and its three terms."""
        a = np.empty(7)
        self._chk(self.lib.chapsim_io_bc_scalars(self.h, a.ctypes.data, 7))
        return dict(zip(_lib.IO_BC_SCALARS, a.tolist()))

    # TG-only entries do not apply
    def solverrk3_mom_tg(self, ns):
        raise ChapsimError(4, "not a TG context")
