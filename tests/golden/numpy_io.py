"""Independent numpy restatement of CHAPSim's IO-section RK3 substep.

Test infrastructure only: a second implementation of the x-periodic IO
section, written to cross-check the C++ oracle.  It differs from the oracle
in every non-trivial step: the stencils are whole-array shifts, the FISHPACK
Poisson solve (real RFFTF/RFFTB transforms and a TRID0 sweep per mode in the
reference) is done with complex numpy FFTs in x and z and scipy's banded LU
per (kx, kz) mode, the semi-implicit scheme's MOMFA_io factors (TDMAIJI_CYC
and TDMAIJJ_nonCYC in the reference) by batched dense LU, the table splines
are built and evaluated with numpy (searchsorted), and the synthetic
property table is integrated with numpy.

Arrays are numpy views of the Fortran layout F(1:nx, 0:ny+1, 1:nz): shape
(nz, ny+2, nx), so a[k-1, j, i-1] is F(i, j, k).

Reference files restated (paths relative to the CHAPSim1WW project root):
src/SOLVERRK3_ENG_IO.f90:1-77, src/RHS_ENERGY_EXPLICIT.f90:1-150,
src/THERM_PROP_UPDATE.f90:2-291, src/Flow_State.f90:963-990,1015-1070,
1693-1787, src/BC_WALL.f90:522-627, src/MASSFLUX_CALC_IO.f90:1-311,
src/SOLVERRK3_MOM_IO.f90:1-168, src/CONVECTION_X.f90:77-176,
src/CONVECTION_Y.f90:125-230, src/CONVECTION_Z.f90:113-200,
src/DIVG.f90:58-259, src/VISCOUS_X_EXPLICIT_io.f90:1-112,
src/VISCOUS_Y_EXPLICIT_io.f90 and src/VISCOUS_Z_EXPLICIT_io.f90 (channel
branches), src/RHS_MOM_EXPLICIT_io.f90:1-297,
src/possion3d_fishpack_reform.f90:29-547, src/PRESSURE_CORRECTION.f90:86-122,
src/VELO_CORRECTION.f90:107-185, src/INITIAL_FL_THEML_FLD_io.f90:133-172,
352-381,481-560,653-682; the semi-implicit scheme (visthemflg = 1):
src/VISCOUS_X_EXPLICIT_io.f90:124-286, src/VISCOUS_Y_EXPLICIT_io.f90:264-424,
src/VISCOUS_Z_EXPLICIT_io.f90:289-460, src/RHS_MOM_EXPLICIT_io.f90:79-95,
src/MOMFA_io.f90:17-377, src/TDMA_COEF.f90:77-116,
src/MASSFLUX_CALC_IO.f90:316-399, src/PRESSURE_CORRECTION.f90:100-110.

The decisions shared with the oracle and the library: the Poisson mean mode
takes phi(ny) = 0; the reference-state shortcuts of the table look-ups are
off; the initial thermal state is the table at h = 0; the initial velocity is
the counter-based TG recipe scaled to unit bulk mass flux.
"""
import numpy as np
from scipy.linalg import solve_banded

from numpy_tg import TALP, TGAM, TROH, TG


def fmm_spline(x, y):
    """CUBIC_SPLINE (Forsythe, Malcolm & Moler): coefficients b, c, d."""
    n = len(x)
    b, c, d = np.zeros(n), np.zeros(n), np.zeros(n)
    d[0] = x[1] - x[0]
    c[1] = (y[1] - y[0]) / d[0]
    for i in range(1, n - 1):
        d[i] = x[i + 1] - x[i]
        b[i] = 2.0 * (d[i - 1] + d[i])
        c[i + 1] = (y[i + 1] - y[i]) / d[i]
        c[i] = c[i + 1] - c[i]
    # end conditions from third divided differences
    b[0], b[-1] = -d[0], -d[n - 2]
    c[0] = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0])
    c[-1] = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4])
    c[0] = c[0] * d[0] * d[0] / (x[3] - x[0])
    c[-1] = -c[-1] * d[n - 2] * d[n - 2] / (x[n - 1] - x[n - 4])
    for i in range(1, n):
        t = d[i - 1] / b[i - 1]
        b[i] -= t * d[i - 1]
        c[i] -= t * c[i - 1]
    c[-1] /= b[-1]
    for i in range(n - 2, -1, -1):
        c[i] = (c[i] - d[i] * c[i + 1]) / b[i]
    b[-1] = (y[-1] - y[-2]) / d[-2] + d[-2] * (c[-2] + 2.0 * c[-1])
    b[:-1] = (y[1:] - y[:-1]) / d[:-1] - d[:-1] * (c[1:] + 2.0 * c[:-1])
    d[:-1] = (c[1:] - c[:-1]) / d[:-1]
    c *= 3.0
    d[-1] = d[-2]
    return b, c, d


class Spline:
    """NIST_SLEVAL: cubic on the bracketing interval; outside the table is an error."""

    def __init__(self, x, y):
        self.x, self.y = np.asarray(x, float), np.asarray(y, float)
        self.b, self.c, self.d = fmm_spline(self.x, self.y)

    def __call__(self, u):
        u = np.asarray(u, float)
        if not np.all((u > self.x[0]) & (u < self.x[-1])):
            raise ValueError("table look-up outside the table")
        i = np.searchsorted(self.x, u, side="right") - 1
        dx = u - self.x[i]
        return self.y[i] + dx * (self.b[i] + dx * (self.c[i] + dx * self.d[i]))


def synth_table(n=4096):
    """Synthetic table of the heated IO configuration: h in [-1, 1],
    cp = 1 + 8 exp(-(h/0.1)^2), T = int_{-1}^h dh/cp (composite Simpson,
    64 panels per table interval), rho = 1/(1+2T), mu = k = rho^-1/2."""
    H = -1.0 + 2.0 * np.arange(n) / (n - 1)
    m = 64
    wts = np.where(np.arange(m + 1) % 2 == 1, 4.0, 2.0)
    wts[0] = wts[-1] = 1.0
    hh = (H[1:] - H[:-1]) / m
    pts = H[:-1, None] + np.arange(m + 1)[None, :] * hh[:, None]
    pts[:, -1] = H[1:]
    seg = (wts[None, :] / (1.0 + 8.0 * np.exp(-(pts / 0.1) ** 2))).sum(axis=1) * hh / 3.0
    T = np.concatenate([[0.0], np.cumsum(seg)])
    D = 1.0 / (1.0 + 2.0 * T)
    M = 1.0 / np.sqrt(D)
    return H, T, D, M, M.copy()


class IO(TG):
    """x-periodic IO section (explicit viscous scheme, constant mass flux);
    the y mesh and the Poisson y-operator are the TG restatement's."""

    def __init__(self, nx, ny, nz, lx, lz, str2=2.0, istr2=1, ren=2800.0, dt=1e-3, thermal=0, prt=0.71,
                 qw=(1.0, 1.0), table=None, visc_scheme=0, isothermal=0):
        super().__init__(nx, ny, nz, lx, lz, str2=str2, istr2=istr2, ren=ren, dt=dt)
        self.thermal, self.qw, self.visc = thermal, qw, visc_scheme
        self.iso = (bool(isothermal & 1), bool(isothermal & 2))  # BCWALLHEAT bottom, top
        self.drhoi = {c: np.zeros((nz, ny + 2, nx)) for c in (1, 2, 3)}
        self.cvisc, self.cthecd = 1.0 / ren, 1.0 / ren / prt
        shape = (nz, ny + 2, nx)
        z = lambda: np.zeros(shape)
        self.g = {c: z() for c in (1, 2, 3)}
        self.g0 = {c: z() for c in (1, 2, 3)}
        self.ex0 = {c: z() for c in (1, 2, 3)}
        self.drho, self.rhoh, self.h, self.rhse0 = z(), z(), z(), z()
        self.T, self.D, self.D0, self.mu, self.mu0, self.k = (np.ones(shape) for _ in range(6))
        if thermal:
            H, Tt, D, M, K = (np.asarray(c, float) for c in (table if table is not None else synth_table())[:5])
            self.ht, self.td, self.tm, self.tk = Spline(H, Tt), Spline(Tt, D), Spline(Tt, M), Spline(Tt, K)
            th = Spline(Tt, H)
            # WALL_ISOTHERMAL_GIVEN: T, h, rho, mu, k at each iso-thermal wall's temperature
            self.wall = [None if not self.iso[s] else
                         tuple(float(v) for v in (qw[s], th(np.array([qw[s]]))[0], self.td(np.array([qw[s]]))[0],
                                                  self.tm(np.array([qw[s]]))[0], self.tk(np.array([qw[s]]))[0]))
                         for s in (0, 1)]
            n = len(H)
            hs = H[0] + np.arange(1, 3 * n) * (H[-1] - H[0]) / (3 * n)
            self.rhohmax = max(-1e-14, float(np.max(Spline(H, D)(hs) * hs)))

    # ---------------------------------------------------------- helpers
    def X(self, a, di=0, dj=0, dk=0):
        """a(i+di, j+dj, k+dk) over the interior rows j = 1..ny (periodic i, k)."""
        b = np.roll(a, shift=(-dk, -di), axis=(0, 2)) if (di or dk) else a
        return b[:, 1 + dj:self.ny + 1 + dj, :]

    def row(self, v, dj=0):
        return v[1 + dj:self.ny + 1 + dj][None, :, None]

    def interior(self, a, val):
        a[:, 1:self.ny + 1, :] = val

    def bc_vec(self, f):
        """BC_WALL_Q / BC_WALL_G: u, w ghosts 0; v = 0 on and beyond the walls."""
        ny = self.ny
        f[1][:, 0, :] = 0.0; f[3][:, 0, :] = 0.0; f[2][:, 1, :] = 0.0; f[2][:, 0, :] = 0.0
        f[1][:, ny + 1, :] = 0.0; f[3][:, ny + 1, :] = 0.0; f[2][:, ny + 1, :] = 0.0

    def bulk_of(self, a):
        return np.sum(a[:, 1:self.ny + 1] / self.row(self.dyfi)) / self.dzi / (self.area * self.nx)

    def div(self, G):
        X = self.X
        return ((X(G[1], 1) - X(G[1])) * self.dxi + (X(G[2], 0, 1) - X(G[2])) * self.row(self.dyfi) +
                (X(G[3], 0, 0, 1) - X(G[3])) * self.dzi)

    # ---------------------------------------------------------- staggered rho, mu
    def rho_stg(self):
        """DENSITY_Staggered on the u, v, w faces (rows 1..ny)."""
        if not self.thermal:
            return 1.0, 1.0, 1.0
        X, D, D0 = self.X, self.D, self.D0
        rx = (X(D) + X(D, -1) + X(D0) + X(D0, -1)) * 0.25
        rz = (X(D) + X(D, 0, 0, -1) + X(D0) + X(D0, 0, 0, -1)) * 0.25
        ry = (self.row(self.wff) * (X(D) + X(D0)) + self.row(self.wfb) * (X(D, 0, -1) + X(D0, 0, -1))) * 0.5
        return rx, ry, rz

    def mu_stg(self):
        """MU_Staggered: the xy-edge (1), xz-edge (2) and yz-edge (3) viscosities,
        rows 1..ny+1 of 1 and 3 (walls from the ghost cells), rows 1..ny of 2."""
        ny = self.ny
        m, m0 = self.mu, self.mu0
        xm = lambda a: np.roll(a, 1, axis=2)
        zm = lambda a: np.roll(a, 1, axis=0)
        s1, s2, s3 = np.zeros(m.shape), np.zeros(m.shape), np.zeros(m.shape)
        ex = m + xm(m) + m0 + xm(m0)
        ez = zm(m) + m + zm(m0) + m0
        wf, wb = self.wff[2:ny + 1][None, :, None], self.wfb[2:ny + 1][None, :, None]
        s1[:, 2:ny + 1] = (ex[:, 2:ny + 1] * wf + ex[:, 1:ny] * wb) * 0.25
        s3[:, 2:ny + 1] = (ez[:, 2:ny + 1] * wf + ez[:, 1:ny] * wb) * 0.25
        s2[:, 1:ny + 1] = (m + xm(m) + m0 + xm(m0) + zm(m) + zm(xm(m)) + zm(m0) + zm(xm(m0)))[:, 1:ny + 1] * 0.125
        for s in (s1, s3):
            s[:, 1] = 0.5 * (m0[:, 0] + m[:, 0])
            s[:, ny + 1] = 0.5 * (m0[:, ny + 1] + m[:, ny + 1])
        return s1, s2, s3

    # ---------------------------------------------------------- energy
    def table_props(self, h):
        T = self.ht(h)
        return T, self.td(T), self.tm(T), self.tk(T)

    def wall_thermal(self):
        """BC_WALL_ISOFLUX: ghost enthalpy extrapolated, ghost properties from the
        table; BC_WALL_ISOTHERMAL on an iso-thermal wall: the wall values."""
        ny, h = self.ny, self.h
        hb = 2.0 * h[:, 1] - self.wff[2] * h[:, 2] - self.wfb[2] * h[:, 1]
        ht = 2.0 * h[:, ny] - self.wff[ny] * h[:, ny] - self.wfb[ny] * h[:, ny - 1]
        for side, j, hg in ((0, 0, hb), (1, ny + 1, ht)):
            if self.iso[side]:
                Tw, hw, Dw, Mw, Kw = self.wall[side]
                self.h[:, j], self.T[:, j], self.D[:, j], self.mu[:, j], self.k[:, j] = hw, Tw, Dw, Mw, Kw
                self.rhoh[:, j] = hw * Dw
                continue
            T, D, M, K = self.table_props(hg)
            self.h[:, j], self.T[:, j], self.D[:, j], self.mu[:, j], self.k[:, j] = hg, T, D, M, K
            self.rhoh[:, j] = hg * D

    def eng(self, ns):
        """SOLVERRK3_ENG_IO: RHS_ENERGY_EXPLICIT, the RK3 update with the RHOHmax
        limiter, ENTHALPY/DENSITY_UPDATE, THERM_PROP_UPDATE, wall ghosts."""
        ny, X, row = self.ny, self.X, self.row
        self.mu0 = self.mu.copy()
        self.D0 = self.D.copy()
        H, T, K, G, G0 = self.h, self.T, self.k, self.g, self.g0
        wff, wfb, wffp, wfbp = row(self.wff), row(self.wfb), row(self.wff, 1), row(self.wfb, 1)
        dxr = ((X(H, 1) + X(H)) * (X(G0[1], 1) + X(G[1], 1)) - (X(H) + X(H, -1)) * (X(G0[1]) + X(G[1]))) * (self.dxi * 0.25)
        dyr = ((wffp * X(H, 0, 1) + wfbp * X(H)) * (X(G0[2], 0, 1) + X(G[2], 0, 1)) -
               (wff * X(H) + wfb * X(H, 0, -1)) * (X(G0[2]) + X(G[2]))) * (row(self.dyfi) * 0.5)
        dzr = ((X(H, 0, 0, 1) + X(H)) * (X(G0[3], 0, 0, 1) + X(G[3], 0, 0, 1)) -
               (X(H) + X(H, 0, 0, -1)) * (X(G0[3]) + X(G[3]))) * (self.dzi * 0.25)
        dxk = ((X(K, 1) + X(K)) * (X(T, 1) - X(T)) - (X(K) + X(K, -1)) * (X(T) - X(T, -1))) * (self.dxi ** 2 * 0.5 * self.cthecd)
        c_up = self.dyci[2:ny + 2].copy()
        c_dn = self.dyci[1:ny + 1].copy()
        if not self.iso[1]:
            c_up[-1] = 1.0
        if not self.iso[0]:
            c_dn[0] = 1.0
        k_up = (wffp * X(K, 0, 1) + wfbp * X(K)) * (X(T, 0, 1) - X(T)) * c_up[None, :, None]
        k_dn = (wff * X(K) + wfb * X(K, 0, -1)) * (X(T) - X(T, 0, -1)) * c_dn[None, :, None]
        if not self.iso[0]:
            k_dn[:, 0, :] = -self.qw[0]  # heat flux into the fluid through the bottom wall
        if not self.iso[1]:
            k_up[:, -1, :] = self.qw[1]  # and through the top wall
        dyk = (k_up - k_dn) * (row(self.dyfi) * self.cthecd)
        dzk = ((X(K, 0, 0, 1) + X(K)) * (X(T, 0, 0, 1) - X(T)) - (X(K, 0, 0, -1) + X(K)) * (X(T) - X(T, 0, 0, -1))) * (self.dzi ** 2 * 0.5 * self.cthecd)
        R = -dxr - dyr - dzr + dxk + dyk + dzk
        rh = np.minimum(self.rhohmax + 1e-14, X(self.rhoh) + TGAM[ns] * self.dt * R + TROH[ns] * self.dt * X(self.rhse0))
        self.interior(self.rhoh, rh)
        self.interior(self.rhse0, R)
        D = self.td(self.ht(rh / X(self.D)))
        h = rh / D
        T, D, M, Kp = self.table_props(h)
        for a, v in ((self.h, h), (self.T, T), (self.D, D), (self.mu, M), (self.k, Kp)):
            self.interior(a, v)
        self.wall_thermal()

    # ---------------------------------------------------------- momentum
    def prep(self, ns):
        """DENSITY_TIME_DERIVATION (thermal), DENSITY_implicit_add (thermal,
        semi-implicit scheme), then VELOCITY_CALC_io: u = G / rho_stag."""
        if self.thermal:
            self.interior(self.drho, ((TGAM[ns] + TROH[ns]) * self.div(self.g) + TROH[ns] * self.div(self.g0)) /
                          (TGAM[ns] - 2.0))
        X, G = self.X, self.g
        rx, ry, rz = self.rho_stg()
        if self.thermal and self.visc:
            D0 = self.D0
            for c in (1, 2, 3):
                self.drhoi[c][:] = 0.0
            self.interior(self.drhoi[1], 1.0 / rx - 1.0 / ((X(D0) + X(D0, -1)) * 0.5))
            self.interior(self.drhoi[3], 1.0 / rz - 1.0 / ((X(D0) + X(D0, 0, 0, -1)) * 0.5))
            d2 = 1.0 / ry - 1.0 / (self.row(self.wff) * X(D0) + self.row(self.wfb) * X(D0, 0, -1))
            self.drhoi[2][:, 2:self.ny + 1, :] = d2[:, 1:, :]
        self.interior(self.q[1], X(G[1]) / rx)
        self.interior(self.q[3], X(G[3]) / rz)
        self.q[2][:, 2:self.ny + 1, :] = (X(G[2]) / ry)[:, 1:, :]
        self.bc_vec(self.q)

    def mom(self, ns):
        """SOLVERRK3_MOM_IO: convection + explicit viscous terms, RHS_MOM_EXPLICIT_io
        with the constant-mass-flux gradient, MASSFLUX_CALC_IO, DIVG_io, the
        FISHPACK Poisson solve, PRCALC_io, MASSFLUX_UPDATE_IO."""
        self.g0 = {c: self.g[c].copy() for c in (1, 2, 3)}
        ex, ey, ez, ex_conv, ey_conv, ez_conv = self.mom_terms()
        ny, X, row = self.ny, self.X, self.row
        gx, gy, gz = self.g[1], self.g[2], self.g[3]
        dycj, dxi, dzi = row(self.dyci), self.dxi, self.dzi
        if self.visc:
            self.mom_semi_implicit(ns, ex_conv, ey_conv, ez_conv)
            return
        # RK3 combination and pressure gradient
        p, dt, alp = self.p, self.dt, TALP[ns]
        rx = (TGAM[ns] * ex + TROH[ns] * X(self.ex0[1])) * dt - (X(p) - X(p, -1)) * (alp * dt * dxi)
        ry = (TGAM[ns] * ey + TROH[ns] * X(self.ex0[2])) * dt - (X(p) - X(p, 0, -1)) * (alp * dt * dycj)
        rz = (TGAM[ns] * ez + TROH[ns] * X(self.ex0[3])) * dt - (X(p) - X(p, 0, 0, -1)) * (alp * dt * dzi)
        self.interior(self.ex0[1], ex)
        self.interior(self.ex0[3], ez)
        self.ex0[2][:, 2:ny + 1, :] = ey[:, 1:, :]
        rx = rx - np.sum(rx / row(self.dyfi)) / self.volm  # DPGRNS: constant mass flux
        gx[:, 1:ny + 1, :] += rx
        gz[:, 1:ny + 1, :] += rz
        gy[:, 2:ny + 1, :] += ry[:, 1:, :]
        self.bc_vec(self.g)
        self.project(ns)

    def mom_terms(self):
        """The convection + explicit viscous terms of the three momentum
        components on the interior (with the bare convection terms)."""
        ny, X, row = self.ny, self.X, self.row
        u, v, w = self.q[1], self.q[2], self.q[3]
        gx, gy, gz = self.g[1], self.g[2], self.g[3]
        wff, wfb, wffp, wfbp = row(self.wff), row(self.wfb), row(self.wff, 1), row(self.wfb, 1)
        dyfj, dycj, dycp, dyfm = row(self.dyfi), row(self.dyci), row(self.dyci, 1), row(self.dyfi, -1)
        dxi, dzi, cv = self.dxi, self.dzi, self.cvisc
        if self.thermal:
            ms = self.mu_stg()
            M = lambda di=0, dj=0, dk=0: 0.5 * (X(self.mu0, di, dj, dk) + X(self.mu, di, dj, dk))
            S1, S2, S3 = ((lambda di=0, dj=0, dk=0, s=s: X(s, di, dj, dk)) for s in ms)
        else:
            M = S1 = S2 = S3 = lambda *a: 1.0

        def divu(di=0, dj=0, dk=0):  # DIVG_U_io: div u / 3 at the cell (i+di, j+dj, k+dk)
            return ((X(u, di + 1, dj, dk) - X(u, di, dj, dk)) * dxi +
                    (X(v, di, dj + 1, dk) - X(v, di, dj, dk)) * row(self.dyfi, dj) +
                    (X(w, di, dj, dk + 1) - X(w, di, dj, dk)) * dzi) / 3.0

        # x-momentum at the u faces
        ex = -(((X(gx, 1) + X(gx)) * (X(u, 1) + X(u)) - (X(gx) + X(gx, -1)) * (X(u) + X(u, -1))) * (dxi * 0.25) +
               ((X(gy, 0, 1) + X(gy, -1, 1)) * (wffp * X(u, 0, 1) + wfbp * X(u)) -
                (X(gy) + X(gy, -1)) * (wff * X(u) + wfb * X(u, 0, -1))) * (dyfj * 0.5) +
               ((X(gz, 0, 0, 1) + X(gz, -1, 0, 1)) * (X(u, 0, 0, 1) + X(u)) -
                (X(gz) + X(gz, -1)) * (X(u) + X(u, 0, 0, -1))) * (dzi * 0.25))
        d11 = (M() * ((X(u, 1) - X(u)) * dxi - divu()) - M(-1) * ((X(u) - X(u, -1)) * dxi - divu(-1))) * (2.0 * dxi * cv)
        d12 = (S1(0, 1) * ((X(u, 0, 1) - X(u)) * dycp + (X(v, 0, 1) - X(v, -1, 1)) * dxi) -
               S1() * ((X(u) - X(u, 0, -1)) * dycj + (X(v) - X(v, -1)) * dxi)) * (dyfj * cv)
        d13 = (S2(0, 0, 1) * ((X(u, 0, 0, 1) - X(u)) * dzi + (X(w, 0, 0, 1) - X(w, -1, 0, 1)) * dxi) -
               S2() * ((X(u) - X(u, 0, 0, -1)) * dzi + (X(w) - X(w, -1)) * dxi)) * (dzi * cv)
        ex_conv, ex = ex, ex + d11 + d12 + d13
        # y-momentum at the v faces (row 1 is the wall and is dropped)
        ey = -(((wff * X(gx, 1) + wfb * X(gx, 1, -1)) * (X(v, 1) + X(v)) -
                (wff * X(gx) + wfb * X(gx, 0, -1)) * (X(v) + X(v, -1))) * (dxi * 0.5) +
               ((X(gy, 0, 1) + X(gy)) * (X(v, 0, 1) + X(v)) - (X(gy) + X(gy, 0, -1)) * (X(v) + X(v, 0, -1))) * (dycj * 0.25) +
               ((wff * X(gz, 0, 0, 1) + wfb * X(gz, 0, -1, 1)) * (X(v, 0, 0, 1) + X(v)) -
                (wff * X(gz) + wfb * X(gz, 0, -1)) * (X(v) + X(v, 0, 0, -1))) * (dzi * 0.5))
        d21 = (S1(1) * ((X(v, 1) - X(v)) * dxi + (X(u, 1) - X(u, 1, -1)) * dycj) -
               S1() * ((X(v) - X(v, -1)) * dxi + (X(u) - X(u, 0, -1)) * dycj)) * (dxi * cv)
        d22 = (M() * ((X(v, 0, 1) - X(v)) * dyfj - divu()) - M(0, -1) * ((X(v) - X(v, 0, -1)) * dyfm - divu(0, -1))) * (2.0 * dycj * cv)
        d23 = (S3(0, 0, 1) * ((X(v, 0, 0, 1) - X(v)) * dzi + (X(w, 0, 0, 1) - X(w, 0, -1, 1)) * dycj) -
               S3() * ((X(v) - X(v, 0, 0, -1)) * dzi + (X(w) - X(w, 0, -1)) * dycj)) * (dzi * cv)
        ey_conv, ey = ey, ey + d21 + d22 + d23
        # z-momentum at the w faces
        ez = -(((X(gx, 1) + X(gx, 1, 0, -1)) * (X(w, 1) + X(w)) - (X(gx) + X(gx, 0, 0, -1)) * (X(w) + X(w, -1))) * (dxi * 0.25) +
               ((X(gy, 0, 1) + X(gy, 0, 1, -1)) * (wffp * X(w, 0, 1) + wfbp * X(w)) -
                (X(gy) + X(gy, 0, 0, -1)) * (wff * X(w) + wfb * X(w, 0, -1))) * (dyfj * 0.5) +
               ((X(gz, 0, 0, 1) + X(gz)) * (X(w, 0, 0, 1) + X(w)) - (X(gz) + X(gz, 0, 0, -1)) * (X(w) + X(w, 0, 0, -1))) * (dzi * 0.25))
        d31 = (S2(1) * ((X(w, 1) - X(w)) * dxi + (X(u, 1) - X(u, 1, 0, -1)) * dzi) -
               S2() * ((X(w) - X(w, -1)) * dxi + (X(u) - X(u, 0, 0, -1)) * dzi)) * (dxi * cv)
        d32 = (S3(0, 1) * ((X(w, 0, 1) - X(w)) * dycp + (X(v, 0, 1) - X(v, 0, 1, -1)) * dzi) -
               S3() * ((X(w) - X(w, 0, -1)) * dycj + (X(v) - X(v, 0, 0, -1)) * dzi)) * (dyfj * cv)
        d33 = (M() * ((X(w, 0, 0, 1) - X(w)) * dzi - divu()) - M(0, 0, -1) * ((X(w) - X(w, 0, 0, -1)) * dzi - divu(0, 0, -1))) * (2.0 * dzi * cv)
        ez_conv, ez = ez, ez + d31 + d32 + d33
        return ex, ey, ez, ex_conv, ey_conv, ez_conv

    def project(self, ns):
        """DIVG_io, the FISHPACK solve, PRCALC_io (the semi-implicit branch with
        the physical right-hand side), MASSFLUX_UPDATE_IO."""
        ny, X, row = self.ny, self.X, self.row
        p, dt, alp = self.p, self.dt, TALP[ns]
        gx, gy, gz = self.g[1], self.g[2], self.g[3]
        dxi, dzi, dycj = self.dxi, self.dzi, row(self.dyci)
        rhs = (self.div(self.g) + X(self.drho)) / (dt * alp)
        phi = self.poisson_io(rhs)
        self.phi[:] = 0.0
        self.interior(self.phi, phi)
        self.bc_copy(self.phi)
        if self.visc:
            self.interior(p, X(p) + X(self.phi) - 0.5 * alp * dt * self.cvisc * rhs)
        else:
            self.interior(p, X(p) + X(self.phi))
        self.bc_copy(p)
        f = self.phi
        gx[:, 1:ny + 1, :] -= (X(f) - X(f, -1)) * (dt * alp * dxi)
        gz[:, 1:ny + 1, :] -= (X(f) - X(f, 0, 0, -1)) * (dt * alp * dzi)
        gy[:, 2:ny + 1, :] -= ((X(f) - X(f, 0, -1)) * (dt * alp * dycj))[:, 1:, :]
        self.bc_vec(self.g)

    # ---------------------------------------------------------- semi-implicit scheme
    def stg_fields(self):
        """MU_STG 1-3 and RHO_STG 1-3 as full arrays (ones with the energy
        equation off); RHO_STG(2) row 0 keeps its allocation value 1."""
        ny, X = self.ny, self.X
        shape = self.D.shape
        if not self.thermal:
            one = np.ones(shape)
            return (one, one, one), (one, one, one)
        s1, s2, s3 = self.mu_stg()
        D, D0 = self.D, self.D0
        r1, r2, r3 = np.ones(shape), np.ones(shape), np.ones(shape)
        self.interior(r1, (X(D) + X(D, -1) + X(D0) + X(D0, -1)) * 0.25)
        self.interior(r3, (X(D) + X(D, 0, 0, -1) + X(D0) + X(D0, 0, 0, -1)) * 0.25)
        ry = (self.row(self.wff) * (X(D) + X(D0)) + self.row(self.wfb) * (X(D, 0, -1) + X(D0, 0, -1))) * 0.5
        r2[:, 2:ny + 1] = ry[:, 1:]
        r2[:, 1] = 0.5 * (D0[:, 0] + D[:, 0])
        r2[:, ny + 1] = 0.5 * (D0[:, ny + 1] + D[:, ny + 1])
        return (s1, s2, s3), (r1, r2, r3)

    def par_viscous(self):
        """VISCOUS_PAR_EXPLT_X/Y/Z_io: per component the explicit part, the part
        treated by the factors and the density part (DRHOI_STG)."""
        ny, X, row = self.ny, self.X, self.row
        u, v, w = self.q[1], self.q[2], self.q[3]
        gx, gy, gz = self.g[1], self.g[2], self.g[3]
        r1, r2, r3 = self.drhoi[1], self.drhoi[2], self.drhoi[3]
        mu = self.mu
        (s1, s2, s3), _ = self.stg_fields()
        dxi, dzi, cv = self.dxi, self.dzi, self.cvisc
        dyfj, dycj, dycp, dyfm = row(self.dyfi), row(self.dyci), row(self.dyci, 1), row(self.dyfi, -1)
        out = {}
        # x (rows 1..ny)
        c1, c2, c32 = -2.0 / 3.0 * dxi * cv, dyfj * cv, dzi * cv
        fe = X(mu) * ((X(v, 0, 1) - X(v)) * dyfj + (X(w, 0, 0, 1) - X(w)) * dzi)
        fi = X(mu) * ((X(u, 1) - X(u)) * dxi)
        fa = X(mu) * ((X(gx, 1) * X(r1, 1) - X(gx) * X(r1)) * dxi)
        be = X(mu, -1) * ((X(v, -1, 1) - X(v, -1)) * dyfj + (X(w, -1, 0, 1) - X(w, -1)) * dzi)
        bi = X(mu, -1) * ((X(u) - X(u, -1)) * dxi)
        ba = X(mu, -1) * ((X(gx) * X(r1) - X(gx, -1) * X(r1, -1)) * dxi)
        d11 = ((fe - be) * c1, (fi - bi) * c1 * (-2.0), (fa - ba) * c1 * (-2.0))
        vp, vc = X(s1, 0, 1), X(s1)
        fe = vp * ((X(v, 0, 1) - X(v, -1, 1)) * dxi)
        fi = vp * ((X(u, 0, 1) - X(u)) * dycp)
        fa = vp * ((X(gx, 0, 1) * X(r1, 0, 1) - X(gx) * X(r1)) * dycp)
        be = vc * ((X(v) - X(v, -1)) * dxi)
        bi = vc * ((X(u) - X(u, 0, -1)) * dycj)
        ba = vc * ((X(gx) * X(r1) - X(gx, 0, -1) * X(r1, 0, -1)) * dycj)
        d12 = ((fe - be) * c2, (fi - bi) * c2, (fa - ba) * c2)
        vp, vc = X(s2, 0, 0, 1), X(s2)
        fe = vp * ((X(w, 0, 0, 1) - X(w, -1, 0, 1)) * dxi)
        fi = vp * ((X(u, 0, 0, 1) - X(u)) * dzi)
        fa = vp * ((X(u, 0, 0, 1) * X(r1, 0, 0, 1) - X(u) * X(r1)) * dzi)  # Q_io, as written
        be = vc * ((X(w) - X(w, -1)) * dxi)
        bi = vc * ((X(u) - X(u, 0, 0, -1)) * dzi)
        ba = vc * ((X(u) * X(r1) - X(u, 0, 0, -1) * X(r1, 0, 0, -1)) * dzi)
        d13 = ((fe - be) * c32, (fi - bi) * c32, (fa - ba) * c32)
        out[1] = tuple(d11[t] + d12[t] + d13[t] for t in range(3))
        # y (rows 2..ny; row 1 dropped)
        c1, c3, c2 = dxi * cv, dzi * cv, -2.0 / 3.0 * dycj * cv
        fe = X(mu) * ((X(u, 1) - X(u)) * dxi + (X(w, 0, 0, 1) - X(w)) * dzi)
        fi = X(mu) * ((X(v, 0, 1) - X(v)) * dyfj)
        fa = X(mu) * ((X(gy, 0, 1) * X(r2, 0, 1) - X(gy) * X(r2)) * dyfj)
        be = X(mu, 0, -1) * ((X(u, 1, -1) - X(u, 0, -1)) * dxi + (X(w, 0, -1, 1) - X(w, 0, -1)) * dzi)
        bi = X(mu, 0, -1) * ((X(v) - X(v, 0, -1)) * dyfm)
        ba = X(mu, 0, -1) * ((X(gy) * X(r2) - X(gy, 0, -1) * X(r2, 0, -1)) * dyfm)
        d22 = ((fe - be) * c2, (fi - bi) * c2 * (-2.0), (fa - ba) * c2 * (-2.0))
        vp, vc = X(s1, 1), X(s1)
        fe = vp * ((X(u, 1) - X(u, 1, -1)) * dycj)
        fi = vp * ((X(v, 1) - X(v)) * dxi)
        fa = vp * ((X(gy, 1) * X(r2, 1) - X(gy) * X(r2)) * dxi)
        be = vc * ((X(u) - X(u, 0, -1)) * dycj)
        bi = vc * ((X(v) - X(v, -1)) * dxi)
        ba = vc * ((X(gy) * X(r2) - X(gy, -1) * X(r2, -1)) * dxi)
        d21 = ((fe - be) * c1, (fi - bi) * c1, (fa - ba) * c1)
        vp, vc = X(s3, 0, 0, 1), X(s3)
        fe = vp * ((X(w, 0, 0, 1) - X(w, 0, -1, 1)) * dycj)
        fi = vp * ((X(v, 0, 0, 1) - X(v)) * dzi)
        fa = vp * ((X(gy, 0, 0, 1) * X(r2, 0, 0, 1) - X(gy) * X(r2)) * dzi)
        be = vc * ((X(w) - X(w, 0, -1)) * dycj)
        bi = vc * ((X(v) - X(v, 0, 0, -1)) * dzi)
        ba = vc * ((X(gy) * X(r2) - X(gy, 0, 0, -1) * X(r2, 0, 0, -1)) * dzi)
        d23 = ((fe - be) * c3, (fi - bi) * c3, (fa - ba) * c3)
        out[2] = tuple(d21[t] + d22[t] + d23[t] for t in range(3))
        # z (rows 1..ny)
        c1, c3, c2 = dxi * cv, -2.0 / 3.0 * dzi * cv, dyfj * cv
        fe = X(mu) * ((X(u, 1) - X(u)) * dxi + (X(v, 0, 1) - X(v)) * dyfj)
        fi = X(mu) * ((X(w, 0, 0, 1) - X(w)) * dzi)
        fa = X(mu) * ((X(gz, 0, 0, 1) * X(r3, 0, 0, 1) - X(gz) * X(r3)) * dzi)
        be = X(mu, 0, 0, -1) * ((X(u, 1, 0, -1) - X(u, 0, 0, -1)) * dxi + (X(v, 0, 1, -1) - X(v, 0, 0, -1)) * dyfj)
        bi = X(mu, 0, 0, -1) * ((X(w) - X(w, 0, 0, -1)) * dzi)
        ba = X(mu, 0, 0, -1) * ((X(gz) * X(r3) - X(gz, 0, 0, -1) * X(r3, 0, 0, -1)) * dzi)
        d33 = ((fe - be) * c3, (fi - bi) * c3 * (-2.0), (fa - ba) * c3 * (-2.0))
        vp, vc = X(s2, 1), X(s2)
        fe = vp * ((X(u, 1) - X(u, 1, 0, -1)) * dzi)
        fi = vp * ((X(w, 1) - X(w)) * dxi)
        fa = vp * ((X(gz, 1) * X(r3, 1) - X(gz) * X(r3)) * dxi)
        be = vc * ((X(u) - X(u, 0, 0, -1)) * dzi)
        bi = vc * ((X(w) - X(w, -1)) * dxi)
        ba = vc * ((X(gz) * X(r3) - X(gz, -1) * X(r3, -1)) * dxi)
        d31 = ((fe - be) * c1, (fi - bi) * c1, (fa - ba) * c1)
        vp, vc = X(s3, 0, 1), X(s3)
        fe = vp * ((X(v, 0, 1) - X(v, 0, 1, -1)) * dzi)
        fi = vp * ((X(w, 0, 1) - X(w)) * dycp)
        fa = vp * ((X(gz, 0, 1) * X(r3, 0, 1) - X(gz) * X(r3)) * dycp)
        be = vc * ((X(v) - X(v, 0, 0, -1)) * dzi)
        bi = vc * ((X(w) - X(w, 0, -1)) * dycj)
        ba = vc * ((X(gz) * X(r3) - X(gz, 0, -1) * X(r3, 0, -1)) * dycj)
        d32 = ((fe - be) * c2, (fi - bi) * c2, (fa - ba) * c2)
        out[3] = tuple(d31[t] + d32[t] + d33[t] for t in range(3))
        return out

    @staticmethod
    def tri_solve(a, b, c, r, cyclic):
        """Batched dense LU of tridiagonal lines along the last axis:
        a x(i-1) + b x(i) + c x(i+1) = r (indices mod n when cyclic)."""
        n = a.shape[-1]
        M = np.zeros(a.shape + (n,))
        idx = np.arange(n)
        M[..., idx, idx] = b
        M[..., idx[1:], idx[:-1]] = a[..., 1:]
        M[..., idx[:-1], idx[1:]] = c[..., :-1]
        if cyclic:
            M[..., 0, n - 1] = a[..., 0]
            M[..., n - 1, 0] = c[..., n - 1]
        return np.linalg.solve(M, r[..., None])[..., 0]

    def momfa(self, ns, comp, rhs):
        """MOMFA_io: x, z, y factor solves of component comp on RHS_io (rows
        1..ny array), then G += dG from row N2I."""
        ny, X = self.ny, self.X
        j0 = 1 if comp != 2 else 2  # first row (index into 1..ny) solved in x and z
        facoe = 0.5 * TALP[ns] * self.dt * self.cvisc
        (s1, s2, s3), (r1, r2, r3) = self.stg_fields()
        rs = {1: r1, 2: r2, 3: r3}[comp]
        vis = self.mu
        # x
        c1, c2 = facoe * 4.0 / 3.0 * self.dxi ** 2, facoe * self.dxi ** 2
        if comp == 1:
            amu, apu = -c1 * X(vis, -1), -c1 * X(vis)
        elif comp == 2:
            amu, apu = -c2 * X(s1), -c2 * X(s1, 1)
        else:
            amu, apu = -c2 * X(s2), -c2 * X(s2, 1)
        a, c, b = amu / X(rs, -1), apu / X(rs, 1), 1.0 - (amu + apu) / X(rs)
        sl = slice(j0 - 1, ny)
        rhs[:, sl] = self.tri_solve(a[:, sl], b[:, sl], c[:, sl], rhs[:, sl], True)
        # z
        c1, c2 = facoe * 4.0 / 3.0 * self.dzi ** 2, facoe * self.dzi ** 2
        if comp == 1:
            amu, apu = -c2 * X(s2), -c2 * X(s2, 0, 0, 1)
        elif comp == 2:
            amu, apu = -c2 * X(s3), -c2 * X(s3, 0, 0, 1)
        else:
            amu, apu = -c1 * X(vis, 0, 0, -1), -c1 * X(vis)
        a, c, b = amu / X(rs, 0, 0, -1), apu / X(rs, 0, 0, 1), 1.0 - (amu + apu) / X(rs)
        tz = lambda f: np.transpose(f[:, sl], (1, 2, 0))  # (rows, x, z)
        rhs[:, sl] = np.transpose(self.tri_solve(tz(a), tz(b), tz(c), tz(rhs), True), (2, 0, 1))
        # y (rows 1..ny for every component)
        jj = np.arange(1, ny + 1)
        am, ap = self.amvr[comp][jj][None, :, None], self.apvr[comp][jj][None, :, None]
        if comp in (1, 3):
            fmu = s1 if comp == 1 else s3
            amvr1 = 4.0 / (2.0 / self.dyci[2] + 1.0 / self.dyfi[1]) * (2.0 * self.dyfi[1])
            apvrn = 4.0 / (2.0 / self.dyci[ny] + 1.0 / self.dyfi[ny]) * (2.0 * self.dyfi[ny])
            amu = -facoe * am * X(fmu)
            apu = -facoe * ap * X(fmu, 0, 1)
            amu[:, 0] = -facoe * amvr1 * (X(vis)[:, 0] + X(vis, 0, -1)[:, 0]) * 0.5
            apu[:, -1] = -facoe * apvrn * (X(vis)[:, -1] + X(vis, 0, 1)[:, -1]) * 0.5
            a, c = amu / X(rs, 0, -1), apu / X(rs, 0, 1)
            a[:, 0] = 0.0
            c[:, -1] = 0.0
        else:
            cy = facoe * 4.0 / 3.0
            amu, apu = -cy * am * X(vis, 0, -1), -cy * ap * X(vis)
            a, c = amu / X(rs, 0, -1), apu / X(rs)
            c[:, 0] = apu[:, 0] / X(rs, 0, 1)[:, 0]
            a[:, 0] = 0.0
            c[:, -1] = 0.0
        b = 1.0 - (amu + apu) / X(rs)
        ty = lambda f: np.transpose(f, (0, 2, 1))  # (z, x, rows)
        x = np.transpose(self.tri_solve(ty(a), ty(b), ty(c), ty(rhs), False), (0, 2, 1))
        self.g[comp][:, j0:ny + 1] += x[:, j0 - 1:]

    def mom_semi_implicit(self, ns, cx, cy, cz):
        """SOLVERRK3_MOM_IO with visthemflg = 1: per component the split
        viscous terms, RHS_MOM_EXPLICIT_io's implicit branch, MOMFA_io."""
        ny, X, row = self.ny, self.X, self.row
        p, dt, alp = self.p, self.dt, TALP[ns]
        par = self.par_viscous()
        conv = {1: cx, 2: cy, 3: cz}
        pg = {1: (X(p) - X(p, -1)) * (alp * dt * self.dxi),
              2: (X(p) - X(p, 0, -1)) * (alp * dt * row(self.dyci)),
              3: (X(p) - X(p, 0, 0, -1)) * (alp * dt * self.dzi)}
        for comp in (1, 2, 3):
            ex, im, ad = par[comp]
            explt = ex + conv[comp]
            r = (TGAM[ns] * explt + TROH[ns] * X(self.ex0[comp])) * dt
            r = r + alp * dt * im + 0.5 * (alp * dt) * ad
            r = r - pg[comp]
            if comp == 2:
                self.ex0[2][:, 2:ny + 1] = explt[:, 1:]
                r[:, 0] = 0.0
            else:
                self.interior(self.ex0[comp], explt)
            if comp == 1:
                r = r - np.sum(r / row(self.dyfi)) / self.volm  # DPGRNS
            self.momfa(ns, comp, r)
        self.bc_vec(self.g)
        self.project(ns)

    def poisson_io(self, rhs):
        """FISHPACK_POIS3D_SIMPLE's operator diagonalised with complex FFTs in x
        and z; the mean mode drops its last equation and takes phi(ny) = 0."""
        nx, ny, nz = self.nx, self.ny, self.nz
        F = np.fft.fft(np.fft.fft(rhs, axis=2), axis=0)  # (kz, j, kx)
        lam_x = -4.0 * self.dxi ** 2 * np.sin(np.pi * np.arange(nx) / nx) ** 2
        lam_z = -4.0 * self.dzi ** 2 * np.sin(np.pi * np.arange(nz) / nz) ** 2
        am, ac, ap = self.amph[1:ny + 1], self.acph[1:ny + 1], self.apph[1:ny + 1]
        out = np.zeros_like(F)
        ab = np.zeros((3, ny), dtype=complex)
        ab[0, 1:] = ap[:-1]
        ab[2, :-1] = am[1:]
        for a in range(nz):
            for b in range(nx):
                ab[1] = ac + lam_x[b] + lam_z[a]
                if a == 0 and b == 0:
                    out[a, :-1, b] = solve_banded((1, 1), ab[:, :-1], F[a, :-1, b])
                else:
                    out[a, :, b] = solve_banded((1, 1), ab, F[a, :, b])
        return np.real(np.fft.ifft(np.fft.ifft(out, axis=0), axis=2))

    # ---------------------------------------------------------- driver
    def init_random(self, seed, amp):
        """TG velocity recipe scaled to unit bulk mass flux (VELO2MASSFLUX,
        Unified_massflux), h = 0 with the table's properties, then
        CALC_INITIALIZATION_io (energy with NS = 0, momentum with NS = 0)."""
        ny = self.ny
        if self.thermal:
            T0, D0, M0, K0 = (float(x[0]) for x in self.table_props(np.array([0.0])))
        else:
            T0 = D0 = M0 = K0 = 1.0
        for a, val in ((self.T, T0), (self.D, D0), (self.D0, D0), (self.mu, M0), (self.mu0, M0), (self.k, K0)):
            a[:] = val
        for a in (self.h, self.rhoh, self.rhse0, self.drho):
            a[:] = 0.0
        super().init_random(seed, amp)
        r_face = (D0 + D0 + D0 + D0) * 0.25
        r_v = (self.wff * (D0 + D0) + self.wfb * (D0 + D0)) * 0.5

        def velo2massflux():
            for c in (1, 2, 3):
                self.g[c][:] = 0.0
            self.g[1][:, 1:ny + 1] = self.q[1][:, 1:ny + 1] * r_face
            self.g[3][:, 1:ny + 1] = self.q[3][:, 1:ny + 1] * r_face
            self.g[2][:, 2:ny + 1] = self.q[2][:, 2:ny + 1] * r_v[2:ny + 1][None, :, None]

        velo2massflux()
        gm = self.bulk_of(self.g[1])
        for c in (1, 2, 3):
            self.q[c] /= gm
        velo2massflux()
        self.bc_vec(self.q)
        self.p[:] = 0.0
        for c in (1, 2, 3):
            self.g0[c][:] = 0.0
            self.ex0[c][:] = 0.0
        if self.thermal:
            self.wall_thermal()
            self.eng(0)
        self.mom(0)

    def substep(self, ns):
        if self.thermal:
            self.eng(ns)
        self.prep(ns)
        self.mom(ns)

    def divmax(self):
        """max |div G + drho| over the cells (DIVGCK_io)."""
        return float(np.abs(self.div(self.g) + self.X(self.drho)).max())


def io_stats(f, dxi, dzi, dyfi, dyci, thermal):
    """PP_MEAN_ZX_FLOW_Xperiodic_IO (src/processing/PP_MEAN_ZX.f90:299-872),
    channel branch, as whole-array shifts: (ny, 360) xz-plane averages of the
    cell-centred U, G, p, the velocity gradient D and (thermal) T, rho, h,
    mu, k and the h and T gradients, in the library's output order.  f maps
    u, v, w, p, gx, gy, gz (and h, t, rho, mu, k) to (nz, ny + 2, nx) arrays;
    dyfi and dyci are 1-based arrays of length ny + 2."""
    nz, ny2, nx = f["u"].shape
    ny = ny2 - 2

    def S(a, di=0, dj=0, dk=0):
        b = np.roll(a, shift=(-dk, -di), axis=(0, 2)) if (di or dk) else a
        return b[:, 1 + dj:ny + 1 + dj, :]

    u, v, w = f["u"], f["v"], f["w"]
    U = [(S(u) + S(u, 1)) * 0.5, (S(v) + S(v, 0, 1)) * 0.5, (S(w) + S(w, 0, 0, 1)) * 0.5]
    G = [(S(f["gx"]) + S(f["gx"], 1)) * 0.5, (S(f["gy"]) + S(f["gy"], 0, 1)) * 0.5,
         (S(f["gz"]) + S(f["gz"], 0, 0, 1)) * 0.5]
    yc = dyci[2:ny + 2][None, :, None]
    yj = dyci[1:ny + 1][None, :, None]
    yf = dyfi[1:ny + 1][None, :, None]
    cc = lambda a, di=0, dj=0, dk=0, ax=0: (S(a, di, dj, dk) + S(a, di + (ax == 0), dj + (ax == 1), dk + (ax == 2))) * 0.5
    D = [[None] * 3 for _ in range(3)]
    D[0][0] = (S(u, 1) - S(u)) * dxi
    D[0][1] = ((cc(u, 0, 1) - U[0]) * yc + (U[0] - cc(u, 0, -1)) * yj) * 0.5
    D[0][2] = (cc(u, 0, 0, 1) - cc(u, 0, 0, -1)) * dzi * 0.5
    D[1][0] = (cc(v, 1, ax=1) - cc(v, -1, ax=1)) * dxi * 0.5
    D[1][1] = (S(v, 0, 1) - S(v)) * yf
    D[1][2] = (cc(v, 0, 0, 1, ax=1) - cc(v, 0, 0, -1, ax=1)) * dzi * 0.5
    D[2][0] = (cc(w, 1, ax=2) - cc(w, -1, ax=2)) * dxi * 0.5
    D[2][1] = ((cc(w, 0, 1, ax=2) - U[2]) * yc + (U[2] - cc(w, 0, -1, ax=2)) * yj) * 0.5
    D[2][2] = (S(w, 0, 0, 1) - S(w)) * dzi
    p = S(f["p"])
    Dl = [D[l // 3][l % 3] for l in range(9)]
    vals = []
    add = vals.append
    for m in range(3):
        add(U[m])
    add(p)
    for m in range(3):
        add(G[m])
    for m in range(3):
        add(U[m] * p)
    for m in range(3):
        for n in range(m, 3):
            add(U[m] * U[n])
    for m in range(3):
        for n in range(m, 3):
            add(U[m] * G[n])
    for m in range(3):
        for n in range(m, 3):
            for h in range(n, 3):
                add(U[m] * U[n] * U[h])
    for m in range(3):
        for n in range(m, 3):
            for h in range(n, 3):
                add(U[m] * G[n] * U[h])
    for l in range(9):
        add(Dl[l])
    for l in range(9):
        add(Dl[l] * p)
    for l1 in range(9):
        for l2 in range(9):
            add(Dl[l1] * Dl[l2])
    zero = np.zeros_like(p)
    if thermal:
        h, T, R, MU, K = (f[n] for n in ("h", "t", "rho", "mu", "k"))

        def grad(a):
            return [(S(a, 1) - S(a, -1)) * dxi * 0.5,
                    ((S(a, 0, 1) - S(a)) * yc + (S(a) - S(a, 0, -1)) * yj) * 0.5,
                    (S(a, 0, 0, 1) - S(a, 0, 0, -1)) * dzi * 0.5]

        dh, dT = grad(h), grad(T)
        T, R, H, MU, K = S(T), S(R), S(h), S(MU), S(K)
        for a in (T, R, H, MU, T * T, R * R, H * H, H * R, H * p):
            add(a)
        for l in range(9):
            add(Dl[l] * MU)
        for l in range(9):
            add(Dl[l] * MU * H)
        for l in range(9):
            for m in range(3):
                add(Dl[l] * MU * U[m])
        for l1 in range(9):
            for l2 in range(9):
                add(Dl[l1] * Dl[l2] * MU)
        for m in range(3):
            add(H * U[m])
        for m in range(3):
            add(H * G[m])
        for m in range(3):
            for n in range(m, 3):
                add(R * H * U[m] * U[n])
        for m in range(3):
            add(dh[m])
        for m in range(3):
            add(dh[m] * p)
        for m in range(3):
            add(dT[m] * K)
        for m in range(3):
            for n in range(3):
                add(dT[m] * K * U[n])
        for m in range(3):
            for l in range(9):
                add(dT[m] * K * Dl[l])
        for m in range(3):
            for l in range(9):
                add(dh[m] * MU * Dl[l])
    else:
        vals += [zero] * 219
    return np.stack([a.sum(axis=(0, 2)) / (nx * nz) for a in vals], axis=1)


class IOCoupled(IO):
    """The coupled inflow / outflow section (TGFLOWFLG: non-periodic BCX_io),
    a numpy restatement written beside the C++ oracle's.  Arrays carry the x
    ghost columns: shape (nz, ny + 2, nx + 2), a[k-1, j, i] is F(i, j, k) for
    i = 0 .. NCL1_io + 1 (src/MEMALLOCT.f90:154-168); x neighbours do not wrap
    (src/INDEXSET.f90:25-32).  Per substep (src/SOLVE.f90:119-134 with
    src/SOLVERRK3_MOM_IO.f90:15-168 and src/SOLVERRK3_ENG_IO.f90:57-64):
    BC_TINLET_FLOW from the TG arrays set by set_inlet (src/BC_INLET.f90:2-51),
    BC_COUTLET_MOM_RK3 with CONVCTION_OUTLET_U and CHK_MassConsv_io
    (src/BC_COUTLET_MOM_RK3.f90:2-174, src/processing/CHK_conservation.f90:
    2-71), the x-momentum from the second face (NXI = 2) without the constant
    mass-flux forcing, MU_STG = 1 on the ghost faces, DIVG_io and
    FISHPACK_POIS3D_SIMPLE on the IO arrays with the x transform of BCX_io
    (here: the documented FFTPACK sums as dense matrices), PRCALC_io, and
    MASSFLUX_UPDATE_IO from the second face to the outlet face against
    DPH_io(NCL1_io + 1) = 0 (src/VELO_CORRECTION.f90:124-139); the energy
    substep adds BC_TINLET_THERML (src/BC_INLET.f90:54-76) and
    BC_COUTLET_ENEG_RK3 (src/BC_COUTLET_ENEG_RK3.f90:2-41).  The shared
    decisions: the initial outlet ghost column is a copy of the last interior
    column; the boundary operators' RK3 memory starts at zero."""

    LP = {(1, 1): 2, (1, 2): 3, (2, 2): 4, (2, 1): 5}

    def __init__(self, nx, ny, nz, lx, lz, bcx=(2, 1), **kw):
        super().__init__(nx, ny, nz, lx, lz, **kw)
        self._mesh = dict(nx=nx, ny=ny, nz=nz, lx=lx, lz=lz,
                          **{k: kw[k] for k in ("str2", "istr2", "ren", "dt") if k in kw})
        shape = (nz, ny + 2, nx + 2)
        z = lambda: np.zeros(shape)
        self.q = [None] + [z() for _ in range(3)]
        self.p, self.phi = z(), z()
        self.g = {c: z() for c in (1, 2, 3)}
        self.g0 = {c: z() for c in (1, 2, 3)}
        self.ex0 = {c: z() for c in (1, 2, 3)}
        self.drho, self.rhoh, self.h, self.rhse0 = z(), z(), z(), z()
        self.T, self.D, self.D0, self.mu, self.mu0, self.k = (np.ones(shape) for _ in range(6))
        self.lp = self.LP[tuple(bcx)]
        self.conv0 = {c: np.zeros((nz, ny + 2)) for c in (1, 2, 3)}
        self.conv0_eng = np.zeros((nz, ny + 2))
        self.tg = None
        self.bcs = {}

    def set_inlet(self, tu, tv, tw, tp):
        """The TG section's u, v, w, p, (nz, ny + 2, nx_tg)."""
        self.tg = [np.array(a, dtype=float) for a in (tu, tv, tw, tp)]

    # ---------------------------------------------------------- layout
    def X(self, a, di=0, dj=0, dk=0):
        b = np.roll(a, -dk, axis=0) if dk else a
        return b[:, 1 + dj:self.ny + 1 + dj, 1 + di:self.nx + 1 + di]

    def interior(self, a, val):
        a[:, 1:self.ny + 1, 1:self.nx + 1] = val

    def bc_vec(self, f):
        ny, c = self.ny, slice(1, self.nx + 1)
        f[1][:, 0, c] = 0.0; f[3][:, 0, c] = 0.0; f[2][:, 1, c] = 0.0; f[2][:, 0, c] = 0.0
        f[1][:, ny + 1, c] = 0.0; f[3][:, ny + 1, c] = 0.0; f[2][:, ny + 1, c] = 0.0

    def bc_copy(self, f):
        c = slice(1, self.nx + 1)
        f[:, 0, c] = f[:, 1, c]
        f[:, self.ny + 1, c] = f[:, self.ny, c]

    def mu_stg(self):
        """MU_Staggered on IC = 1..NCL1_io; the ghost faces keep 1."""
        ny, nx = self.ny, self.nx
        m, m0 = self.mu, self.mu0
        xm = lambda a: np.concatenate([np.zeros_like(a[..., :1]), a[..., :-1]], axis=2)
        zm = lambda a: np.roll(a, 1, axis=0)
        s1, s2, s3 = np.ones(m.shape), np.ones(m.shape), np.ones(m.shape)
        ex = m + xm(m) + m0 + xm(m0)
        ez = zm(m) + m + zm(m0) + m0
        wf, wb = self.wff[2:ny + 1][None, :, None], self.wfb[2:ny + 1][None, :, None]
        c = slice(1, nx + 1)
        s1[:, 2:ny + 1, c] = ((ex[:, 2:ny + 1] * wf + ex[:, 1:ny] * wb) * 0.25)[..., c]
        s3[:, 2:ny + 1, c] = ((ez[:, 2:ny + 1] * wf + ez[:, 1:ny] * wb) * 0.25)[..., c]
        s2[:, 1:ny + 1, c] = ((m + xm(m) + m0 + xm(m0) + zm(m) + zm(xm(m)) + zm(m0) + zm(xm(m0)))[:, 1:ny + 1] * 0.125)[..., c]
        for s in (s1, s3):
            s[:, 1, c] = 0.5 * (m0[:, 0, c] + m[:, 0, c])
            s[:, ny + 1, c] = 0.5 * (m0[:, ny + 1, c] + m[:, ny + 1, c])
        return s1, s2, s3

    def wall_thermal(self):
        """BC_WALL_THERMAL(IMAIND): the interior columns."""
        ny, c, h = self.ny, slice(1, self.nx + 1), self.h
        hb = 2.0 * h[:, 1, c] - self.wff[2] * h[:, 2, c] - self.wfb[2] * h[:, 1, c]
        ht = 2.0 * h[:, ny, c] - self.wff[ny] * h[:, ny, c] - self.wfb[ny] * h[:, ny - 1, c]
        for j, hg in ((0, hb), (ny + 1, ht)):
            T, D, M, K = self.table_props(hg)
            self.h[:, j, c], self.T[:, j, c], self.D[:, j, c], self.mu[:, j, c], self.k[:, j, c] = hg, T, D, M, K
            self.rhoh[:, j, c] = hg * D

    # ---------------------------------------------------------- boundary operators
    def u_outlet(self):
        """CONVCTION_OUTLET_U: (max + min) / 2 of 0.5 (u(NCL1) + u(NCL1 + 1))."""
        ny, nx = self.ny, self.nx
        ucc = 0.5 * (self.q[1][:, 1:ny + 1, nx] + self.q[1][:, 1:ny + 1, nx + 1])
        return 0.5 * (ucc.max() + ucc.min())

    def inlet(self):
        tu, tv, tw, tp = self.tg
        q, g = self.q, self.g
        q[1][:, :, 0], q[2][:, :, 0], q[3][:, :, 0] = tu[:, :, -1], tv[:, :, -1], tw[:, :, -1]
        g[1][:, :, 0], g[2][:, :, 0], g[3][:, :, 0] = tu[:, :, -1] * 1.0, tv[:, :, -1] * 1.0, tw[:, :, -1] * 1.0
        q[1][:, :, 1] = tu[:, :, 0]
        g[1][:, :, 1] = q[1][:, :, 1] * (1.0 + self.D[:, :, 1]) * 0.5
        self.p[:, :, 0] = tp[:, :, -1]
        self.D[:, :, 0] = 1.0

    def outlet_mom(self, ns):
        ny, nx = self.ny, self.nx
        U = self.u_outlet()
        coe1 = self.dxi * U
        rho = lambda: (self.D[:, :, nx] + self.D[:, :, nx + 1]) * 0.5
        for c in (1, 2, 3):
            j0 = 2 if c == 2 else 1
            go, gi = self.g[c][:, j0:ny + 1, nx + 1], self.g[c][:, j0:ny + 1, nx]
            conv = -(go - gi) * coe1
            rhs = TGAM[ns] * conv + TROH[ns] * self.conv0[c][:, j0:ny + 1]
            self.conv0[c][:, j0:ny + 1] = conv
            self.g[c][:, j0:ny + 1, nx + 1] = go + self.dt * rhs
            self.q[c][:, j0:ny + 1, nx + 1] = self.g[c][:, j0:ny + 1, nx + 1] / rho()[:, j0:ny + 1]
        w = 1.0 / self.dyfi[1:ny + 1][None, :]
        fin = np.sum(self.g[1][:, 1:ny + 1, 1] * w) / self.dzi
        fout = np.sum(self.g[1][:, 1:ny + 1, nx + 1] * w) / self.dzi
        mass = np.sum(self.X(self.drho) / self.row(self.dyfi)) / self.dzi / self.dxi
        scaling = (fin - mass) / fout
        self.bcs.update(u_outlet=U, scaling=scaling, inflow=fin, outflow=fout, mass_rate=mass)
        gn = self.g[1][:, 1:ny + 1, nx + 1]
        self.g[1][:, 1:ny + 1, nx + 1] = gn * (scaling - 1.0) + gn
        self.q[1][:, 1:ny + 1, nx + 1] = self.g[1][:, 1:ny + 1, nx + 1] / rho()[:, 1:ny + 1]
        for f in (self.g, self.q):  # BC_WALL_G_io / BC_WALL_Q_io on the outlet column
            f[1][:, 0, nx + 1] = 0.0; f[3][:, 0, nx + 1] = 0.0; f[2][:, 1, nx + 1] = 0.0; f[2][:, 0, nx + 1] = 0.0
            f[1][:, ny + 1, nx + 1] = 0.0; f[2][:, ny + 1, nx + 1] = 0.0; f[3][:, ny + 1, nx + 1] = 0.0

    def outlet_eng(self, ns):
        ny, nx = self.ny, self.nx
        U = self.u_outlet()
        rh = self.rhoh[:, 1:ny + 1, nx + 1]
        conv = -self.dxi * U * (rh - self.rhoh[:, 1:ny + 1, nx])
        rhs = TGAM[ns] * conv + TROH[ns] * self.conv0_eng[:, 1:ny + 1]
        self.conv0_eng[:, 1:ny + 1] = conv
        rh = rh + self.dt * rhs
        self.rhoh[:, 1:ny + 1, nx + 1] = rh
        D = self.td(self.ht(rh / self.D[:, 1:ny + 1, nx + 1]))
        h = rh / D
        T, D, M, K = self.table_props(h)
        for a, v in ((self.h, h), (self.T, T), (self.D, D), (self.mu, M), (self.k, K)):
            a[:, 1:ny + 1, nx + 1] = v
        hh = self.h[:, :, nx + 1]
        for j, hg in ((0, 2.0 * hh[:, 1] - self.wff[2] * hh[:, 2] - self.wfb[2] * hh[:, 1]),
                      (ny + 1, 2.0 * hh[:, ny] - self.wff[ny] * hh[:, ny] - self.wfb[ny] * hh[:, ny - 1])):
            T, D, M, K = self.table_props(hg)
            self.h[:, j, nx + 1], self.T[:, j, nx + 1], self.D[:, j, nx + 1] = hg, T, D
            self.mu[:, j, nx + 1], self.k[:, j, nx + 1], self.rhoh[:, j, nx + 1] = M, K, hg * D

    # ---------------------------------------------------------- substeps
    def eng(self, ns):
        super().eng(ns)
        for a, val in ((self.T, 1.0), (self.k, 1.0), (self.D, 1.0), (self.mu, 1.0), (self.rhoh, 0.0), (self.h, 0.0)):
            a[:, :, 0] = val  # BC_TINLET_THERML
        self.outlet_eng(ns)

    def prep(self, ns):
        if self.thermal:
            self.interior(self.drho, ((TGAM[ns] + TROH[ns]) * self.div(self.g) + TROH[ns] * self.div(self.g0)) /
                          (TGAM[ns] - 2.0))
        X, G, c = self.X, self.g, slice(1, self.nx + 1)
        rx, ry, rz = self.rho_stg()
        self.interior(self.q[1], X(G[1]) / rx)
        self.interior(self.q[3], X(G[3]) / rz)
        self.q[2][:, 2:self.ny + 1, c] = (X(G[2]) / ry)[:, 1:, :]
        self.bc_vec(self.q)

    def mom(self, ns):
        ny, nx, X, row = self.ny, self.nx, self.X, self.row
        self.g0 = {c: self.g[c].copy() for c in (1, 2, 3)}
        self.inlet()
        self.outlet_mom(ns)
        ex, ey, ez, _, _, _ = self.mom_terms()
        p, dt, alp, dxi, dzi, dycj = self.p, self.dt, TALP[ns], self.dxi, self.dzi, row(self.dyci)
        rx = (TGAM[ns] * ex + TROH[ns] * X(self.ex0[1])) * dt - (X(p) - X(p, -1)) * (alp * dt * dxi)
        ry = (TGAM[ns] * ey + TROH[ns] * X(self.ex0[2])) * dt - (X(p) - X(p, 0, -1)) * (alp * dt * dycj)
        rz = (TGAM[ns] * ez + TROH[ns] * X(self.ex0[3])) * dt - (X(p) - X(p, 0, 0, -1)) * (alp * dt * dzi)
        c, c2 = slice(1, nx + 1), slice(2, nx + 1)  # all faces, faces from the second (NXI = 2)
        self.ex0[1][:, 1:ny + 1, c2] = ex[:, :, 1:]
        self.ex0[3][:, 1:ny + 1, c] = ez
        self.ex0[2][:, 2:ny + 1, c] = ey[:, 1:, :]
        self.g[1][:, 1:ny + 1, c2] += rx[:, :, 1:]
        self.g[3][:, 1:ny + 1, c] += rz
        self.g[2][:, 2:ny + 1, c] += ry[:, 1:, :]
        self.bc_vec(self.g)
        self.project(ns)

    def project(self, ns):
        ny, nx, X, row = self.ny, self.nx, self.X, self.row
        p, dt, alp = self.p, self.dt, TALP[ns]
        rhs = (self.div(self.g) + X(self.drho)) / (dt * alp)
        self.phi[:] = 0.0
        self.interior(self.phi, self.poisson_io(rhs))
        self.bc_copy(self.phi)
        self.interior(p, X(p) + X(self.phi))
        self.bc_copy(p)
        f, c, c2 = self.phi, slice(1, nx + 1), slice(2, nx + 2)
        # x flux from the second face to the outlet face: f(i) - f(i - 1) with f(NCL1 + 1) = 0
        fx = f[:, 1:ny + 1, 1:nx + 2] - f[:, 1:ny + 1, 0:nx + 1]
        self.g[1][:, 1:ny + 1, c2] -= fx[:, :, 1:] * (dt * alp * self.dxi)
        self.g[3][:, 1:ny + 1, c] -= (X(f) - X(f, 0, 0, -1)) * (dt * alp * self.dzi)
        self.g[2][:, 2:ny + 1, c] -= ((X(f) - X(f, 0, -1)) * (dt * alp * row(self.dyci)))[:, 1:, :]
        self.bc_vec(self.g)

    def poisson_io(self, rhs):
        """FISHPACK_POIS3D_SIMPLE with the x transform of LP as the matrices of
        FFTPACK's documented sums, complex FFTs in z, banded y solves."""
        nx, ny, nz, lp = self.nx, self.ny, self.nz, self.lp
        n = nx
        i = np.arange(1, n + 1)[:, None]
        k = np.arange(1, n + 1)[None, :]
        lrdel = ((lp - 1) * (lp - 3) * (lp - 5)) // 3
        sc = n + lrdel
        di = {2: 0.0, 3: 0.5, 4: 1.0, 5: 0.5}[lp]
        xrt = -4.0 * self.dxi ** 2 * np.sin((np.arange(1, n + 1) - di) * np.pi / (2.0 * sc)) ** 2
        scalx = 4.0 * sc if lp in (3, 5) else 2.0 * sc
        sign = np.where((i - 1) % 2 == 1, -1.0, 1.0)
        if lp == 2:
            fw = 2.0 * np.sin(k * i * np.pi / (n + 1)); bw = fw
        elif lp == 3:
            fw = np.where(k == n, sign, 2.0 * np.sin((2.0 * i - 1.0) * k * np.pi / (2.0 * n)))
            bw = 4.0 * np.sin((2.0 * k - 1.0) * i * np.pi / (2.0 * n))
        elif lp == 4:
            fw = np.where(k == 1, 1.0, np.where(k == n, sign, 2.0 * np.cos((k - 1) * (i - 1) * np.pi / (n - 1)))); bw = fw
            xrt[0] = 0.0
        else:
            fw = np.where(k == 1, 1.0, 2.0 * np.cos((2.0 * i - 1.0) * (k - 1) * np.pi / (2.0 * n)))
            bw = 4.0 * np.cos((2.0 * k - 1.0) * (i - 1) * np.pi / (2.0 * n))
        X = np.einsum('ik,zjk->zji', fw, rhs)           # (kz, j, x-mode)
        F = np.fft.fft(X, axis=0)
        lam_z = -4.0 * self.dzi ** 2 * np.sin(np.pi * np.arange(nz) / nz) ** 2
        am, ac, ap = self.amph[1:ny + 1], self.acph[1:ny + 1], self.apph[1:ny + 1]
        out = np.zeros_like(F)
        ab = np.zeros((3, ny), dtype=complex)
        ab[0, 1:] = ap[:-1]
        ab[2, :-1] = am[1:]
        for a in range(nz):
            for b in range(nx):
                ab[1] = ac + xrt[b] + lam_z[a]
                if xrt[b] == 0.0 and a == 0:
                    out[a, :-1, b] = solve_banded((1, 1), ab[:, :-1], F[a, :-1, b])
                else:
                    out[a, :, b] = solve_banded((1, 1), ab, F[a, :, b])
        Y = np.real(np.fft.ifft(out, axis=0))
        return np.einsum('ik,zjk->zji', bw, Y) / (scalx * nz) * nz

    def init_random(self, seed, amp):
        """The x-periodic recipe on the interior (velocity, unit bulk mass
        flux), the outlet ghost column a copy of the last interior column, then
        the coupled NS = 0 projection."""
        base = IO(thermal=0, **self._mesh)
        TG.init_random(base, seed, amp)  # the TG velocity recipe on the interior layout
        ny, nx = self.ny, self.nx
        if self.thermal:
            T0, D0, M0, K0 = (float(x[0]) for x in self.table_props(np.array([0.0])))
        else:
            T0 = D0 = M0 = K0 = 1.0
        for a, val in ((self.T, T0), (self.D, D0), (self.D0, D0), (self.mu, M0), (self.mu0, M0), (self.k, K0)):
            a[:] = val
        for a in (self.h, self.rhoh, self.rhse0, self.drho, self.p, self.phi):
            a[:] = 0.0
        for c in (1, 2, 3):
            self.conv0[c][:] = 0.0
            self.g0[c][:] = 0.0
            self.ex0[c][:] = 0.0
        self.conv0_eng[:] = 0.0
        r_face = (D0 + D0 + D0 + D0) * 0.25
        r_v = (self.wff * (D0 + D0) + self.wfb * (D0 + D0)) * 0.5
        q = {c: base.q[c].copy() for c in (1, 2, 3)}

        def velo2massflux():
            g = {c: np.zeros_like(q[c]) for c in (1, 2, 3)}
            g[1][:, 1:ny + 1] = q[1][:, 1:ny + 1] * r_face
            g[3][:, 1:ny + 1] = q[3][:, 1:ny + 1] * r_face
            g[2][:, 2:ny + 1] = q[2][:, 2:ny + 1] * r_v[2:ny + 1][None, :, None]
            return g

        g = velo2massflux()
        gm = np.sum(g[1][:, 1:ny + 1] / self.row(self.dyfi)) / self.dzi / (self.area * nx)
        for c in (1, 2, 3):
            q[c] /= gm
        g = velo2massflux()
        for f in (q,):
            f[1][:, 0] = 0.0; f[3][:, 0] = 0.0; f[2][:, 1] = 0.0; f[2][:, 0] = 0.0
            f[1][:, ny + 1] = 0.0; f[3][:, ny + 1] = 0.0; f[2][:, ny + 1] = 0.0
        for c in (1, 2, 3):
            self.q[c][:] = 0.0
            self.g[c][:] = 0.0
            self.q[c][:, :, 1:nx + 1] = q[c]
            self.g[c][:, :, 1:nx + 1] = g[c]
            self.q[c][:, :, nx + 1] = q[c][:, :, nx - 1]
            self.g[c][:, :, nx + 1] = g[c][:, :, nx - 1]
        if self.thermal:
            self.wall_thermal()
            self.eng(0)
        self.mom(0)
