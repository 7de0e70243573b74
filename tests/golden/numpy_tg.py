"""Independent numpy restatement of CHAPSim's TG RK3 substep.

Test infrastructure only.  It exists to cross-check the C++ oracle with a
second implementation that uses different algorithms for every solve:
the cyclic Crank-Nicolson factors (reference: TDMAIJI_CYC, a two-sweep
elimination) are solved here as circulant systems by FFT, the non-cyclic
y-factors and the Poisson y-lines (reference: TDMAIJJ_nonCYC Thomas sweeps)
by scipy's banded LU, and the x/z transforms by numpy.fft.

Arrays are numpy views of the reference's Fortran layout F(1:nx, 0:ny+1, 1:nz):
shape (nz, ny+2, nx) in C order, so a[k-1, j, i-1] is F(i, j, k).

Reference files restated (paths relative to the CHAPSim1WW project root):
src/COORDJR.f90:27-143,427-450; src/TDMA_COEF.f90:53-119;
src/CONVECTION_X.f90:23-74; src/CONVECTION_Y.f90:22-91;
src/CONVECTION_Z.f90:22-75; src/RHS_CvLpGpS_tg.f90:29-213;
src/MOMFA_tg.f90:17-240; src/DIVG.f90:21-57;
src/possion3d_FFT99.f90:155-220,254-488; src/VELO_CORRECTION.f90:19-105;
src/PRESSURE_CORRECTION.f90:1-24; src/BC_WALL.f90:204-408.
"""
import numpy as np
from scipy.linalg import solve_banded

TGAM = np.array([1.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0])
TROH = np.array([0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0])
TALP = TGAM + TROH


def splitmix64(x):
    m = (1 << 64) - 1
    x = (x + 0x9E3779B97F4A7C15) & m
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
    return x ^ (x >> 31)


def splitmix64_np(x):
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def rnd_pm1(seed, comp, nx, ny, nz):
    """Uniform [-1,1) draws keyed by (seed, comp, i, j, k); shape (nz, ny, nx)."""
    k, j, i = np.meshgrid(np.arange(1, nz + 1, dtype=np.uint64), np.arange(1, ny + 1, dtype=np.uint64),
                          np.arange(1, nx + 1, dtype=np.uint64), indexing="ij")
    ctr = (np.uint64(comp) << np.uint64(60)) ^ (k << np.uint64(40)) ^ (j << np.uint64(20)) ^ i
    with np.errstate(over="ignore"):
        x = splitmix64_np(np.uint64(splitmix64(int(seed))) ^ ctr)
    u = (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return -1.0 + 2.0 * u


class TG:
    def __init__(self, nx, ny, nz, lx, lz, str2=2.0, istr2=1, ren=2800.0, dt=1e-3, flowdrvtp=1, cfgv=0.0):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.ren, self.dt, self.flowdrvtp, self.cfgv = ren, dt, flowdrvtp, cfgv
        self.dxi = nx / lx
        self.dzi = nz / lz
        nnd2 = ny + 1
        jn = np.arange(1, nnd2 + 1)
        if istr2 == 1:
            ynd = np.tanh(str2 * ((jn - 1) / (nnd2 - 1) - 0.5)) / np.tanh(str2 * 0.5)
            ycc = np.tanh(str2 * ((np.arange(1, ny + 1) - 0.5) / (nnd2 - 1) - 0.5)) / np.tanh(str2 * 0.5)
        else:
            ynd = -1.0 + (jn - 1) * (2.0 / ny)
            ycc = 0.5 * (ynd[:-1] + ynd[1:])
        # 1-based arrays padded to index 0..ny+1
        pad = lambda a, lo: np.concatenate([np.zeros(lo), a, np.zeros(ny + 2 - lo - len(a))])
        self.ynd = pad(ynd, 1)
        self.ycc = pad(ycc, 1)
        self.dyfi = pad(1.0 / np.diff(ynd), 1)
        dyci = np.zeros(ny + 2)
        dyci[2:nnd2] = 1.0 / (0.5 * (self.ynd[3:nnd2 + 1] - self.ynd[1:nnd2 - 1]))
        dyci[1] = 2.0 / (self.ynd[2] - self.ynd[1])
        dyci[nnd2] = 2.0 / (self.ynd[nnd2] - self.ynd[ny])
        self.dyci = dyci
        wff = np.zeros(ny + 2); wfb = np.zeros(ny + 2)
        jc = np.arange(2, ny + 1)
        wff[jc] = (self.ynd[jc] - self.ycc[jc - 1]) / (self.ycc[jc] - self.ycc[jc - 1])
        wfb[jc] = (self.ycc[jc] - self.ynd[jc]) / (self.ycc[jc] - self.ycc[jc - 1])
        wfb[1], wff[1], wfb[nnd2], wff[nnd2] = 1.0, 0.0, 0.0, 1.0
        self.wff, self.wfb = wff, wfb
        self.volm = nx * nz * np.sum(1.0 / self.dyfi[1:ny + 1])
        self.area = nz * np.sum(1.0 / self.dyfi[1:ny + 1]) / self.dzi
        # Poisson y-operator
        amph = np.zeros(ny + 2); apph = np.zeros(ny + 2)
        j = np.arange(1, ny + 1)
        amph[j] = self.dyfi[j] * self.dyci[j]
        apph[j] = self.dyfi[j] * self.dyci[j + 1]
        amph[1] *= 0.5
        apph[ny] *= 0.5
        acph = -(amph + apph)
        acph[1] += amph[1]; amph[1] = 0.0
        acph[ny] += apph[ny]; apph[ny] = 0.0
        self.amph, self.acph, self.apph = amph, acph, apph
        # viscous y-operators
        self.amvr = {}; self.acvr = {}; self.apvr = {}
        for idr in (1, 3):
            am = np.zeros(ny + 2); ac = np.zeros(ny + 2); ap = np.zeros(ny + 2)
            j = np.arange(2, ny)
            am[j] = self.dyfi[j] * self.dyci[j]
            ap[j] = self.dyfi[j] * self.dyci[j + 1]
            ac[j] = -(am[j] + ap[j])
            u = 4.0 / (2.0 / self.dyci[2] + 1.0 / self.dyfi[1])
            ap[1] = u * self.dyci[2]; ac[1] = -u * (self.dyci[2] + 2.0 * self.dyfi[1])
            u = 4.0 / (2.0 / self.dyci[ny] + 1.0 / self.dyfi[ny])
            am[ny] = u * self.dyci[ny]; ac[ny] = -u * (2.0 * self.dyfi[ny] + self.dyci[ny])
            self.amvr[idr], self.acvr[idr], self.apvr[idr] = am, ac, ap
        am = np.zeros(ny + 2); ac = np.zeros(ny + 2); ap = np.zeros(ny + 2)
        j = np.arange(2, ny + 1)
        am[j] = self.dyfi[j - 1] * self.dyci[j]
        ap[j] = self.dyfi[j] * self.dyci[j]
        ac[j] = -(am[j] + ap[j])
        ac[1] = 1.0; ac[nnd2] = 1.0
        self.amvr[2], self.acvr[2], self.apvr[2] = am, ac, ap
        kx = np.arange(nx // 2 + 1)
        self.ak1 = 2.0 * (1.0 - np.cos(2.0 * np.pi * kx / nx)) * self.dxi ** 2
        kz = np.arange(nz)
        self.ak3 = 2.0 * (1.0 - np.cos(2.0 * np.pi * kz / nz)) * self.dzi ** 2
        shp = (nz, ny + 2, nx)
        self.q = [None] + [np.zeros(shp) for _ in range(3)]
        self.p = np.zeros(shp)
        self.phi = np.zeros(shp)
        self.rhsphi = np.zeros(shp)
        self.h0 = [None] + [np.zeros(shp) for _ in range(3)]

    # ---- helpers (axis 2 = x, axis 0 = z, axis 1 = y with ghosts)
    @staticmethod
    def xp(a): return np.roll(a, -1, axis=2)
    @staticmethod
    def xm(a): return np.roll(a, 1, axis=2)
    @staticmethod
    def zp(a): return np.roll(a, -1, axis=0)
    @staticmethod
    def zm(a): return np.roll(a, 1, axis=0)

    def bc_q(self):
        ny = self.ny
        u, v, w = self.q[1], self.q[2], self.q[3]
        u[:, 0, :] = 0; w[:, 0, :] = 0; v[:, 1, :] = 0; v[:, 0, :] = 0
        u[:, ny + 1, :] = 0; w[:, ny + 1, :] = 0; v[:, ny + 1, :] = 0

    def bc_copy(self, f):
        f[:, 0, :] = f[:, 1, :]
        f[:, self.ny + 1, :] = f[:, self.ny, :]

    def convection(self):
        ny = self.ny
        u, v, w = self.q[1], self.q[2], self.q[3]
        J = slice(1, ny + 1); Jp = slice(2, ny + 2); Jm = slice(0, ny)
        Y = lambda a: a.reshape(1, -1, 1)
        wff_j, wfb_j = Y(self.wff[1:ny + 1]), Y(self.wfb[1:ny + 1])
        wff_p, wfb_p = Y(self.wff[2:ny + 2]), Y(self.wfb[2:ny + 2])
        dyfi = Y(self.dyfi[1:ny + 1])
        dxi, dzi = self.dxi, self.dzi
        uc, up_, um_ = u[:, J], self.xp(u)[:, J], self.xm(u)[:, J]
        h11 = ((up_ + uc) ** 2 - (um_ + uc) ** 2) * 0.25 * dxi
        vm = v + self.xm(v)
        h12 = (vm[:, Jp] * (wff_p * u[:, Jp] + wfb_p * u[:, J]) - vm[:, J] * (wff_j * u[:, J] + wfb_j * u[:, Jm])) * 0.5 * dyfi
        wxm = w + self.xm(w)
        h13 = (self.zp(wxm)[:, J] * (self.zp(u)[:, J] + uc) - wxm[:, J] * (uc + self.zm(u)[:, J])) * 0.25 * dzi
        H1 = np.zeros_like(u); H1[:, J] = -(h11 + h12 + h13)
        # y-momentum, faces j = 2..ny
        J2 = slice(2, ny + 1); J2m = slice(1, ny); J2p = slice(3, ny + 2)
        wf, wb = Y(self.wff[2:ny + 1]), Y(self.wfb[2:ny + 1])
        dyci = Y(self.dyci[2:ny + 1])
        ui = wf * u[:, J2] + wb * u[:, J2m]
        h21 = (self.xp(ui) * (self.xp(v)[:, J2] + v[:, J2]) - ui * (v[:, J2] + self.xm(v)[:, J2])) * 0.5 * dxi
        h22 = ((v[:, J2p] + v[:, J2]) ** 2 - (v[:, J2] + v[:, J2m]) ** 2) * 0.25 * dyci
        wi = wf * w[:, J2] + wb * w[:, J2m]
        h23 = (self.zp(wi) * (self.zp(v)[:, J2] + v[:, J2]) - wi * (v[:, J2] + self.zm(v)[:, J2])) * 0.5 * dzi
        H2 = np.zeros_like(u); H2[:, J2] = -(h21 + h22 + h23)
        # z-momentum
        uzm = u + self.zm(u)
        h31 = (self.xp(uzm)[:, J] * (self.xp(w)[:, J] + w[:, J]) - uzm[:, J] * (w[:, J] + self.xm(w)[:, J])) * 0.25 * dxi
        vzm = v + self.zm(v)
        h32 = (vzm[:, Jp] * (wff_p * w[:, Jp] + wfb_p * w[:, J]) - vzm[:, J] * (wff_j * w[:, J] + wfb_j * w[:, Jm])) * 0.5 * dyfi
        wc = w[:, J]
        h33 = ((self.zp(w)[:, J] + wc) ** 2 - (wc + self.zm(w)[:, J]) ** 2) * 0.25 * dzi
        H3 = np.zeros_like(u); H3[:, J] = -(h31 + h32 + h33)
        return [None, H1, H2, H3]

    def cyc_solve(self, r, beta_h2, axis):
        """(1 - beta delta) x = r, periodic along axis, by FFT (circulant)."""
        n = r.shape[axis]
        lam = 1.0 + 2.0 * beta_h2 * (1.0 - np.cos(2.0 * np.pi * np.arange(n) / n))
        shape = [1, 1, 1]; shape[axis] = n
        return np.real(np.fft.ifft(np.fft.fft(r, axis=axis) / lam.reshape(shape), axis=axis))

    def y_solve(self, a, b, c, r):
        """Tridiagonal along axis 1 (rows 0..m-1) for every (k, i) line."""
        m = len(b)
        ab = np.zeros((3, m))
        ab[0, 1:] = c[:-1]; ab[1] = b; ab[2, :-1] = a[1:]
        nz, _, nx = r.shape
        rr = np.transpose(r, (1, 0, 2)).reshape(m, -1)
        x = solve_banded((1, 1), ab, rr)
        return np.transpose(x.reshape(m, nz, nx), (1, 0, 2))

    def substep(self, ns):
        ny, dt = self.ny, self.dt
        H = self.convection()
        rhs = np.zeros_like(self.p)
        facoe = 0.5 * TALP[ns] * dt / self.ren
        Y = lambda a: a.reshape(1, -1, 1)
        for idr in (1, 2, 3):
            q = self.q[idr]
            j0 = 2 if idr == 2 else 1
            J = slice(j0, ny + 1); Jp = slice(j0 + 1, ny + 2); Jm = slice(j0 - 1, ny)
            lap = ((self.xp(q) - 2 * q + self.xm(q)) * self.dxi ** 2 + (self.zp(q) - 2 * q + self.zm(q)) * self.dzi ** 2)[:, J]
            lap = lap + q[:, Jp] * Y(self.apvr[idr][j0:ny + 1]) + q[:, J] * Y(self.acvr[idr][j0:ny + 1]) + q[:, Jm] * Y(self.amvr[idr][j0:ny + 1])
            r = dt * (TGAM[ns] * H[idr][:, J] + TROH[ns] * self.h0[idr][:, J] + TALP[ns] / self.ren * lap)
            self.h0[idr][:, J] = H[idr][:, J]
            p = self.p
            if idr == 1:
                gp = (p - self.xm(p))[:, J] * self.dxi
            elif idr == 2:
                gp = (p[:, J] - p[:, Jm]) * Y(self.dyci[j0:ny + 1])
            else:
                gp = (p - self.zm(p))[:, J] * self.dzi
            rhs[:, J] = r - TALP[ns] * dt * gp
            if idr == 1:
                if self.flowdrvtp == 1:
                    dp = np.sum(rhs[:, 1:ny + 1] / Y(self.dyfi[1:ny + 1])) / self.volm
                else:
                    dp = -0.5 * self.cfgv * TALP[ns] * dt
                rhs[:, J] -= dp
            rhs[:, J] = self.cyc_solve(rhs[:, J], facoe * self.dxi ** 2, 2)
            rhs[:, J] = self.cyc_solve(rhs[:, J], facoe * self.dzi ** 2, 0)
            jj = np.arange(1, ny + 1)
            a = -facoe * self.amvr[idr][jj]; b = 1.0 - facoe * self.acvr[idr][jj]; c = -facoe * self.apvr[idr][jj]
            rhs[:, 1:ny + 1] = self.y_solve(a, b, c, rhs[:, 1:ny + 1])
            q[:, J] += rhs[:, J]
        self.bc_q()
        # divergence -> Poisson rhs
        u, v, w = self.q[1], self.q[2], self.q[3]
        J = slice(1, ny + 1)
        d = ((self.xp(u) - u)[:, J] * self.dxi + (v[:, 2:ny + 2] - v[:, J]) * Y(self.dyfi[1:ny + 1]) + (self.zp(w) - w)[:, J] * self.dzi)
        self.rhsphi = np.zeros_like(self.p)
        self.rhsphi[:, J] = d / (dt * TALP[ns])
        self.phi = np.zeros_like(self.p)
        self.phi[:, J] = self.poisson(self.rhsphi[:, J])
        self.bc_copy(self.phi)
        phi = self.phi
        u[:, J] -= (phi - self.xm(phi))[:, J] * dt * TALP[ns] * self.dxi
        w[:, J] -= (phi - self.zm(phi))[:, J] * dt * TALP[ns] * self.dzi
        v[:, 2:ny + 1] -= (phi[:, 2:ny + 1] - phi[:, 1:ny]) * dt * TALP[ns] * Y(self.dyci[2:ny + 1])
        self.bc_q()
        be = 0.5 * TALP[ns] * dt / self.ren
        self.p[:, J] += phi[:, J] - be * self.rhsphi[:, J]
        self.bc_copy(self.p)

    def poisson(self, rhs):
        nz, ny, nx = rhs.shape
        s = np.fft.fft(np.fft.rfft(rhs, axis=2) / nx, axis=0) / nz  # (kz, j, kx)
        out = np.zeros_like(s)
        jj = np.arange(1, ny + 1)
        for kz in range(nz):
            for kx in range(nx // 2 + 1):
                a = self.amph[jj].copy(); c = self.apph[jj].copy()
                b = self.acph[jj] - self.ak1[kx] - self.ak3[kz]
                f = s[kz, :, kx].copy()
                if kx == 0 and kz == 0:
                    a[0] = 0.0; c[0] = 0.0; f[0] = 0.0
                ab = np.zeros((3, ny), dtype=complex)
                ab[0, 1:] = c[:-1]; ab[1] = b; ab[2, :-1] = a[1:]
                out[kz, :, kx] = solve_banded((1, 1), ab, f)
        g = np.fft.ifft(out, axis=0) * nz
        g[:, :, 0] = g[:, :, 0].real
        if nx % 2 == 0:
            g[:, :, nx // 2] = g[:, :, nx // 2].real
        return np.fft.irfft(g, n=nx, axis=2) * nx

    def bulk(self):
        ny = self.ny
        return np.sum(self.q[1][:, 1:ny + 1] / self.dyfi[1:ny + 1].reshape(1, -1, 1)) / self.dzi / (self.area * self.nx)

    def divmax(self):
        ny = self.ny
        u, v, w = self.q[1], self.q[2], self.q[3]
        J = slice(1, ny + 1)
        d = ((self.xp(u) - u)[:, J] * self.dxi + (v[:, 2:ny + 2] - v[:, J]) * self.dyfi[1:ny + 1].reshape(1, -1, 1) + (self.zp(w) - w)[:, J] * self.dzi)
        return np.abs(d).max()

    def init_random(self, seed, amp):
        nx, ny, nz = self.nx, self.ny, self.nz
        for c in (1, 2, 3):
            self.q[c][:] = 0.0
            self.q[c][:, 1:ny + 1, :] = amp * rnd_pm1(seed, c, nx, ny, nz)
        self.q[2][:, 1, :] = 0.0
        for c in (1, 2, 3):
            m = self.q[c][:, 1:ny + 1, :].mean(axis=(0, 2), keepdims=True)
            self.q[c][:, 1:ny + 1, :] -= m
        self.q[1][:, 1:ny + 1, :] += (1.5 * (1.0 - self.ycc[1:ny + 1] ** 2)).reshape(1, -1, 1)
        self.q[2][:, 1, :] = 0.0
        self.q[1] /= self.bulk()
        self.bc_q()
        self.p[:] = 0.0
        for c in (1, 2, 3):
            self.h0[c][:] = 0.0
