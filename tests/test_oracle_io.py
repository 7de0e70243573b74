"""CPU checks of the IO-section oracle against properties the reference's own
algorithm guarantees (no GPU): the FISHPACK Poisson solve inverts the
discrete Laplacian (CHECK_FFT_SOLVER's residual, src/PRESSURE_CORRECTION.f90:
159-202), the projection leaves div G + DrhoDtP at round-off (DIVGCK_io), the
constant-mass-flux forcing keeps the bulk mass flux, and one energy substep
changes the total rho h by exactly the iso-flux wall heat input (conservative
flux form of RHS_ENERGY_EXPLICIT)."""
import math
import os
import sys

import numpy as np
import pytest

from oracle.pyoracle import OracleIO, OracleTG, synth_table
from tests.conftest import relerr


def laplacian(o, phi, nx, ny, nz, lx, lz, str2=2.0):
    t = OracleTG(nx, ny, nz, lx=lx, lz=lz, str2=str2)
    am, ac, ap = (np.concatenate([[0.0], t.coef(w), [0.0]]) for w in (6, 7, 8))
    dxqi, dzqi = (nx / lx) ** 2, (nz / lz) ** 2
    f = phi[:, 1:ny + 1, :]
    lap = (np.roll(f, -1, 2) - 2 * f + np.roll(f, 1, 2)) * dxqi + (np.roll(f, -1, 0) - 2 * f + np.roll(f, 1, 0)) * dzqi
    lap += am[1:ny + 1, None] * phi[:, 0:ny, :] + ac[1:ny + 1, None] * f + ap[1:ny + 1, None] * phi[:, 2:ny + 2, :]
    return lap


@pytest.mark.parametrize("thermal", [0, 1])
def test_io_poisson_residual_and_projection(thermal):
    nx, ny, nz, lx, lz = 24, 16, 12, 8 * math.pi, 4 * math.pi / 3
    o = OracleIO(nx, ny, nz, lx=lx, lz=lz, thermal=thermal)
    o.init_random(4, 0.1)
    for ns in (1, 2):
        o.substep(ns)
        rhs = o.get("rhsphi")[:, 1:ny + 1, :]
        res = laplacian(o, o.get("phi"), nx, ny, nz, lx, lz) - rhs
        assert np.abs(res).max() <= 1e-10 * np.abs(rhs).max()
        assert o.divmax() < 1e-11
    # the mean mode is pinned at the last row (TRID0's zero branch)
    assert abs(o.get("phi")[:, ny, :].mean()) < 1e-12 * np.abs(o.get("phi")).max()
    assert abs(o.bulk(1) - 1.0) < 1e-12


def test_io_energy_substep_conserves_wall_heat_input():
    nx, ny, nz = 16, 12, 8
    qb, qt, ren, prt, dt = 0.7, 1.3, 2800.0, 0.71, 1e-3
    o = OracleIO(nx, ny, nz, qw=(qb, qt), ren=ren, prt=prt, dt=dt)
    o.init_random(6, 0.1)
    o.step(1)
    dyfi = 1.0 / np.diff(np.tanh(2.0 * (np.arange(ny + 1) / ny - 0.5)) / np.tanh(1.0))
    before = (o.get("rhoh")[:, 1:ny + 1, :] / dyfi[None, :, None]).sum()
    o.eng(1)  # gamma = 8/15, zeta = 0
    after = (o.get("rhoh")[:, 1:ny + 1, :] / dyfi[None, :, None]).sum()
    expect = (8.0 / 15.0) * dt * (qb + qt) / (ren * prt) * nx * nz
    assert abs((after - before) - expect) <= 1e-12 * abs(expect) + 1e-15 * abs(before)


def test_io_rhohmax_and_table_state():
    o = OracleIO(16, 12, 8)
    H, T, D = synth_table(4096)[:3]
    hs = H[0] + np.arange(1, 3 * 4096) * (H[-1] - H[0]) / (3 * 4096)
    # the spline maximum of D h sits next to the sampled table maximum
    assert abs(o.rhohmax() - (np.interp(hs, H, D) * hs).max()) < 1e-6
    o.init_random(1, 0.1)
    assert o.bad_cells() == 0
    h = o.get("h")
    assert np.all(np.abs(h[:, 1:-1, :]) < 1e-2)


GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
IO_GOLDEN = ["io_16x12x8_seed3", "io_heated_16x10x8_seed7", "io_si_16x12x8_seed3", "io_si_heated_16x10x8_seed7"]


def load_io_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = list(z["meta"]) + [0.0] * (15 - len(z["meta"]))  # visc_scheme defaults to explicit
    nx, ny, nz, lx, lz, ren, dt, seed, amp, steps, thermal, prt, qb, qt, visc = meta
    kw = dict(lx=lx, lz=lz, ren=ren, dt=dt, thermal=int(thermal), prt=prt, qw=(qb, qt), visc_scheme=int(visc))
    return z, (int(nx), int(ny), int(nz)), int(seed), amp, int(steps), kw


@pytest.mark.parametrize("name", IO_GOLDEN)
def test_oracle_io_matches_golden(name):
    """The C++ oracle against the fixtures of the independent numpy
    restatement (tests/golden/numpy_io.py), explicit and semi-implicit
    viscous schemes: FP64 within 1e-10 relative."""
    z, dims, seed, amp, steps, kw = load_io_golden(name)
    o = OracleIO(*dims, **kw)
    o.init_random(seed, amp)
    for n, key in (("gx", "ns0_gx"), ("gy", "ns0_gy"), ("p", "ns0_p")):
        assert relerr(o.get(n), z[key]) < 1e-10, n
    o.step(steps)
    names = [("gx", "end_gx"), ("gy", "end_gy"), ("gz", "end_gz"), ("p", "end_p"), ("u", "end_u"),
             ("ex0x", "end_ex0x")]
    if kw["thermal"]:
        names += [("h", "end_h"), ("rho", "end_rho"), ("mu", "end_mu"), ("rhse0", "end_rhse0")]
    for n, key in names:
        assert relerr(o.get(n), z[key]) < 1e-10, n
    assert o.divmax() < 1e-12 and float(z["end_divmax"]) < 1e-12
    assert abs(o.bulk(1) - float(z["end_bulk_g"])) < 1e-12
    assert o.bad_cells() == 0


def test_oracle_io_matches_numpy_restatement_heated():
    """A configuration outside the fixtures, run live through both CPU
    implementations: uniform y mesh, one RK3 step, unequal wall fluxes."""
    sys.path.insert(0, GOLDEN)
    from numpy_io import IO
    dims, lx, lz = (20, 14, 12), 2 * math.pi, math.pi
    n = IO(*dims, lx, lz, istr2=0, ren=1200.0, dt=1.5e-3, thermal=1, qw=(0.4, 1.1))
    o = OracleIO(*dims, lx=lx, lz=lz, istr2=0, ren=1200.0, dt=1.5e-3, thermal=1, qw=(0.4, 1.1))
    n.init_random(11, 0.15)
    o.init_random(11, 0.15)
    for ns in (1, 2, 3):
        n.substep(ns)
        o.substep(ns)
    for name, a in (("gx", n.g[1]), ("gy", n.g[2]), ("gz", n.g[3]), ("p", n.p), ("h", n.h), ("mu", n.mu),
                    ("ex0y", n.ex0[2])):
        assert relerr(o.get(name), a) < 1e-10, name


@pytest.mark.parametrize("thermal", [0, 1])
def test_oracle_io_semi_implicit_scheme(thermal):
    """visthemflg = 1 (VISCOUS_PAR_EXPLT_*_io + MOMFA_io): the projection keeps
    div G + DrhoDtP at round-off, and from the same settled state one step of
    the semi-implicit scheme differs from the explicit one by O(dt^2) (the
    Crank-Nicolson and explicit treatments of the viscous terms agree to
    first order; halving dt quarters the difference)."""
    diffs = []
    for dt in (1e-3, 5e-4):
        e = OracleIO(24, 16, 12, thermal=thermal, dt=1e-3, ren=500.0)
        i = OracleIO(24, 16, 12, thermal=thermal, dt=1e-3, ren=500.0)
        for o in (e, i):
            o.init_random(3, 0.2)
            o.step(2)  # settle the pressure left by projecting the seeded field
            o.set_dt(dt)
        i.set_scheme(1)
        e.step()
        i.step()
        assert i.divmax() < 1e-12 and i.bad_cells() == 0
        diffs.append(max(np.abs(e.get(n) - i.get(n)).max() for n in ("gx", "gy", "gz")))
    assert 3.5 < diffs[0] / diffs[1] < 4.5, diffs
    assert diffs[0] < 1e-6


IO_STAT_GROUPS = (("U1", 4), ("G1", 3), ("UP", 3), ("U2", 6), ("UG", 6), ("U3", 10), ("UGU", 10), ("DVDL1", 9),
                  ("DVDLP", 9), ("DVDL2", 81), ("T1", 1), ("D1", 1), ("H1", 1), ("M1", 1), ("T2", 1), ("D2", 1),
                  ("H2", 1), ("DH", 1), ("PH", 1), ("DVDL1M", 9), ("DVDL1MH", 9), ("DVDL1MU", 27), ("DVDL2M", 81),
                  ("UH", 3), ("GH", 3), ("U2DH", 6), ("DhDL1", 3), ("DhDLP", 3), ("DTDLK", 3), ("DTDLKU", 9),
                  ("DTDLKDVDL", 27), ("DHDLMDVDL", 27))


@pytest.mark.parametrize("thermal", [0, 1])
def test_oracle_io_statistics_match_numpy_restatement(thermal):
    """PP_MEAN_ZX_FLOW_Xperiodic_IO: the oracle's loop restatement against the
    numpy whole-array restatement on the oracle's own fields after one RK3
    step, 1e-12 per statistic group (relative to the group's largest value);
    without the energy equation the thermal groups are zero."""
    sys.path.insert(0, GOLDEN)
    from numpy_io import IO, io_stats
    dims = (20, 14, 12)
    o = OracleIO(*dims, thermal=thermal)
    o.init_random(6, 0.15)
    o.step(1)
    n = IO(*dims, 8 * math.pi, 4 * math.pi / 3)
    names = ("u", "v", "w", "p", "gx", "gy", "gz") + (("h", "t", "rho", "mu", "k") if thermal else ())
    b = io_stats({f: o.get(f) for f in names}, n.dxi, n.dzi, n.dyfi, n.dyci, thermal)
    a = o.stats()
    assert a.shape == b.shape == (dims[1], 360)
    lo = 0
    for name, width in IO_STAT_GROUPS:
        x, y = a[:, lo:lo + width], b[:, lo:lo + width]
        lo += width
        if not thermal and lo > 141:
            assert not np.any(x), name
            continue
        assert np.abs(x - y).max() <= 1e-12 * max(np.abs(y).max(), 1e-300), name
    assert lo == 360
    # DVDL2 is symmetric in (m,h) <-> (n,p)
    d2 = a[:, 60:141].reshape(-1, 9, 9)
    assert np.allclose(d2, np.transpose(d2, (0, 2, 1)), rtol=0, atol=1e-14 * np.abs(d2).max())


@pytest.mark.parametrize("walls", [3, 1, 2])
def test_oracle_io_isothermal_walls_match_numpy_restatement(walls):
    """BCWALLHEAT = isoThermalWall (BC_WALL_ISOTHERMAL, WALL_ISOTHERMAL_GIVEN
    and the wall rows of RHS_ENERGY_EXPLICIT) on both walls or one: the
    oracle against the numpy restatement after one RK3 step, FP64 within
    1e-10; the ghost rows hold the wall values; a wall hotter than the fluid
    heats the first row and a colder one cools it."""
    sys.path.insert(0, GOLDEN)
    from numpy_io import IO
    dims, lx, lz, tw = (20, 14, 12), 2 * math.pi, math.pi, (0.95, 0.80)
    n = IO(*dims, lx, lz, istr2=0, ren=1200.0, dt=1.5e-3, thermal=1, qw=tw, isothermal=walls)
    o = OracleIO(*dims, lx=lx, lz=lz, istr2=0, ren=1200.0, dt=1.5e-3, thermal=1, qw=tw, isothermal=walls)
    n.init_random(11, 0.15)
    o.init_random(11, 0.15)
    h0 = o.get("h")
    for ns in (1, 2, 3):
        n.substep(ns)
        o.substep(ns)
    for name, a in (("gx", n.g[1]), ("gy", n.g[2]), ("p", n.p), ("h", n.h), ("t", n.T), ("mu", n.mu),
                    ("rho", n.D)):
        assert relerr(o.get(name), a) < 1e-10, name
    T, h = o.get("t"), o.get("h")
    ny = dims[1]
    for side, j, jin in ((0, 0, 1), (1, ny + 1, ny)):
        if walls & (1 << side):
            assert np.all(T[:, j, :] == tw[side])
            # T(h = 0) of the table is about 0.867: 0.95 heats, 0.80 cools
            dh = h[:, jin, :].mean() - h0[:, jin, :].mean()
            assert (dh > 0) if tw[side] > 0.867 else (dh < 0), (side, dh)
    assert o.divmax() < 1e-11


@pytest.mark.parametrize("bcx", [(1, 1), (1, 2), (2, 2), (2, 1)])
def test_io_poisson_nonperiodic_x_inverts_the_operator(bcx):
    """FISHPACK_POIS3D_SIMPLE with non-periodic x (BCX_io Dirichlet 1 /
    Neumann 2 at inlet / outlet: FISHPACK's SINT, SINQ, COST, COSQ transforms,
    src/possion3d_fishpack_reform.f90:104-163 and FFTPACK's definitions): the
    solution satisfies the discrete Poisson equation whose x-ends follow the
    transform's basis (Dirichlet: zero one node beyond; Neumann: even about
    the end node), periodic z and the y-operator of TDMA_PHI_COEF, to 1e-10 of
    the right-hand side.  Neumann at both ends is singular in its mean mode;
    TRID0 pins that mode at the last row, whose equation is then left out.
    The section's fields carry the x ghost columns (the coupled layout);
    the solve reads and writes the interior columns."""
    nx, ny, nz, lx, lz = 20, 16, 12, 8 * math.pi, 4 * math.pi / 3
    o = OracleIO(nx, ny, nz, lx=lx, lz=lz, thermal=0)
    o.set_bcx(*bcx)
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal((nz, ny + 2, nx + 2))
    o.set("rhsphi", rhs)
    o.pois3d()
    phi = o.get("phi")
    assert not phi[..., 0].any() and not phi[..., -1].any()  # ghost columns untouched
    phi, rhs = phi[..., 1:nx + 1], rhs[..., 1:nx + 1]
    t = OracleTG(nx, ny, nz, lx=lx, lz=lz)
    am, ac, ap = (np.concatenate([[0.0], t.coef(w), [0.0]]) for w in (6, 7, 8))
    dxqi, dzqi = (nx / lx) ** 2, (nz / lz) ** 2
    f = phi[:, 1:ny + 1, :]
    zero = np.zeros_like(f[..., :1])
    left = zero if bcx[0] == 1 else f[..., 1:2]    # Dirichlet: phi_0 = 0; Neumann: phi_0 = phi_2
    right = zero if bcx[1] == 1 else f[..., -2:-1]  # phi_{N+1} = 0, or phi_{N+1} = phi_{N-1}
    fx = np.concatenate([left, f, right], axis=2)
    lap = (fx[..., 2:] - 2 * f + fx[..., :-2]) * dxqi + (np.roll(f, -1, 0) - 2 * f + np.roll(f, 1, 0)) * dzqi
    lap += am[1:ny + 1, None] * phi[:, 0:ny, :] + ac[1:ny + 1, None] * f + ap[1:ny + 1, None] * phi[:, 2:ny + 2, :]
    res = lap - rhs[:, 1:ny + 1, :]
    rows = ny - 1 if bcx == (2, 2) else ny
    assert np.abs(res[:, :rows, :]).max() <= 1e-10 * np.abs(rhs).max(), np.abs(res[:, :rows, :]).max()


@pytest.mark.parametrize("lp", [3, 5])
@pytest.mark.parametrize("n", [96, 128, 192])
def test_quarter_wave_transforms_fast_route_matches_the_sums(lp, n):
    """SINQF / SINQB (LP 3) and COSQF / COSQB (LP 5) through the N-point DFT
    (the route the oracle takes on lines longer than 64 and the library on
    every line) against FFTPACK's documented sums, to round-off; forward then
    backward returns 4 N times the input."""
    from oracle.pyoracle import load
    L = load()
    rng = np.random.default_rng(n + lp)
    x = rng.standard_normal(n)
    for fwd in (1, 0):
        a, b = x.copy(), x.copy()
        assert L.oracle_fftpack_real(lp, fwd, n, a.ctypes.data, 0) == 0
        assert L.oracle_fftpack_real(lp, fwd, n, b.ctypes.data, 1) == 0
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), (fwd, np.abs(a - b).max())
    y = x.copy()
    assert L.oracle_fftpack_real(lp, 1, n, y.ctypes.data, 1) == 0
    assert L.oracle_fftpack_real(lp, 0, n, y.ctypes.data, 1) == 0
    assert np.abs(y / (4 * n) - x).max() <= 1e-12
