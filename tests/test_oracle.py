"""CPU tests of the FP64 oracle (the checker): agreement with the golden
fixtures of the independent numpy restatement, and the reference's own
self-checks restated as assertions."""
import math
import os
import sys

import numpy as np
import pytest

from tests.conftest import relerr

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN)


@pytest.fixture(scope="module")
def ora():
    from oracle import pyoracle
    pyoracle.load()
    return pyoracle


@pytest.mark.parametrize("name", ["tg_16x12x8_seed0", "tg_24x16x12_seed5"])
def test_oracle_matches_golden(ora, name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    nx, ny, nz, lx, lz, ren, dt, seed, amp, steps = z["meta"]
    o = ora.OracleTG(int(nx), int(ny), int(nz), lx=lx, lz=lz, ren=ren, dt=dt)
    o.init_random(int(seed), amp)
    for n in ("u", "v", "w"):
        assert relerr(o.get(n), z["init_" + n]) < 1e-14
    o.substep(0)
    for n in ("u", "v", "w", "p"):
        assert relerr(o.get(n), z["ns0_" + n]) < 1e-10, n
    o.step(int(steps))
    for n in ("u", "v", "w", "p"):
        assert relerr(o.get(n), z["end_" + n]) < 1e-10, n
    for n in ("h0u", "h0v", "h0w"):
        assert relerr(o.get(n)[:, 1:-1, :], z["end_" + n][:, 1:-1, :]) < 1e-10, n
    assert abs(o.divmax() - float(z["end_divmax"])) < 1e-13


def test_projection_divergence_free(ora):
    """DIVGCK after every substep (src/DIVGCK.f90:16-58) is at round-off."""
    o = ora.OracleTG(24, 16, 12)
    o.init_random(3, 0.1)
    assert o.divmax() > 1e-3
    o.substep(0)
    assert o.divmax() < 1e-12
    for _ in range(2):
        o.step()
        assert o.divmax() < 1e-12


def test_poisson_residual(ora):
    """CHECK_FFT_SOLVER (src/PRESSURE_CORRECTION.f90:159-202): |L phi - rhs|."""
    o = ora.OracleTG(32, 24, 16)
    rng = np.random.default_rng(0)
    rhs = np.zeros(o.shape)
    rhs[:, 1:-1, :] = rng.standard_normal((16, 24, 32))
    o.set("rhsphi", rhs)
    o.pois3d()
    assert o.pois_residual() < 1e-9 * np.abs(rhs).max()


def test_analytic_poisson(ora):
    """TEST_POISSON (src/SOLVERRK3_MOM_IO.f90:171-202): rhs = -4 sin x cos x."""
    nx, ny, nz, lx = 64, 16, 8, 4 * math.pi
    o = ora.OracleTG(nx, ny, nz, lx=lx)
    x = (np.arange(nx) + 0.5) * lx / nx
    rhs = np.zeros(o.shape)
    rhs[:, 1:-1, :] = (-4.0 * np.sin(x) * np.cos(x))[None, None, :]
    o.set("rhsphi", rhs)
    o.pois3d()
    m = round(lx / math.pi)
    ak1 = 2.0 * (1.0 - math.cos(2.0 * math.pi * m / nx)) * (nx / lx) ** 2
    exact = 2.0 * np.sin(2.0 * x) / ak1
    assert np.abs(o.get("phi")[:, 1:-1, :] - exact[None, None, :]).max() < 1e-12


def test_constant_bulk_velocity(ora):
    """Constant mass flux (FLOWDRVTP = 1, src/RHS_CvLpGpS_tg.f90:183-198)."""
    o = ora.OracleTG(32, 24, 16)
    o.init_random(1, 0.1)
    o.substep(0)
    for _ in range(5):
        o.step()
    assert abs(o.bulk() - 1.0) < 1e-9


def test_laminar_poiseuille_steady(ora):
    """u = 1.5(1-y^2) (LAMPOISLPROF.f90:49-56) stays steady under constant mass
    flux; the remaining drift is discretisation error of the stretched grid."""
    o = ora.OracleTG(16, 32, 8)
    o.init_poiseuille()
    u0 = o.get("u")
    for _ in range(10):
        o.step()
    u1 = o.get("u")
    assert np.abs(u1 - u0).max() < 1e-4
    assert np.abs(o.get("v")).max() < 1e-12
    assert o.divmax() < 1e-13


def test_mesh_and_coefficients(ora):
    """COORDJR / TDMA_COEF identities (src/COORDJR.f90:27-143,427-490,
    src/TDMA_COEF.f90:53-119)."""
    o = ora.OracleTG(16, 20, 8)
    ynd = o.coef(0)
    assert abs(ynd[0] + 1) < 1e-15 and abs(ynd[-1] - 1) < 1e-15
    assert np.all(np.diff(ynd) > 0)
    wff, wfb = o.coef(4), o.coef(5)
    assert np.allclose(wff + wfb, 1.0, atol=1e-14)
    amph, acph, apph = o.coef(6), o.coef(7), o.coef(8)
    assert np.allclose(amph + acph + apph, 0.0, atol=1e-9)  # Neumann rows sum to zero
    assert amph[0] == 0 and apph[-1] == 0
    dyfi = o.coef(2)
    assert abs(np.sum(1.0 / dyfi) - 2.0) < 1e-13
    assert abs(o.L.oracle_tg_volm(o.h) - 16 * 8 * 2.0) < 1e-10


def test_cyclic_and_noncyclic_tdma_against_dense(ora):
    """Substep increments of a one-component problem equal a dense solve: the
    x, z, y Crank-Nicolson factors of MOMFA_tg (src/MOMFA_tg.f90:17-240)
    compared with numpy on the same right-hand side through the numpy
    restatement, which uses circulant FFT and banded LU solves."""
    from numpy_tg import TG
    o = ora.OracleTG(12, 10, 8, lx=1.0, lz=1.0, ren=10.0, dt=0.01)
    t = TG(12, 10, 8, 1.0, 1.0, ren=10.0, dt=0.01)
    o.init_random(4, 0.2)
    t.init_random(4, 0.2)
    for ns in (0, 1, 2, 3):
        o.substep(ns)
        t.substep(ns)
    for n, a in (("u", t.q[1]), ("v", t.q[2]), ("w", t.q[3]), ("p", t.p)):
        assert relerr(o.get(n), a) < 1e-11, n


def test_oracle_rejects_bad_config(ora):
    with pytest.raises(ValueError):
        ora.OracleTG(7, 8, 8)
