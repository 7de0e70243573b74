"""CPU checks of the IO-section oracle against properties the reference's own
algorithm guarantees (no GPU): the FISHPACK Poisson solve inverts the
discrete Laplacian (CHECK_FFT_SOLVER's residual, src/PRESSURE_CORRECTION.f90:
159-202), the projection leaves div G + DrhoDtP at round-off (DIVGCK_io), the
constant-mass-flux forcing keeps the bulk mass flux, and one energy substep
changes the total rho h by exactly the iso-flux wall heat input (conservative
flux form of RHS_ENERGY_EXPLICIT)."""
import math

import numpy as np
import pytest

from oracle.pyoracle import OracleIO, OracleTG, synth_table


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
