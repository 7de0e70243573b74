"""CPU checks of the oracle's restatement of the coupled inflow/outflow
boundary operators of the IO section (BC_TINLET_FLOW, BC_COUTLET_MOM_RK3
with CHK_MassConsv_io, BC_COUTLET_ENEG_RK3) against a second restatement in
numpy, and the mass balance the outlet rescaling closes.  The reference ships
no tests or golden data for these routines, so they are pinned against the
reference's source lines only (src/BC_INLET.f90:2-76,
src/BC_COUTLET_MOM_RK3.f90:2-174, src/processing/CHK_conservation.f90:2-71,
src/BC_COUTLET_ENEG_RK3.f90:2-41)."""
import math

import numpy as np

from oracle.pyoracle import OracleIO, OracleTG

GAM = (1.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
ZETA = (0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0)
NY, NZ = 12, 8
LX_IO, LZ = 8 * math.pi, 4 * math.pi / 3


def _pair(thermal=1, table=None):
    t = OracleTG(16, NY, NZ, lz=LZ)
    t.init_random(3, 0.1)
    t.substep(0)
    o = OracleIO(24, NY, NZ, lx=LX_IO, lz=LZ, thermal=thermal, table=table)
    o.init_random(5, 0.1)
    return t, o


def _mesh():
    t = OracleTG(16, NY, NZ, lz=LZ)
    dyfi = t.coef(2)  # DYFI(1:ny)
    return dyfi, NZ / LZ, 24 / LX_IO


def test_inlet_copies_tg_planes():
    t, o = _pair()
    tu, tv, tw, tp = (t.get(n) for n in ("u", "v", "w", "p"))
    d1 = o.get("rho")[:, :, 0]
    o.bc_tinlet_flow(tu, tv, tw, tp)
    assert np.array_equal(o.get_plane("in_u"), tu[:, :, -1])
    assert np.array_equal(o.get_plane("in_v"), tv[:, :, -1])
    assert np.array_equal(o.get_plane("in_w"), tw[:, :, -1])
    assert np.array_equal(o.get_plane("in_p"), tp[:, :, -1])
    assert np.array_equal(o.get_plane("in_rho"), np.ones((NZ, NY + 2)))
    assert np.array_equal(o.get_plane("in_gx"), tu[:, :, -1])  # u * rho(0) with rho(0) = 1
    assert np.array_equal(o.get("u")[:, :, 0], tu[:, :, 0])
    assert np.array_equal(o.get("gx")[:, :, 0], tu[:, :, 0] * (1.0 + d1) * 0.5)


def test_outlet_momentum_matches_numpy_and_closes_the_mass_balance():
    t, o = _pair()
    rng = np.random.default_rng(7)
    dyfi, dzi, dxi = _mesh()
    # a state with a non-zero density history and outlet planes near the interior
    drho = 1e-3 * rng.standard_normal(o.shape)
    o.set("drho", drho)
    u, gx, gy, gz, rho = (o.get(n) for n in ("u", "gx", "gy", "gz", "rho"))
    planes = {}
    for name, base in (("out_u", u), ("out_gx", gx), ("out_gy", gy), ("out_gz", gz), ("out_rho", rho)):
        planes[name] = base[:, :, -1] * (1.0 + 0.05 * rng.standard_normal((NZ, NY + 2)))
        o.set_plane(name, planes[name])
    conv0 = {c: np.zeros((NZ, NY + 2)) for c in "xyz"}
    gout = {"x": planes["out_gx"].copy(), "y": planes["out_gy"].copy(), "z": planes["out_gz"].copy()}
    uout = planes["out_u"].copy()
    dt = 1e-3
    for ns in (1, 2, 3):
        o.bc_coutlet_mom_rk3(ns)
        # numpy restatement
        ucc = (u[:, 1:NY + 1, -1] + uout[:, 1:NY + 1]) * 0.5
        U = 0.5 * (ucc.max() + ucc.min())
        rho_f = (rho[:, :, -1] + planes["out_rho"]) * 0.5
        for c, g in (("x", gx), ("y", gy), ("z", gz)):
            j0 = 2 if c == "y" else 1
            sl = (slice(None), slice(j0, NY + 1))
            conv = -(gout[c][sl] - g[:, j0:NY + 1, -1]) * dxi * U
            rhs = GAM[ns] * conv + ZETA[ns] * conv0[c][sl]
            conv0[c][sl] = conv
            gout[c][sl] = gout[c][sl] + dt * rhs
        fin = (gx[:, 1:NY + 1, 0] / dyfi[None, :]).sum() / dzi
        fout = (gout["x"][:, 1:NY + 1] / dyfi[None, :]).sum() / dzi
        mass = (drho[:, 1:NY + 1, :] / dyfi[None, :, None]).sum() / dzi / dxi
        s = (fin - mass) / fout
        gout["x"][:, 1:NY + 1] = gout["x"][:, 1:NY + 1] * (s - 1.0) + gout["x"][:, 1:NY + 1]
        for c in "xyz":
            gout[c][:, 0] = 0.0
            gout[c][:, NY + 1] = 0.0
        gout["y"][:, 1] = 0.0
        uout = gout["x"] / rho_f
        uout[:, 0] = 0.0
        uout[:, NY + 1] = 0.0
        sc = o.bc_scalars()
        assert abs(sc["u_outlet"] - U) <= 1e-14 * abs(U)
        assert abs(sc["scaling"] - s) <= 1e-12
        for c in "xyz":
            a, b = o.get_plane(f"out_g{c}"), gout[c]
            assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), (ns, c)
            assert np.abs(o.get_plane(f"conv0_{c}") - conv0[c]).max() <= 1e-12 * max(np.abs(conv0[c]).max(), 1e-300)
        assert np.abs(o.get_plane("out_u") - uout).max() <= 1e-12 * np.abs(uout).max()
        # the rescaled outflow closes inflow - d(rho)/dt = outflow
        fout_new = (o.get_plane("out_gx")[:, 1:NY + 1] / dyfi[None, :]).sum() / dzi
        assert abs(fin - mass - fout_new) <= 1e-12 * abs(fin)


def test_outlet_energy_constant_table():
    """Constant properties (rho = mu = k = 1, T = h): the outlet rho h update
    and the isoflux ghost rows against numpy."""
    H = np.linspace(-1.0, 1.0, 4096)
    one = np.ones_like(H)
    table = (H, H.copy(), one, one.copy(), one.copy())
    t, o = _pair(thermal=1, table=table)
    rng = np.random.default_rng(11)
    dyfi, dzi, dxi = _mesh()
    rhoh = 0.1 * rng.standard_normal(o.shape)
    o.set("rhoh", rhoh)
    o.set_plane("out_rhoh", 0.1 * rng.standard_normal((NZ, NY + 2)))
    o.set_plane("out_rho", np.ones((NZ, NY + 2)))
    o.set_plane("out_u", o.get("u")[:, :, -1])
    u = o.get("u")
    rh = o.get_plane("out_rhoh")
    c0 = np.zeros((NZ, NY + 2))
    t2 = OracleTG(16, NY, NZ, lz=LZ)
    wff, wfb = t2.coef(4), t2.coef(5)  # YCL2ND_WFF/WFB(1:ny+1)
    dt = 1e-3
    for ns in (1, 2, 3):
        o.bc_coutlet_eneg_rk3(ns)
        ucc = (u[:, 1:NY + 1, -1] + o.get_plane("out_u")[:, 1:NY + 1]) * 0.5
        U = 0.5 * (ucc.max() + ucc.min())
        conv = -dxi * U * (rh[:, 1:NY + 1] - rhoh[:, 1:NY + 1, -1])
        rhs = GAM[ns] * conv + ZETA[ns] * c0[:, 1:NY + 1]
        c0[:, 1:NY + 1] = conv
        rh[:, 1:NY + 1] = rh[:, 1:NY + 1] + dt * rhs
        h = rh.copy()  # rho = 1
        h[:, 0] = 2.0 * h[:, 1] - wff[1] * h[:, 2] - wfb[1] * h[:, 1]
        h[:, NY + 1] = 2.0 * h[:, NY] - wff[NY - 1] * h[:, NY] - wfb[NY - 1] * h[:, NY - 1]
        rh[:, 0], rh[:, NY + 1] = h[:, 0], h[:, NY + 1]
        assert abs(o.bc_scalars()["u_outlet_eng"] - U) <= 1e-14 * abs(U)
        assert np.abs(o.get_plane("out_rhoh") - rh).max() <= 1e-14
        assert np.abs(o.get_plane("out_h") - h).max() <= 1e-14
        assert np.abs(o.get_plane("out_t") - h).max() <= 1e-14
        assert np.abs(o.get_plane("conv0_eng") - c0).max() <= 1e-14
