"""GPU parity of the coupled inflow/outflow boundary operators of the IO
section (BC_TINLET_FLOW + BC_TINLET_THERML, BC_COUTLET_MOM_RK3 with
CHK_MassConsv_io, BC_COUTLET_ENEG_RK3) against the oracle's restatement,
through the C ABI.  Both sides start from the same state: the fields the
operators read are copied from the library into the oracle, and both get the
same outlet planes.  Tolerance: the inlet copies bitwise, everything else
1e-10 relative (the mass-rate sum runs in a different order)."""
import math

import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-10
READ = ("u", "v", "w", "p", "gx", "gy", "gz", "rho", "rhoh", "h", "t", "mu", "k", "drho")
OUT_FLOW = ("out_u", "out_v", "out_w", "out_gx", "out_gy", "out_gz", "conv0_x", "conv0_y", "conv0_z")
OUT_ENG = ("out_rhoh", "out_h", "out_t", "out_rho", "out_mu", "out_k", "conv0_eng")


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _setup(nxt, nxi, ny, nz, seed=4):
    _need_gpu()
    from chapsim1ww_b200 import IOChannel, TGChannel
    from oracle.pyoracle import OracleIO, synth_table
    lz = 4 * math.pi / 3
    table = synth_table(4096)
    tg = TGChannel(nxt, ny, nz, lz=lz)
    tg.random_fl_fld_tg(seed, 0.1, project=True)
    g = IOChannel(nxi, ny, nz, lz=lz, table=table)
    o = OracleIO(nxi, ny, nz, lz=lz, table=table)
    g.random_fl_theml_fld_io(seed + 1, 0.1)
    g.solverrk3_eng_io(1)
    g.solverrk3_mom_io(1)  # a non-zero density history
    for n in READ:
        o.set(n, g.get_field(n))
    rng = np.random.default_rng(seed)
    shape = (nz, ny + 2)
    for name, base in (("out_u", "u"), ("out_v", "v"), ("out_w", "w"), ("out_gx", "gx"), ("out_gy", "gy"),
                       ("out_gz", "gz"), ("out_rho", "rho"), ("out_h", "h"), ("out_t", "t"), ("out_mu", "mu"),
                       ("out_k", "k")):
        p = g.get_field(base)[:, :, -1] * (1.0 + 0.02 * rng.standard_normal(shape))
        g.set_plane(name, p)
        o.set_plane(name, p)
    p = g.get_field("rhoh")[:, :, -1] + 1e-3 * rng.standard_normal(shape)
    g.set_plane("out_rhoh", p)
    o.set_plane("out_rhoh", p)
    return tg, g, o


@pytest.mark.parametrize("dims", [(16, 24, 12, 8), (32, 48, 20, 40)])
def test_inlet_outlet_parity(dims):
    tg, g, o = _setup(*dims)
    # inlet: copies and one product, bitwise
    g.bc_tinlet_flow(tg)
    o.bc_tinlet_flow(*(tg.get_field(n) for n in ("u", "v", "w", "p")))
    for name in ("in_u", "in_v", "in_w", "in_gx", "in_gy", "in_gz", "in_p", "in_rho"):
        assert np.array_equal(g.get_plane(name), o.get_plane(name)), name
    for n in ("u", "gx"):
        assert np.array_equal(g.get_field(n), o.get(n)), n
    # outlet momentum, three substeps (the RK3 memory terms carry over)
    for ns in (1, 2, 3):
        g.bc_coutlet_mom_rk3(ns)
        o.bc_coutlet_mom_rk3(ns)
        errs = {n: relerr(g.get_plane(n), o.get_plane(n)) for n in OUT_FLOW}
        assert all(e <= TOL for e in errs.values()), (ns, errs)
        sg, so = g.bc_scalars(), o.bc_scalars()
        for key in ("u_outlet", "scaling", "inflow", "outflow", "mass_rate"):
            assert abs(sg[key] - so[key]) <= TOL * max(abs(so[key]), 1e-300), (ns, key, sg[key], so[key])
        assert abs(sg["balance"] - so["balance"]) <= TOL * abs(so["inflow"])
    # outlet energy, three substeps, table properties
    for ns in (1, 2, 3):
        g.bc_coutlet_eneg_rk3(ns)
        o.bc_coutlet_eneg_rk3(ns)
        errs = {n: relerr(g.get_plane(n), o.get_plane(n)) for n in OUT_ENG}
        assert all(e <= TOL for e in errs.values()), (ns, errs)
        assert abs(g.bc_scalars()["u_outlet_eng"] - o.bc_scalars()["u_outlet_eng"]) <= TOL
    assert g.bad_cells() == 0


def test_outlet_rescaling_closes_the_mass_balance():
    """After the outlet momentum operator the outflow through the ghost plane
    equals the inflow minus the volume integral of d(rho)/dt."""
    tg, g, o = _setup(16, 24, 12, 8, seed=9)
    g.bc_tinlet_flow(tg)
    g.bc_coutlet_mom_rk3(1)
    sc = g.bc_scalars()
    out_gx = g.get_plane("out_gx")
    from oracle.pyoracle import OracleTG
    dyfi = OracleTG(16, 12, 8, lz=4 * math.pi / 3).coef(2)  # DYFI(1:ny), the same y mesh
    dzi = 8 / (4 * math.pi / 3)
    fout_new = (out_gx[:, 1:13] / dyfi[None, :]).sum() / dzi
    assert abs(sc["inflow"] - sc["mass_rate"] - fout_new) <= 1e-12 * abs(sc["inflow"])


def test_boundary_operator_errors():
    _need_gpu()
    from chapsim1ww_b200 import ChapsimError, IOChannel, TGChannel
    tg = TGChannel(16, 10, 8)
    io = IOChannel(24, 12, 8, thermal=0)
    with pytest.raises(ChapsimError):
        io.bc_tinlet_flow(tg)  # ny differs
    with pytest.raises(ChapsimError):
        io.bc_coutlet_eneg_rk3(1)  # no energy equation
    with pytest.raises(ChapsimError):
        io.bc_coutlet_mom_rk3(4)
    with pytest.raises(ValueError):
        io.set_plane("out_u", np.zeros(3))
