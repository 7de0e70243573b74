"""GPU parity of the coupled TG -> IO step (TGFLOWFLG) against the oracle.

A TG section feeds the inlet of an IO section with Dirichlet / Neumann x ends
(BCX_io, src/READINI.f90:117-131; the reference's example 2, 1), whose
outlet is convective.  Both the library (chapsim_io_set_inlet,
chapsim_step_coupled: SOLVE's substep loop, src/SOLVE.f90:119-134) and the
oracle (TG oracle + coupled IO oracle, substep by substep) start from the
same seeded fields; after the steps every field of both sections, the IO
ghost columns included, agrees within 1e-10 relative (max |a - b| / max |b|,
FP64).  The graph-replayed pair step equals the eager substeps bitwise, the
inlet face carries the TG's first face exactly, and the IO section's
divergence vanishes to round-off in every column but the first.
"""
import math
import os

import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-10
TG_F = ("u", "v", "w", "p")
IO_FLOW = ("u", "v", "w", "p", "gx", "gy", "gz", "g0x", "g0y", "g0z", "ex0x", "ex0y", "ex0z")
IO_THERMAL = ("h", "t", "rho", "mu", "k", "rhoh", "rho0", "mu0", "drho", "rhse0")


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _table(kind):
    if kind == "constant":  # constant-property passive heat: rho = mu = k = 1, T = h
        h = np.linspace(-1.0, 1.0, 4096)
        one = np.ones_like(h)
        return [h, h.copy(), one, one.copy(), one.copy()]
    from oracle.pyoracle import synth_table
    return synth_table(4096)[:5]


def _pair(nxt, nxi, ny, nz, bcx=(2, 1), thermal=1, table="constant", seed=1):
    _need_gpu()
    from chapsim1ww_b200 import IOChannel, TGChannel
    from oracle.pyoracle import OracleIO, OracleTG
    lz = 4 * math.pi / 3
    tab = _table(table) if thermal else None
    tg = TGChannel(nxt, ny, nz, lz=lz)
    ot = OracleTG(nxt, ny, nz, lz=lz)
    tg.random_fl_fld_tg(seed, 0.1, project=False)  # the oracle's TG field, then both project
    ot.init_random(seed, 0.1)
    tg.solverrk3_mom_tg(0)
    ot.substep(0)
    g = IOChannel(nxi, ny, nz, lz=lz, thermal=thermal, table=tab, bcx=bcx)
    o = OracleIO(nxi, ny, nz, lz=lz, thermal=thermal, table=tab)
    o.set_bcx(*bcx)
    g.set_inlet(tg)
    o.set_inlet(*[ot.get(f) for f in TG_F])
    g.random_fl_theml_fld_io(seed + 1, 0.1)
    o.init_random(seed + 1, 0.1)
    return tg, ot, g, o


def _oracle_steps(ot, o, n):
    for _ in range(n):
        for ns in (1, 2, 3):
            ot.substep(ns)
            o.set_inlet(*[ot.get(f) for f in TG_F])
            o.substep(ns)


def _compare(tg, ot, g, o, thermal, what):
    errs = {"tg_" + n: relerr(tg.get_field(n), ot.get(n)) for n in TG_F}
    for n in IO_FLOW + (IO_THERMAL if thermal else ()):
        errs[n] = relerr(g.get_field(n), o.get(n))
    print(what + ": " + ", ".join(f"{n} {e:.1e}" for n, e in errs.items()))
    for n, e in errs.items():
        assert e <= TOL, (what, n, e)


@pytest.mark.parametrize("case", [
    dict(nxt=16, nxi=24, ny=16, nz=12, bcx=(2, 1), thermal=1, table="constant"),
    dict(nxt=32, nxi=40, ny=20, nz=16, bcx=(2, 1), thermal=1, table="synthetic"),
    dict(nxt=16, nxi=24, ny=18, nz=8, bcx=(2, 1), thermal=0),
    dict(nxt=16, nxi=20, ny=16, nz=12, bcx=(1, 1), thermal=1, table="constant"),
    # two x tiles of the TMA-staged momentum RHS (nx >= 36)
    dict(nxt=32, nxi=72, ny=24, nz=20, bcx=(2, 1), thermal=1, table="synthetic"),
    dict(nxt=32, nxi=64, ny=16, nz=12, bcx=(2, 1), thermal=0),
])
def test_coupled_step_parity(case):
    tg, ot, g, o = _pair(**case)
    thermal = case["thermal"]
    _compare(tg, ot, g, o, thermal, f"{case} after the initial field")
    g.step_coupled(tg, 3)
    _oracle_steps(ot, o, 3)
    _compare(tg, ot, g, o, thermal, f"{case} after 3 steps")
    b, bo = g.bc_scalars(), o.bc_scalars()
    for k in ("u_outlet", "scaling", "inflow", "outflow"):
        assert abs(b[k] - bo[k]) <= TOL * max(1.0, abs(bo[k])), (k, b[k], bo[k])
    # BC_TINLET_FLOW: the first face carries the TG's first-face u exactly
    u, tu = g.get_field("u"), tg.get_field("u")
    assert np.array_equal(u[:, 1:-1, 1], tu[:, 1:-1, 0])
    assert np.array_equal(u[:, :, 0], tu[:, :, -1])
    # DIVGCK_io as the oracle's, and the projection: columns 2..nx
    # divergence-free (Dirichlet outlet), the first one not
    assert abs(g.divgck_io() - o.divmax()) <= TOL * o.divmax()
    dc = _div_columns(g, math.pi * 8)
    scale = np.abs(g.get_field("gx")).max() * g.nx / (8 * math.pi)
    print(f"{case}: div G + DrhoDtP, first column {dc[0]:.2e}, the others <= {dc[1:].max():.2e}")
    assert dc[1:].max() <= 1e-12 * scale and dc[0] > 1e3 * dc[1:].max()
    tg.close()


def _div_columns(g, lx):
    """max over (j, k) of |div G + DrhoDtP| per interior column of an IOChannel."""
    nx, ny, nz = g.nx, g.ny, g.nz
    gx, gy, gz = (g.get_field(n) for n in ("gx", "gy", "gz"))
    dr = g.get_field("drho") if g.iocfg.thermal else np.zeros_like(gx)
    dyfi = 1.0 / np.diff(g.mesh(0))  # DYFI from the y nodes
    dxi, dzi = nx / lx, nz / (4 * math.pi / 3)
    c = slice(1, nx + 1)
    d = ((gx[:, 1:ny + 1, 2:nx + 2] - gx[:, 1:ny + 1, c]) * dxi
         + (gy[:, 2:ny + 2, c] - gy[:, 1:ny + 1, c]) * dyfi[None, :, None]
         + (np.roll(gz, -1, 0)[:, 1:ny + 1, c] - gz[:, 1:ny + 1, c]) * dzi + dr[:, 1:ny + 1, c])
    return np.abs(d).max(axis=(0, 1))


def test_coupled_graph_equals_eager_substeps():
    """chapsim_step_coupled (one captured graph per step) against the same
    substeps launched one by one through the reference-facing entry points."""
    tg, ot, g, o = _pair(24, 32, 16, 12, thermal=1, table="synthetic")
    from chapsim1ww_b200 import IOChannel, TGChannel
    lz = 4 * math.pi / 3
    tg2 = TGChannel(24, 16, 12, lz=lz)
    g2 = IOChannel(32, 16, 12, lz=lz, table=_table("synthetic"), bcx=(2, 1))
    g2.set_inlet(tg2)
    tg2.random_fl_fld_tg(1, 0.1)
    g2.random_fl_theml_fld_io(2, 0.1)
    g.step_coupled(tg, 2)
    for _ in range(2):
        for ns in (1, 2, 3):
            tg2.solverrk3_mom_tg(ns)
            g2.solverrk3_eng_io(ns)
            g2.solverrk3_mom_io(ns)
    for n in TG_F:
        assert np.array_equal(tg.get_field(n), tg2.get_field(n)), n
    for n in IO_FLOW + IO_THERMAL:
        assert np.array_equal(g.get_field(n), g2.get_field(n)), n


def test_coupled_section_refusals():
    """What the coupled section does not run: a step without its inlet
    source, the x-periodic statistics, the learned property kernel and the
    stand-alone boundary operators."""
    _need_gpu()
    from chapsim1ww_b200 import ChapsimError, IOChannel, TGChannel, _lib
    g = IOChannel(16, 12, 8, table=_table("constant"), bcx=(2, 1))
    with pytest.raises(ChapsimError):
        g.random_fl_theml_fld_io(1, 0.1)
    with pytest.raises(ChapsimError):
        g.step(1)
    tg = TGChannel(16, 12, 8)
    g.set_inlet(tg)
    tg.random_fl_fld_tg(1, 0.1)
    g.random_fl_theml_fld_io(2, 0.1)
    g.step(1)  # a frozen inflow: the IO section alone
    for call in (lambda: g.pp_mean_zx(), lambda: g.bc_coutlet_mom_rk3(1), lambda: g.bc_tinlet_flow(tg),
                 lambda: g.therm_prop_update(0)):
        with pytest.raises(ChapsimError):
            call()
    with pytest.raises(ChapsimError):
        IOChannel(16, 12, 8, table=_table("constant"), bcx=(2, 1), visc_scheme=1)
    with pytest.raises(ChapsimError):
        IOChannel(16, 12, 8, table=_table("constant"), bcx=(2, 1), precision=_lib.MIXED)
    # destroying the TG section detaches the IO section, which then refuses to step
    tg.close()
    with pytest.raises(ChapsimError):
        g.solverrk3_mom_io(1)
    g.close()


def test_coupled_restart_files_and_continuation(tmp_path):
    """WRT_INSTANT_VARS_IO / RESTART_INSTANT_VARS_IO of the coupled section
    (src/processing/WRT_VARS_IO.f90:21-60, RESTART_io.f90:16-120): files of
    I = 1..NCL1_io + 1 (the outlet ghost column included, NCL1E in the
    header) named DNS_perioz beside the TG section's DNS_perixz files; the
    restarted section holds the written G, p, T, rho, h on those columns and
    the TG's last column in its inlet ghost column, and one step from the
    restarted state agrees with the oracle given that state."""
    from chapsim1ww_b200 import IOChannel, TGChannel
    from oracle.pyoracle import OracleIO, OracleTG
    d = str(tmp_path) + "/"
    nxt, nxi, ny, nz = 16, 24, 16, 12
    lz = 4 * math.pi / 3
    tg, ot, g, o = _pair(nxt, nxi, ny, nz, thermal=1, table="synthetic")
    g.step_coupled(tg, 2)
    tg.write_instant(d, 6, 0.006)
    g.write_instant(d, 6, 0.006)
    names = sorted(os.listdir(d))
    assert sum(n.startswith("DNS_perixz") for n in names) == 4
    assert sum(n.startswith("DNS_perioz") for n in names) == 7
    u_file = [n for n in names if n.startswith("DNS_perioz") and n.endswith("_U.D")][0]
    hdr = np.fromfile(d + u_file, dtype=np.int32, count=4)
    assert tuple(int(x) for x in hdr) == (nxi + 1, ny, nz, 6)
    assert os.path.getsize(d + u_file) == 16 + 24 + 8 * (nxi + 1) * ny * nz
    tg2 = TGChannel(nxt, ny, nz, lz=lz)
    g2 = IOChannel(nxi, ny, nz, lz=lz, table=_table("synthetic"), bcx=(2, 1))
    g2.set_inlet(tg2)
    assert tg2.read_instant(d, 0.006) == (6, 0.006)
    assert g2.read_instant(d, 0.006) == (6, 0.006)
    for n in ("gx", "gy", "gz", "p", "t", "rho", "h"):
        assert relerr(g2.get_field(n)[:, 1:-1, 1:], g.get_field(n)[:, 1:-1, 1:]) <= 1e-14, n
    u2, tu2 = g2.get_field("u"), tg2.get_field("u")
    assert np.array_equal(u2[:, :, 0], tu2[:, :, -1])
    # the first face: BC_TINLET_FLOW's G, then VELOCITY_CALC_io's G / RHO_STG
    assert relerr(u2[:, 1:-1, 1], tu2[:, 1:-1, 0]) <= 1e-14
    ot2 = OracleTG(nxt, ny, nz, lz=lz)
    for n in TG_F:
        ot2.set(n, tg2.get_field(n))
    o2 = OracleIO(nxi, ny, nz, lz=lz, thermal=1, table=_table("synthetic"))
    o2.set_bcx(2, 1)
    o2.set_inlet(*[ot2.get(f) for f in TG_F])
    for n in IO_FLOW + IO_THERMAL:
        o2.set(n, g2.get_field(n))
    g2.step_coupled(tg2, 1)
    _oracle_steps(ot2, o2, 1)
    _compare(tg2, ot2, g2, o2, 1, "one step after the restart")
    tg.close()
    tg2.close()
