"""GPU parity of the IO-section substep (x-periodic IO channel: energy
equation with table properties, explicit variable-property momentum, FISHPACK
Poisson) against the FP64 CPU oracle.  Tolerance: FP64 within 1e-10 relative
(max |a-b| / max |b|) on every state field after every checked stage; the
library and the oracle get the same table columns."""
import math

import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-10
FLOW = ("u", "v", "w", "p", "gx", "gy", "gz")
THERMAL = ("h", "t", "rho", "mu", "k", "rhoh")


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def pair(nx, ny, nz, thermal=1, seed=2, amp=0.1, **kw):
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import OracleIO, synth_table
    table = synth_table(4096)
    g = IOChannel(nx, ny, nz, thermal=thermal, table=table if thermal else None, **kw)
    o = OracleIO(nx, ny, nz, thermal=thermal, table=table, **kw)
    g.random_fl_theml_fld_io(seed, amp)
    o.init_random(seed, amp)
    return g, o


def compare(g, o, names, tol=TOL, tag=""):
    errs = {n: relerr(g.get_field(n), o.get(n)) for n in names}
    bad = {n: e for n, e in errs.items() if not e <= tol}
    assert not bad, f"{tag}: relative errors above {tol}: {errs}"
    return errs


@pytest.mark.parametrize("dims", [(16, 12, 8), (32, 24, 16), (48, 20, 40)])
def test_io_isothermal_parity(dims):
    g, o = pair(*dims, thermal=0)
    compare(g, o, FLOW, tag="init+projection")
    for step in range(2):
        for ns in (1, 2, 3):
            g.solverrk3_mom_io(ns)
            o.mom(ns)
            compare(g, o, FLOW, tag=f"step{step} ns{ns}")
    compare(g, o, ("ex0x", "ex0y", "ex0z", "g0x", "g0y", "g0z"), tag="state")
    assert g.divgck_io() < 1e-11 and o.divmax() < 1e-11
    assert abs(g.bulk_massflux_io() - o.bulk(1)) < 1e-12


# nx >= 36 runs the TMA z-marching momentum RHS (80: a partial last x tile)
@pytest.mark.parametrize("dims", [(16, 12, 8), (32, 24, 16), (40, 18, 24), (64, 16, 12), (80, 12, 10)])
def test_io_thermal_parity(dims):
    g, o = pair(*dims, thermal=1)
    compare(g, o, FLOW + THERMAL, tag="init+projection")
    for step in range(2):
        for ns in (1, 2, 3):
            g.solverrk3_eng_io(ns)
            o.eng(ns)
            compare(g, o, THERMAL + ("rho0", "mu0", "rhse0"), tag=f"step{step} eng{ns}")
            g.solverrk3_mom_io(ns)
            o.mom(ns)
            compare(g, o, FLOW, tag=f"step{step} mom{ns}")
            # DrhoDtP is built from mass-flux divergences that the previous
            # projection drove to round-off, so it stays at round-off level
            assert np.abs(g.get_field("drho") - o.get("drho")).max() < 1e-9
    assert g.bad_cells() == 0 and o.bad_cells() == 0
    assert g.divgck_io() < 1e-10 and o.divmax() < 1e-10
    assert abs(g.bulk_h_io() - o.bulk(2)) <= 1e-12 * max(1.0, abs(o.bulk(2)))


def test_io_graph_step_matches_eager_bitwise():
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import synth_table
    table = synth_table(4096)
    a = IOChannel(32, 24, 16, table=table)
    b = IOChannel(32, 24, 16, table=table)
    a.random_fl_theml_fld_io(5, 0.1)
    b.random_fl_theml_fld_io(5, 0.1)
    a.step(3)  # two graphs (the G buffers alternate every substep)
    for _ in range(3):
        for ns in (1, 2, 3):
            b.solverrk3_eng_io(ns)
            b.solverrk3_mom_io(ns)
    for n in FLOW + THERMAL + ("g0x", "drho"):
        assert np.array_equal(a.get_field(n), b.get_field(n)), n


@pytest.mark.parametrize("visc", [0, 1])
def test_io_velocity_is_a_result_not_an_input(visc):
    """u, v, w of an IO context are rebuilt from G and the density before
    each substep's momentum stage (VELOCITY_CALC_io, src/SOLVE.f90:131-132)
    and the energy stage does not read them: a step from overwritten u, v, w
    gives the same bits.  The end-to-end benchmark uploads G, p and rho h
    only on this basis."""
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import synth_table
    table = synth_table(4096)
    a = IOChannel(32, 24, 16, table=table, dt=2e-3, visc_scheme=visc)
    b = IOChannel(32, 24, 16, table=table, dt=2e-3, visc_scheme=visc)
    a.random_fl_theml_fld_io(9, 0.1)
    b.random_fl_theml_fld_io(9, 0.1)
    a.step(1)
    b.step(1)
    rng = np.random.default_rng(3)
    for n in ("u", "v", "w"):
        b.set_field(n, rng.standard_normal(b.shape))
    a.step(1)
    b.step(1)
    for n in FLOW + THERMAL:
        assert np.array_equal(a.get_field(n), b.get_field(n)), n


def test_io_fp64_run_to_run_bitwise():
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    out = []
    for _ in range(2):
        c = IOChannel(48, 20, 40)
        c.random_fl_theml_fld_io(7, 0.1)
        c.step(2)
        out.append([c.get_field(n) for n in ("u", "p", "gx", "h", "rho")])
        c.close()
    for x, y in zip(*out):
        assert np.array_equal(x, y)


def test_io_buoyancy_and_pressure_drive_parity():
    g, o = pair(16, 12, 8, thermal=1, gravdir=1, f_a=0.3, flowdrvtp=2, cfgv=8.18e-3)
    compare(g, o, FLOW + THERMAL, tag="init")
    for ns in (1, 2, 3):
        g.solverrk3_eng_io(ns)
        o.eng(ns)
        g.solverrk3_mom_io(ns)
        o.mom(ns)
    compare(g, o, FLOW + THERMAL, tag="step")


def test_io_reference_shortcuts_parity():
    # shortcuts on: the reference-state branches of the look-ups (h = 0 cells
    # keep their properties, T = 1 -> rho = mu = k = 1)
    g, o = pair(16, 12, 8, thermal=1, shortcuts=1)
    compare(g, o, FLOW + THERMAL, tag="init")
    g.step(1)
    o.step(1)
    compare(g, o, FLOW + THERMAL, tag="step")


def test_io_divgck_after_projection_and_errors():
    _need_gpu()
    from chapsim1ww_b200 import IOChannel, ChapsimError
    c = IOChannel(16, 12, 8, thermal=0)
    c.random_fl_theml_fld_io(1, 0.1)
    assert c.divgck_io() < 1e-12
    with pytest.raises(ChapsimError):
        c.solverrk3_eng_io(1)  # thermal off
    with pytest.raises(ChapsimError):
        c._chk(c.lib.chapsim_step_tg(c.h, 1))  # not a TG context


def test_io_density_time_derivation_parity():
    # plant G and G0 with O(1) divergences so DENSITY_TIME_DERIVATION (and the
    # DrhoDtP term of DIVG_io) work on non-trivial values
    g, o = pair(32, 24, 16, thermal=1)
    rng = np.random.default_rng(3)
    for name in ("gx", "gy", "gz", "g0x", "g0y", "g0z"):
        a = g.get_field(name) * (1.0 + 0.05 * rng.standard_normal(g.shape))
        a[:, 0, :] = 0.0
        a[:, -1, :] = 0.0
        if name in ("gy", "g0y"):
            a[:, 1, :] = 0.0
        g.set_field(name, a)
        o.set(name, a)
    for ns in (1, 2, 3):
        g.solverrk3_eng_io(ns)
        o.eng(ns)
        g.solverrk3_mom_io(ns)
        o.mom(ns)
        compare(g, o, FLOW + THERMAL + ("drho",), tag=f"mom{ns}")
    assert np.abs(o.get("drho")).max() > 1e-3


@pytest.mark.parametrize("name", ["io_16x12x8_seed3", "io_heated_16x10x8_seed7", "io_si_16x12x8_seed3",
                                  "io_si_heated_16x10x8_seed7"])
def test_io_golden_fixture(name):
    """The library (graph-replayed full RK3 steps) against the committed
    fixtures of the independent numpy restatement, tests/golden/numpy_io.py
    (explicit and semi-implicit viscous schemes)."""
    _need_gpu()
    import os
    from chapsim1ww_b200 import IOChannel
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    meta = list(z["meta"]) + [0.0] * (15 - len(z["meta"]))
    nx, ny, nz, lx, lz, ren, dt, seed, amp, steps, thermal, prt, qb, qt, visc = meta
    g = IOChannel(int(nx), int(ny), int(nz), lx=lx, lz=lz, ren=ren, dt=dt, thermal=int(thermal), prt=prt,
                  qw=(qb, qt), visc_scheme=int(visc))
    g.random_fl_theml_fld_io(int(seed), amp)
    for n in ("gx", "gy", "p"):
        assert relerr(g.get_field(n), z["ns0_" + n]) < TOL, n
    g.step(int(steps))
    names = ["gx", "gy", "gz", "p", "u", "ex0x"] + (["h", "rho", "mu", "rhse0"] if thermal else [])
    for n in names:
        assert relerr(g.get_field(n), z["end_" + n]) < TOL, n
    assert g.divgck_io() < 1e-12
    assert abs(g.bulk_massflux_io() - float(z["end_bulk_g"])) < 1e-12


@pytest.mark.parametrize("walls,visc", [(3, 0), (1, 0), (2, 1)])
def test_io_isothermal_wall_parity(walls, visc):
    """BCWALLHEAT = isoThermalWall (BC_WALL_ISOTHERMAL, src/BC_WALL.f90:462-515,
    with the wall rows of RHS_ENERGY_EXPLICIT, src/RHS_ENERGY_EXPLICIT.f90:41-72)
    on both walls or one, explicit and semi-implicit viscous terms: the GPU
    against the oracle after every substep of two RK3 steps, FP64 within
    1e-10; the ghost rows hold the wall values."""
    g, o = pair(40, 18, 24, thermal=1, qw=(0.95, 0.80), isothermal=walls, visc_scheme=visc)
    compare(g, o, FLOW + THERMAL, tag="init+projection")
    for step in range(2):
        for ns in (1, 2, 3):
            g.solverrk3_eng_io(ns)
            o.eng(ns)
            compare(g, o, THERMAL + ("rho0", "mu0", "rhse0"), tag=f"step{step} eng{ns}")
            g.solverrk3_mom_io(ns)
            o.mom(ns)
            compare(g, o, FLOW, tag=f"step{step} mom{ns}")
    T = g.get_field("t")
    for side, j in ((0, 0), (1, 19)):
        if walls & (1 << side):
            assert np.all(T[:, j, :] == (0.95, 0.80)[side])
    assert g.bad_cells() == 0 and o.bad_cells() == 0
    assert g.divgck_io() < 1e-10 and o.divmax() < 1e-10


def test_isothermal_wall_outside_table_is_refused():
    _need_gpu()
    from chapsim1ww_b200 import ChapsimError, IOChannel
    from oracle.pyoracle import synth_table
    with pytest.raises(ChapsimError):
        IOChannel(16, 12, 8, table=synth_table(4096), qw=(5.0, 0.8), isothermal=1)


@pytest.mark.parametrize("bcx", [(1, 1), (1, 2), (2, 2), (2, 1)])
def test_io_poisson_nonperiodic_x_parity(bcx):
    """FISHPACK_POIS3D_SIMPLE with Dirichlet / Neumann x ends (BCX_io 1 / 2:
    FISHPACK's SINT, SINQ, COST, COSQ x transforms): chapsim_pois3d against
    the oracle on the same random right-hand side, FP64 within 1e-10 over the
    whole field (interior, the copied ghost rows, the untouched ghost
    columns), two grids."""
    _need_gpu()
    from chapsim1ww_b200 import ChapsimError, IOChannel
    from oracle.pyoracle import OracleIO
    rng = np.random.default_rng(9)
    for dims in ((24, 18, 16), (40, 20, 12)):
        g = IOChannel(*dims, thermal=0, bcx=bcx)
        o = OracleIO(*dims, thermal=0)
        o.set_bcx(*bcx)
        rhs = rng.standard_normal((dims[2], dims[1] + 2, dims[0] + 2))  # with the x ghost columns
        g.set_field("rhsphi", rhs)
        o.set("rhsphi", rhs)
        g.fishpack_pois3d()
        o.pois3d()
        e = relerr(g.get_field("phi"), o.get("phi"))
        assert e <= 1e-10, (dims, e)
        with pytest.raises(ChapsimError):
            g.step(1)  # a coupled section steps only with its TG inlet source
        # a DT change rebuilds the coefficient tables the solve reads: same result
        g.set_dt(2e-3)
        g.fishpack_pois3d()
        assert relerr(g.get_field("phi"), o.get("phi")) <= 1e-10
        g.close()
