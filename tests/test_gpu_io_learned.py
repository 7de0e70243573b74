"""The IO section's mixed precision form and learned property model.

Mixed form (FP64 fields, FP32 Poisson spectra, one FP64-residual refinement
sweep) against the FP64 oracle after init + 3 RK3 steps, stated tolerances:
u, v, w, G, h, T, rho <= 1e-6 and p <= 1e-5 relative (max |a - b| / max |b|),
max |div G + drho/dt| <= 1e-8.

Learned properties on an IO context (chapsim_set_props_mode): the model of a
property engine trained on the context's table and gated at 1e-4 stands in for
the table splines inside SOLVERRK3_ENG_IO's property update
(src/SOLVERRK3_ENG_IO.f90:46-55, src/THERM_PROP_UPDATE.f90:129-205).  A gate
that clears no bin reproduces the table path bit for bit; with the 1e-4 gate
the properties stay within 2e-4 of the table and the flow follows.
"""
import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu

FLOW = ("u", "v", "w", "p", "gx", "gy", "gz")
THERMAL = ("h", "t", "rho", "mu", "k")


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def table():
    _need_gpu()
    from oracle.pyoracle import synth_table
    return synth_table(4096)


@pytest.fixture(scope="module")
def engine(table):
    """Model trained on the table (65,536 samples, seed 2) and gated at 1e-4."""
    from chapsim1ww_b200 import PropertyEngine
    e = PropertyEngine(*table[:6])
    loss = e.train(nsamples=65536, seed=2, steps=20000, lr=3e-3)
    nb, worst = e.gate(tol=1e-4, nbins=256)
    print(f"engine: loss {loss:.3e}, {nb}/256 bins cleared for T, rho, mu, k, worst {worst:.2e}")
    return e


def _pair(table, dims, seed=2, **kw):
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import OracleIO
    g = IOChannel(*dims, table=table, **kw)
    o = OracleIO(*dims, table=table)
    g.random_fl_theml_fld_io(seed, 0.1)
    o.init_random(seed, 0.1)
    return g, o


@pytest.mark.parametrize("dims", [(64, 48, 32), (40, 18, 24)])
def test_io_mixed_form_vs_fp64_oracle(table, dims):
    from chapsim1ww_b200 import MIXED
    g, o = _pair(table, dims, precision=MIXED)
    g.step(3)
    o.step(3)
    errs = {n: relerr(g.get_field(n), o.get(n)) for n in FLOW + ("h", "t", "rho")}
    div = g.divgck_io()
    print(f"IO mixed {dims}, 3 steps: " + ", ".join(f"{n} {e:.2e}" for n, e in errs.items()) + f", div {div:.2e}")
    for n, e in errs.items():
        assert e <= (1e-5 if n == "p" else 1e-6), (n, e)
    assert div <= 1e-8


def test_io_mixed_form_without_refinement(table):
    """The single FP32 Poisson solve, for comparison: errors and divergence
    printed; the divergence gate is what the refinement sweep is for."""
    from chapsim1ww_b200 import MIXED
    g, o = _pair(table, (64, 48, 32), precision=MIXED)
    g.set_refinement(0)
    g.step(3)
    o.step(3)
    errs = {n: relerr(g.get_field(n), o.get(n)) for n in ("u", "p", "gx")}
    print(f"IO mixed without refinement: {errs}, div {g.divgck_io():.2e}")
    assert errs["u"] <= 1e-5 and errs["p"] <= 1e-3


def test_therm_prop_update_table_matches_oracle(table):
    import ctypes

    from chapsim1ww_b200 import IOChannel
    from oracle import pyoracle
    g = IOChannel(40, 18, 24, table=table)
    g.random_fl_theml_fld_io(3, 0.1)
    rng = np.random.default_rng(4)
    h = g.get_field("h")
    h[:, 1:-1, :] = rng.uniform(-0.95, 0.95, h[:, 1:-1, :].shape)
    g.set_field("h", h)
    g.therm_prop_update(mode=0)
    L = pyoracle.load()
    P = ctypes.c_void_p
    L.oracle_therm_prop_update.argtypes = [ctypes.c_int] + [P] * 5 + [ctypes.c_int64] + [P] * 5
    L.oracle_therm_prop_update.restype = ctypes.c_int64
    H, T, D, M, K = [np.ascontiguousarray(c) for c in table[:5]]
    hi = np.ascontiguousarray(h[:, 1:-1, :].ravel())
    out = [np.zeros(len(hi)) for _ in range(4)]
    assert L.oracle_therm_prop_update(len(H), H.ctypes.data, T.ctypes.data, D.ctypes.data, M.ctypes.data,
                                      K.ctypes.data, len(hi), hi.ctypes.data, *[q.ctypes.data for q in out]) == 0
    for name, ref in zip(("t", "rho", "mu", "k"), out):
        got = g.get_field(name)[:, 1:-1, :].ravel()
        assert relerr(got, ref) <= 1e-13, name


def test_learned_mode_with_empty_gate_is_the_table_bitwise(table):
    from chapsim1ww_b200 import IOChannel, PropertyEngine, _lib
    e = PropertyEngine(*table[:6])
    e.train(nsamples=65536, seed=2, steps=500, lr=3e-3)
    assert e.gate(tol=0.0, nbins=64)[0] == 0
    a = IOChannel(48, 20, 40, table=table)
    b = IOChannel(48, 20, 40, table=table)
    a.set_props_mode(_lib.PROPS_MLP, e)
    e.close()  # the context holds its own copy of the model
    for s in (a, b):
        s.random_fl_theml_fld_io(5, 0.1)
        s.step(2)
    for n in FLOW + THERMAL + ("rhoh",):
        assert np.array_equal(a.get_field(n), b.get_field(n)), n


def test_learned_mode_steps_vs_fp64_oracle(table, engine):
    from chapsim1ww_b200 import _lib
    g, o = _pair(table, (64, 48, 32))
    g.set_props_mode(_lib.PROPS_MLP, engine)
    g.step(3)
    o.step(3)
    errs = {n: relerr(g.get_field(n), o.get(n)) for n in FLOW + THERMAL}
    div = g.divgck_io()
    print("learned properties, 64x48x32, 3 steps vs FP64 table oracle: " +
          ", ".join(f"{n} {e:.2e}" for n, e in errs.items()) + f", div {div:.2e}")
    for n in THERMAL:
        assert errs[n] <= 2e-4, (n, errs[n])
    for n in FLOW:
        assert errs[n] <= (1e-3 if n == "p" else 1e-4), (n, errs[n])
    assert div <= 1e-8
    assert g.bad_cells() == 0


def test_therm_prop_update_learned_vs_table(table, engine):
    from chapsim1ww_b200 import IOChannel, _lib
    g = IOChannel(40, 18, 24, table=table)
    g.random_fl_theml_fld_io(3, 0.1)
    rng = np.random.default_rng(8)
    h = g.get_field("h")
    h[:, 1:-1, :] = rng.uniform(-0.95, 0.95, h[:, 1:-1, :].shape)
    g.set_field("h", h)
    g.therm_prop_update(mode=0)
    ref = {n: g.get_field(n)[:, 1:-1, :] for n in ("t", "rho", "mu", "k")}
    g.set_props_mode(_lib.PROPS_MLP, engine)
    g.therm_prop_update(mode=1)
    for n, r in ref.items():
        assert relerr(g.get_field(n)[:, 1:-1, :], r) <= 2e-4, n
