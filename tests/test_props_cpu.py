"""CPU checks of the property-table pieces: the two independent synthetic
table generators agree, the oracle spline (Forsythe-Malcolm-Moler, as
CUBIC_SPLINE, src/Flow_State.f90:1693-1787) reproduces the table nodes and
cubic data exactly, and the property update follows THERM_PROP_UPDATE's
rules."""
import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def L():
    from oracle import pyoracle
    lib = pyoracle.load()
    P = ctypes.c_void_p
    lib.oracle_synth_table.argtypes = [ctypes.c_int] + [P] * 7
    lib.oracle_cubic_spline.argtypes = [ctypes.c_int] + [P] * 5
    lib.oracle_spline_eval.argtypes = [ctypes.c_int] + [P] * 5 + [ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    lib.oracle_therm_prop_update.argtypes = [ctypes.c_int] + [P] * 5 + [ctypes.c_int64] + [P] * 5
    lib.oracle_therm_prop_update.restype = ctypes.c_int64
    return lib


def oracle_table(L, n=4096):
    cols = [np.zeros(n) for _ in range(7)]
    L.oracle_synth_table(n, *[c.ctypes.data for c in cols])
    return cols


def test_table_generators_agree(L):
    from chapsim1ww_b200.props import synthetic_table
    a = synthetic_table(4096)
    b = oracle_table(L)
    for x, y in zip(a, b[:6]):
        assert np.abs(x - y).max() <= 1e-14 * np.abs(y).max()
    H, T, D = b[0], b[1], b[2]
    assert T[0] == 0.0 and np.all(np.diff(T) > 0) and np.all(D > 0)


def test_spline_reproduces_nodes_and_cubics(L):
    x = np.sort(np.random.default_rng(0).uniform(-1, 1, 40))
    y = 2.0 * x ** 3 - x ** 2 + 0.5 * x + 3.0
    b, c, d = np.zeros(40), np.zeros(40), np.zeros(40)
    L.oracle_cubic_spline(40, x.ctypes.data, y.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data)
    out = ctypes.c_double()
    for u in np.linspace(x[0], x[-1], 101)[1:-1]:
        assert L.oracle_spline_eval(40, x.ctypes.data, y.ctypes.data, b.ctypes.data, c.ctypes.data,
                                    d.ctypes.data, u, ctypes.byref(out)) == 0
        # FMM end conditions make the spline exact on cubic data
        assert abs(out.value - (2.0 * u ** 3 - u ** 2 + 0.5 * u + 3.0)) < 1e-11
    for i in range(1, 39):
        L.oracle_spline_eval(40, x.ctypes.data, y.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data, x[i],
                             ctypes.byref(out))
        assert out.value == y[i]
    assert L.oracle_spline_eval(40, x.ctypes.data, y.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data,
                                x[0], ctypes.byref(out)) == -1


def test_prop_update_rules(L):
    H, T, D, M, K, CP, _ = oracle_table(L)
    h = np.array([0.3, 0.0, 5e-11, -0.99, 1.5, -1.0, 0.999])
    Tc, Dc, Mc, Kc = (np.full(7, -7.0) for _ in range(4))
    bad = L.oracle_therm_prop_update(4096, H.ctypes.data, T.ctypes.data, D.ctypes.data, M.ctypes.data,
                                     K.ctypes.data, 7, h.ctypes.data, Tc.ctypes.data, Dc.ctypes.data,
                                     Mc.ctypes.data, Kc.ctypes.data)
    assert bad == 2  # 1.5 and -1.0 (the first node itself is outside, as in the reference)
    for idx in (1, 2, 4, 5):  # |h| < 1e-10 and out-of-range cells are left unchanged
        assert Tc[idx] == -7.0 and Dc[idx] == -7.0
    i = np.searchsorted(H, 0.3) - 1
    assert T[i] <= Tc[0] <= T[i + 1]
    assert abs(Dc[0] - 1.0 / (1.0 + 2.0 * Tc[0])) < 1e-9
    assert abs(Mc[0] - Dc[0] ** -0.5) < 1e-9 and Kc[0] == pytest.approx(Mc[0], abs=1e-12)


def test_mlp_reference_gradient_fd():
    """The numpy reference gradient matches central finite differences."""
    from oracle import mlp_ref
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, mlp_ref.NPARAM)
    x = rng.uniform(-1, 1, 16)
    t = rng.normal(0, 1, (16, 5))
    _, g = mlp_ref.loss_and_grad(p, x, t)
    for idx in rng.choice(mlp_ref.NPARAM, 25, replace=False):
        e = np.zeros_like(p)
        e[idx] = 1e-6
        fd = (mlp_ref.loss_and_grad(p + e, x, t)[0] - mlp_ref.loss_and_grad(p - e, x, t)[0]) / 2e-6
        assert abs(fd - g[idx]) < 1e-7 + 1e-5 * abs(fd)
