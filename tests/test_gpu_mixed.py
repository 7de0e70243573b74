"""Mixed-precision form (FP64 state, FP32 temporaries / FFT, FP64 Poisson
lines and one FP64-residual refinement sweep) against the FP64 oracle.

Stated tolerances (max |a-b| / max |b| after init + NS=0 + 3 steps):
u, v, w <= 1e-6 and p <= 1e-5; max |div u| <= 1e-8 (the metric's gate)."""
import math

import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu
TOL_VEL, TOL_P, TOL_DIV = 1e-6, 1e-5, 1e-8


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("dims", [(64, 48, 32), (48, 20, 40), (128, 96, 64)])
def test_mixed_vs_oracle(dims):
    _need_gpu()
    from chapsim1ww_b200 import MIXED, TGChannel
    from oracle.pyoracle import OracleTG
    g = TGChannel(*dims, precision=MIXED)
    o = OracleTG(*dims)
    g.random_fl_fld_tg(1, 0.1, project=True)
    o.init_random(1, 0.1)
    o.substep(0)
    g.step(3)
    o.step(3)
    errs = {n: relerr(g.get_field(n), o.get(n)) for n in ("u", "v", "w", "p")}
    assert max(errs["u"], errs["v"], errs["w"]) <= TOL_VEL, errs
    assert errs["p"] <= TOL_P, errs
    assert g.divgck_tg() <= TOL_DIV


def test_mixed_divergence_gate_long_run():
    _need_gpu()
    from chapsim1ww_b200 import MIXED, TGChannel
    g = TGChannel(96, 64, 64, precision=MIXED)
    g.random_fl_fld_tg(2, 0.1, project=True)
    g.step(20)
    assert g.divgck_tg() <= TOL_DIV
    assert g.nan_count() == 0
    assert abs(g.bulk_velocity_tg() - 1.0) < 1e-8


def test_mixed_deterministic():
    _need_gpu()
    from chapsim1ww_b200 import MIXED, TGChannel
    outs = []
    for _ in range(2):
        g = TGChannel(64, 32, 32, precision=MIXED)
        g.random_fl_fld_tg(3, 0.1, project=True)
        g.step(4)
        outs.append(g.get_field("u"))
        g.close()
    assert np.array_equal(outs[0], outs[1])
