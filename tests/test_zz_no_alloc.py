"""The allocation-free max |div u| entry point, for callers that may not
allocate device memory when they run the check (a host recording its time
step into its own CUDA graph, where cudaMalloc is not allowed during capture,
or a host that hands out device memory from its own fixed pool).  It must
agree with the context's reduction (chapsim_reduce, CHAPSIM_R_DIVMAX) on
two calls in a row.  The file is named so that pytest collects it last."""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _noalloc_divmax(lib, ch, u, v, w, dyfi, out):
    rc = lib.chapsim_divmax_noalloc(u.data_ptr(), v.data_ptr(), w.data_ptr(), dyfi.data_ptr(), ch.nx, ch.ny, ch.nz,
                                    ch.nx / ch.cfg.lx, ch.nz / ch.cfg.lz, out.data_ptr(), None)
    assert rc == 0, rc


def test_noalloc_divmax_matches_context_reduction_twice():
    _need_gpu()
    import torch
    from chapsim1ww_b200 import TGChannel, _lib
    lib = _lib.load()
    ch = TGChannel(64, 48, 32, lx=4 * math.pi, lz=4 * math.pi / 3)
    ch.random_fl_fld_tg(4, 0.1, project=False)  # not yet projected: div u is O(1)
    dev = "cuda:0"
    fields = {n: torch.empty(ch.n, dtype=torch.float64, device=dev) for n in ("u", "v", "w")}
    dyfi = torch.zeros(ch.ny + 2, dtype=torch.float64, device=dev)
    dyfi[1:ch.ny + 1] = torch.tensor(ch.mesh(2), dtype=torch.float64)
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)

    for call in range(2):
        for n, t in fields.items():
            ch.get_field_device(n, t.data_ptr())
        torch.cuda.synchronize()
        want = ch.divgck_tg()
        _noalloc_divmax(lib, ch, fields["u"], fields["v"], fields["w"], dyfi, out)
        got = out.item()  # synchronises
        assert want > 0.0
        assert abs(got - want) <= 1e-14 * want, (call, got, want)
        ch.step(1)  # second call on a projected field (div u at round-off)


def test_noalloc_rejects_oversized_channels():
    _need_gpu()
    import torch
    from chapsim1ww_b200 import _lib
    lib = _lib.load()
    x = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    # 2048 x 256 x 256 needs 64 * 32 * 256 = 524,288 tiles > 65,536: refused before any access
    rc = lib.chapsim_divmax_noalloc(x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), 2048, 256, 256, 1.0, 1.0,
                                    x.data_ptr(), None)
    assert rc == _lib.ERR_TOO_LARGE if hasattr(_lib, "ERR_TOO_LARGE") else rc == 9
