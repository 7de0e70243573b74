"""Failure path of the bounded device waits.

Every mbarrier wait in the library gives up after a spin limit, records a
code in the context's device error word and returns, so a lost transfer ends
as an error status instead of a hung GPU (the reference's failure path is
ERRHDL's print-and-STOP, src/WRTHDL.f90:18-30).  The hook
chapsim_inject_wait_timeout runs that give-up path on purpose: one kernel
waits, with a spin limit of 1,024 polls, on an mbarrier nothing completes.
Nothing faults, traps or hangs: the wait runs out in microseconds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_wait_timeout_reported_then_context_recovers():
    _need_gpu()
    from chapsim1ww_b200 import ChapsimError, TGChannel
    from chapsim1ww_b200._lib import ERRORS
    a = TGChannel(32, 24, 16)
    b = TGChannel(32, 24, 16)
    for s in (a, b):
        s.random_fl_fld_tg(5, 0.1, project=True)
        s.step(1)
        s.sync()
    assert a.lib.chapsim_inject_wait_timeout(a.h, 1024) == 0
    with pytest.raises(ChapsimError) as ei:
        a.sync()
    assert ERRORS[ei.value.code] == "CHAPSIM_ERR_CUDA"
    assert "wait gave up" in str(ei.value)
    # the word was cleared when it was reported: the context works again and
    # its next steps equal those of a context that never saw the timeout
    a.sync()
    a.step(2)
    b.step(2)
    a.sync()
    for n in ("u", "v", "w", "p"):
        assert np.array_equal(a.get_field(n), b.get_field(n)), n


def test_wait_timeout_hook_rejects_bad_limits():
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    a = TGChannel(32, 24, 16)
    assert a.lib.chapsim_inject_wait_timeout(a.h, 0) == 1
    assert a.lib.chapsim_inject_wait_timeout(a.h, (1 << 20) + 1) == 1
    a.sync()
