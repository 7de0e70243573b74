"""CPU checks of the C ABI library: it loads, it exports every symbol that
include/chapsim.h declares, its config struct matches, and it fails loudly
(no CPU fallback) when no GPU is present."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "chapsim.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(chapsim_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from chapsim1ww_b200 import _lib
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(syms) <= bound, set(syms) - bound


def test_config_struct_layout():
    from chapsim1ww_b200 import _lib
    lib = _lib.load()
    cfg = _lib.ChapsimConfig()
    assert lib.chapsim_config_default(ctypes.byref(cfg)) == 0
    assert cfg.struct_size == ctypes.sizeof(_lib.ChapsimConfig)
    assert (cfg.nx, cfg.ny, cfg.nz) == (64, 64, 64)
    assert abs(cfg.ren - 2800.0) < 1e-12 and cfg.istr2 == 1


def test_create_validates_before_touching_a_device():
    from chapsim1ww_b200 import _lib
    lib = _lib.load()
    cfg = _lib.ChapsimConfig()
    lib.chapsim_config_default(ctypes.byref(cfg))
    h = ctypes.c_void_p()
    cfg.nx = 7  # odd lengths are rejected
    assert lib.chapsim_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    lib.chapsim_config_default(ctypes.byref(cfg))
    cfg.struct_size = 4
    assert lib.chapsim_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert lib.chapsim_destroy(None) == 1
    assert lib.chapsim_sync(None) == 1
    assert lib.chapsim_set_field_async(None, 0, 0, None, 0) == 1
    assert lib.chapsim_get_field_async(None, 0, 0, None, 0) == 1


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from chapsim1ww_b200 import ChapsimError, TGChannel
    with pytest.raises(ChapsimError) as e:
        TGChannel(16, 12, 8)
    assert "NODEVICE" in str(e.value)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from chapsim1ww_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libchapsim.so"))
    with pytest.raises(RuntimeError):
        _lib.load()


def test_header_cites_reference_routines():
    text = open(HEADER).read()
    for name in ("SOLVERRK3_MOM_tg", "FFT99_POIS3D_periodicxz", "VELOUPDT_tg", "DIVG_tg", "DIVGCK_tg"):
        assert name in text
