"""Batched TG channels of uneven sizes (no reference counterpart: the
reference advances one domain per job).

``ChannelBatch`` wraps chapsim_batch_*: every channel is a full TG context;
``step(n)`` replays one captured CUDA graph per time step holding all
channels' substeps as parallel branches; ``autotune()`` picks each channel's
launch shapes by timing.  ``batch64_configs(seed)`` draws the 64-channel
configuration: Nx, Nz in 32..192 step 16, Ny in 32..128 step 16,
Re_b in [2000, 6000], Lx = 4 pi, Lz = 4 pi / 3, dt = 1e-3.
"""
import ctypes
import math

from . import _lib
from .solver import ChapsimError, TGChannel, default_config

M64 = (1 << 64) - 1


def _splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def _uniform(seed, i):
    return (_splitmix64(_splitmix64(seed) ^ i) >> 11) * (1.0 / 9007199254740992.0)


def batch64_configs(seed=3, n=64):
    cfgs = []
    for c in range(n):
        nx = 32 + 16 * int(_uniform(seed, 4 * c) * 11)
        ny = 32 + 16 * int(_uniform(seed, 4 * c + 1) * 7)
        nz = 32 + 16 * int(_uniform(seed, 4 * c + 2) * 11)
        re = 2000.0 + 4000.0 * _uniform(seed, 4 * c + 3)
        cfgs.append(dict(nx=nx, ny=ny, nz=nz, ren=re, lx=4 * math.pi, lz=4 * math.pi / 3, dt=1e-3))
    return cfgs


class _ChannelView(TGChannel):
    """A channel owned by a batch (not destroyed on close)."""

    def __init__(self, lib, handle, cfg):
        self.lib = lib
        self.h = handle
        self.cfg = cfg
        self.nx, self.ny, self.nz = cfg.nx, cfg.ny, cfg.nz
        self.n = lib.chapsim_field_len(handle)

    def close(self):
        self.h = None


class ChannelBatch:
    def __init__(self, cfgs, precision=_lib.FP64, device=0):
        self.lib = _lib.load()
        arr = (_lib.ChapsimConfig * len(cfgs))()
        for i, c in enumerate(cfgs):
            arr[i] = default_config(**c, precision=precision, device=device)
        self._cfgs = arr
        h = ctypes.c_void_p()
        rc = self.lib.chapsim_batch_create(arr, len(cfgs), ctypes.byref(h))
        if rc != _lib.CHAPSIM_OK:
            raise ChapsimError(rc, "chapsim_batch_create failed")
        self.h = h
        self.cells = sum(c["nx"] * c["ny"] * c["nz"] for c in cfgs)
        self.channels = []
        for i in range(len(cfgs)):
            ch = ctypes.c_void_p()
            self._chk(self.lib.chapsim_batch_channel(self.h, i, ctypes.byref(ch)))
            self.channels.append(_ChannelView(self.lib, ch, arr[i]))

    def _chk(self, rc):
        if rc != _lib.CHAPSIM_OK:
            raise ChapsimError(rc, self.lib.chapsim_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            for c in self.channels:
                c.close()
            self.lib.chapsim_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_random(self, seed=3, amp=0.1, project=True):
        self._chk(self.lib.chapsim_batch_init_random(self.h, seed, amp, 1 if project else 0))

    def autotune(self, reps=3):
        self._chk(self.lib.chapsim_batch_autotune(self.h, reps))

    def step(self, n=1):
        self._chk(self.lib.chapsim_batch_step(self.h, n))

    def sync(self):
        self._chk(self.lib.chapsim_batch_sync(self.h))

    def stream(self):
        s = ctypes.c_void_p()
        self._chk(self.lib.chapsim_batch_get_stream(self.h, ctypes.byref(s)))
        return s.value

    def kernels_per_step(self):
        n = ctypes.c_int64()
        self._chk(self.lib.chapsim_batch_kernels_per_step(self.h, ctypes.byref(n)))
        return n.value
