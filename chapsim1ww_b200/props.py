"""Thermal property engine: THERM_PROP_UPDATE on the GPU (table cubic
splines) and the learned property model (MLP h -> T, rho, mu, k, cp).

``PropertyEngine.update(h, ...)`` mirrors THERM_PROP_UPDATE(IREGION)
(src/THERM_PROP_UPDATE.f90:129-205 of the CHAPSim1WW reference) on device
arrays: h -> T by the H-spline, then mu, k, rho by the T-splines; cells with
|h| < 1e-10 are left unchanged, as in the reference; cells outside the table
are left unchanged and reported (the reference STOPs).

``synthetic_table(n)`` builds the non-dimensional table of the heated IO
configuration: h in [-1, 1], cp = 1 + 8 exp(-(h/0.1)^2), T = int_{-1}^h dh/cp,
rho = 1/(1+2T), mu = k = rho^-1/2.
"""
import ctypes

import numpy as np

from . import _lib
from .solver import ChapsimError

NPARAM = 64 + 64 + 64 * 64 + 64 + 5 * 64 + 5
NBASE = 6  # the model's polynomial base per output: degree 5 in x = (h - hmid) / hhalf
NNORM = 2 + 2 * 5 + 5 * NBASE  # hmid, hhalf, mean[5], std[5], base[5][6]


def synthetic_table(n=4096):
    """Columns H, T, D, M, K, CP of the synthetic table (FP64, host).

    T is integrated from the table's lower end, T(-1) = 0: taken from h = 0
    instead, T(-1) = -0.87 and 1 + 2T < 0 below h of about -0.55, i.e. a
    negative density and an undefined viscosity.
    """
    H = np.linspace(-1.0, 1.0, n)
    xg, wg = np.polynomial.legendre.leggauss(8)
    sub = 8  # Gauss-Legendre panels per table interval
    edges = np.linspace(0.0, 1.0, sub + 1)
    lo = H[:-1, None] + (H[1:, None] - H[:-1, None]) * edges[None, :-1]
    hi = H[:-1, None] + (H[1:, None] - H[:-1, None]) * edges[None, 1:]
    mid, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
    pts = mid[:, :, None] + half[:, :, None] * xg[None, None, :]
    f = 1.0 / (1.0 + 8.0 * np.exp(-(pts / 0.1) ** 2))
    cell = np.sum(half[:, :, None] * wg[None, None, :] * f, axis=(1, 2))
    T = np.concatenate([[0.0], np.cumsum(cell)])
    D = 1.0 / (1.0 + 2.0 * T)
    M = D ** -0.5
    K = M.copy()
    CP = 1.0 + 8.0 * np.exp(-(H / 0.1) ** 2)
    return H, T, D, M, K, CP


class PropertyEngine:
    def __init__(self, H, T, D, M, K, CP, device=0):
        self.lib = _lib.load()
        cols = [np.ascontiguousarray(c, dtype=np.float64) for c in (H, T, D, M, K, CP)]
        self._cols = cols
        h = ctypes.c_void_p()
        rc = self.lib.chapsim_props_create(*[c.ctypes.data for c in cols], len(cols[0]), device, ctypes.byref(h))
        if rc != _lib.CHAPSIM_OK:
            raise ChapsimError(rc, "chapsim_props_create failed")
        self.h = h

    def _chk(self, rc):
        if rc != _lib.CHAPSIM_OK:
            raise ChapsimError(rc, self.lib.chapsim_props_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.chapsim_props_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update_device(self, mode, h_ptr, T_ptr, rho_ptr, mu_ptr, k_ptr, cp_ptr, n, raise_on_range=True):
        bad = ctypes.c_int64()
        rc = self.lib.chapsim_props_update(self.h, mode, h_ptr, T_ptr, rho_ptr, mu_ptr, k_ptr, cp_ptr, n,
                                           ctypes.byref(bad))
        if rc == _lib.ERR_RANGE and not raise_on_range:
            return bad.value
        self._chk(rc)
        return bad.value

    def update(self, h, T, rho, mu, k, cp=None, mode=_lib.PROPS_TABLE, raise_on_range=True):
        """torch CUDA float64 tensors (updated in place)."""
        return self.update_device(mode, h.data_ptr(), T.data_ptr(), rho.data_ptr(), mu.data_ptr(), k.data_ptr(),
                                  cp.data_ptr() if cp is not None else None, h.numel(), raise_on_range)

    def train(self, nsamples=65536, seed=2, steps=20000, lr=3e-3):
        loss = ctypes.c_double()
        self._chk(self.lib.chapsim_props_train(self.h, nsamples, seed, steps, lr, ctypes.byref(loss)))
        return loss.value

    def gate(self, tol=1e-4, nbins=256):
        """Judge the model per h-bin and output against the table; returns the
        number of bins where T, rho, mu and k all pass and their worst error."""
        nb = ctypes.c_int()
        worst = ctypes.c_double()
        self._chk(self.lib.chapsim_props_gate(self.h, tol, nbins, ctypes.byref(nb), ctypes.byref(worst)))
        return nb.value, worst.value

    def gate_outputs(self):
        """Per output (T, rho, mu, k, cp) of the last gate call: bins passing
        and worst relative error."""
        bins = (ctypes.c_int * 5)()
        errs = (ctypes.c_double * 5)()
        self._chk(self.lib.chapsim_props_gate_outputs(self.h, bins, errs, 5))
        return list(bins), list(errs)

    def get_params(self):
        p = np.zeros(NPARAM, dtype=np.float32)
        nm = np.zeros(NNORM)
        self._chk(self.lib.chapsim_props_get_params(self.h, p.ctypes.data, NPARAM, nm.ctypes.data, NNORM))
        return p, nm

    def set_params(self, p, norm):
        p = np.ascontiguousarray(p, dtype=np.float32)
        norm = np.ascontiguousarray(norm, dtype=np.float64)
        self._chk(self.lib.chapsim_props_set_params(self.h, p.ctypes.data, NPARAM, norm.ctypes.data, NNORM))

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(NPARAM, dtype=np.float32)
        loss = ctypes.c_double()
        self._chk(self.lib.chapsim_props_loss_grad(self.h, x.ctypes.data, t.ctypes.data, len(x), ctypes.byref(loss),
                                                   g.ctypes.data, NPARAM))
        return loss.value, g
