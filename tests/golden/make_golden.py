"""Generate the committed golden fixtures for the TG and IO substeps.

Run from the repository root:  python tests/golden/make_golden.py

The fixtures come from the independent numpy restatements in numpy_tg.py
(FFT circulant solves and banded LU instead of the reference's Thomas
sweeps) and numpy_io.py (complex FFTs and banded LU instead of FISHPACK's
real transforms and TRID0 sweeps; batched dense LU instead of TDMAIJI_CYC and
TDMAIJJ_nonCYC for the semi-implicit scheme's factor solves), so they pin the
C++ oracle and the CUDA library against a second implementation of the same
algorithm.  The
reference itself (Fortran + MPI) cannot be built in this environment and
ships no golden data.
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from numpy_io import IO  # noqa: E402
from numpy_tg import TG  # noqa: E402

CASES = {
    # name: (nx, ny, nz, lx, lz, ren, dt, seed, amp, steps)
    "tg_16x12x8_seed0": (16, 12, 8, 4 * math.pi, 4 * math.pi / 3, 2800.0, 1e-3, 0, 0.1, 2),
    "tg_24x16x12_seed5": (24, 16, 12, 2 * math.pi, math.pi, 1500.0, 2e-3, 5, 0.1, 1),
}

IO_CASES = {
    # name: (nx, ny, nz, lx, lz, ren, dt, seed, amp, steps, thermal, prt, qw_bot, qw_top[, visc_scheme])
    "io_16x12x8_seed3": (16, 12, 8, 4 * math.pi, 4 * math.pi / 3, 2800.0, 1e-3, 3, 0.1, 2, 0, 0.71, 0.0, 0.0),
    "io_heated_16x10x8_seed7": (16, 10, 8, 8 * math.pi, 4 * math.pi / 3, 2000.0, 2e-3, 7, 0.1, 2, 1, 0.71, 1.0, 0.6),
    # the semi-implicit viscous scheme (visthemflg = 1)
    "io_si_16x12x8_seed3": (16, 12, 8, 4 * math.pi, 4 * math.pi / 3, 1500.0, 2e-3, 3, 0.1, 2, 0, 0.71, 0.0, 0.0, 1),
    "io_si_heated_16x10x8_seed7": (16, 10, 8, 8 * math.pi, 4 * math.pi / 3, 2000.0, 2e-3, 7, 0.1, 2, 1, 0.71, 1.0,
                                   0.6, 1),
}


def run_case(nx, ny, nz, lx, lz, ren, dt, seed, amp, steps):
    t = TG(nx, ny, nz, lx, lz, ren=ren, dt=dt)
    t.init_random(seed, amp)
    out = {"init_u": t.q[1].copy(), "init_v": t.q[2].copy(), "init_w": t.q[3].copy()}
    t.substep(0)
    out.update(ns0_u=t.q[1].copy(), ns0_v=t.q[2].copy(), ns0_w=t.q[3].copy(), ns0_p=t.p.copy())
    for _ in range(steps):
        for ns in (1, 2, 3):
            t.substep(ns)
    out.update(end_u=t.q[1].copy(), end_v=t.q[2].copy(), end_w=t.q[3].copy(), end_p=t.p.copy(),
               end_h0u=t.h0[1].copy(), end_h0v=t.h0[2].copy(), end_h0w=t.h0[3].copy(),
               end_divmax=np.array(t.divmax()), end_bulk=np.array(t.bulk()))
    return out


def run_io_case(nx, ny, nz, lx, lz, ren, dt, seed, amp, steps, thermal, prt, qw_bot, qw_top, visc_scheme=0):
    """Initial field + CALC_INITIALIZATION_io (the state after NS = 0), then
    `steps` full RK3 steps."""
    t = IO(nx, ny, nz, lx, lz, ren=ren, dt=dt, thermal=thermal, prt=prt, qw=(qw_bot, qw_top), visc_scheme=visc_scheme)
    t.init_random(seed, amp)
    out = {"ns0_gx": t.g[1].copy(), "ns0_gy": t.g[2].copy(), "ns0_p": t.p.copy()}
    for _ in range(steps):
        for ns in (1, 2, 3):
            t.substep(ns)
    out.update(end_gx=t.g[1].copy(), end_gy=t.g[2].copy(), end_gz=t.g[3].copy(), end_p=t.p.copy(),
               end_u=t.q[1].copy(), end_ex0x=t.ex0[1].copy(), end_divmax=np.array(t.divmax()),
               end_bulk_g=np.array(t.bulk_of(t.g[1])))
    if thermal:
        out.update(end_h=t.h.copy(), end_rho=t.D.copy(), end_mu=t.mu.copy(), end_rhse0=t.rhse0.copy())
    return out


def main():
    for name, args in CASES.items():
        out = run_case(*args)
        meta = np.array(args, dtype=np.float64)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), meta=meta, **out)
        print(name, "divmax", float(out["end_divmax"]), "bulk", float(out["end_bulk"]))
    for name, args in IO_CASES.items():
        out = run_io_case(*args)
        meta = np.array(args, dtype=np.float64)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), meta=meta, **out)
        print(name, "divmax", float(out["end_divmax"]), "bulk G", float(out["end_bulk_g"]))


if __name__ == "__main__":
    main()
