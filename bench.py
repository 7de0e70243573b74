"""Benchmark of the CHAPSim RK3 step on B200 (libchapsim, sm_100a).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--precision fp64|mixed]

A "step" is one full RK3 time step (substeps NS = 1, 2, 3) of the workload.
Metric: cell-steps/s = cells x steps / seconds.

Default workload (c4_mixed_learned): the metric's comparison on the large
single domain, io_1024x384x512 (201 M cells, Lx = 8 pi, Lz = 2 pi, tanh
stretching beta = 2, Re_b = 10,000, dt = 1e-3, heated with the synthetic
4096-point property table, wall heat flux 1, Pr 0.71, seed 4).  The plain
FP64 form with the table splines and the learned form (the property model,
trained on the GPU on 65,536 table samples, seed 2, gated at 1e-4 over 256
h-bins, in place of the splines; FP64 Poisson spectra, or with --spectra fp32
the mixed form's FP32 spectra plus one FP64-residual refinement sweep)
advance the same seeded state; `value` is the learned form's cell-steps/s,
the FP64 form's figure and their ratio ride along, with the learned form's
error against the FP64 form at full size.
Synthetic seeded initial fields (no public dataset is involved).  With N > 1
GPUs every rank advances its own independent copy (replicas, weak scaling,
no data-path collective); timing is the max over ranks.  Other workloads:
c2_mixed_learned (the same comparison on the heated 384x192x192 channel),
c1_tg_io (the TG channel 256x192x256 feeding the inlet of the IO section
512x192x256, Lx = 8 pi, with constant-property passive heat and a convective
outlet: BCX_io = 2, 1, the coupled step of SOLVE's substep loop), the TG or IO
section alone, the heated IO channel with the semi-implicit viscous scheme,
the 64-channel batch (split across ranks), the CPU-sized 64^3 TG channel.

Arms:
  ours       libchapsim through the C ABI; `value` with the state resident in
             HBM (CUDA-graph replay of the steps), `e2e` through the public API
             with host buffers (upload the state fields from pinned memory,
             one step, download them and max|div| every step).
  reference  the reference algorithm's CPU path: the FP64 oracle port
             (OpenMP, all host threads) on the same workload, rank 0 only.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # TG section of the coupled TG+IO configuration
    "tg_256x192x256": dict(nx=256, ny=192, nz=256, lx=4 * math.pi, lz=4 * math.pi / 3, ren=2800.0, dt=1e-3, seed=1),
    # 64 independent TG channels of uneven sizes (seed 3), mixed precision
    "batch64": dict(batch=True, seed=3),
    # the CPU-runnable plain-method configuration
    "tg_64x64x64": dict(nx=64, ny=64, nz=64, lx=4 * math.pi, lz=4 * math.pi / 3, ren=2800.0, dt=1e-3, seed=0),
    # variable-property heated IO channel, x-periodic, synthetic 4096-point table
    "io_384x192x192": dict(io=True, nx=384, ny=192, nz=192, lx=8 * math.pi, lz=4 * math.pi / 3, ren=2800.0,
                           dt=1e-3, seed=2, thermal=1, prt=0.71, qw=1.0, table="synthetic"),
    # large single domain: 1024x384x512 (201 M cells), Lx = 8 pi, Lz = 2 pi,
    # Re 10,000, heated with the synthetic table; the CPU port times a 32-plane
    # z-slab of it (the same work per cell; a full oracle step needs ~65 GB)
    "io_1024x384x512": dict(io=True, nx=1024, ny=384, nz=512, lx=8 * math.pi, lz=2 * math.pi, ren=10000.0,
                            dt=1e-3, seed=4, thermal=1, prt=0.71, qw=1.0, table="synthetic", cpu_nz=32),
    # the same channel with the semi-implicit viscous scheme (visthemflg = 1)
    "io_384x192x192_si": dict(io=True, nx=384, ny=192, nz=192, lx=8 * math.pi, lz=4 * math.pi / 3, ren=2800.0,
                              dt=1e-3, seed=2, thermal=1, prt=0.71, qw=1.0, table="synthetic", visc_scheme=1),
    # the metric's comparison on the large single domain: the mixed precision
    # form with the learned property model against the plain FP64 form with
    # the table splines, both on io_1024x384x512 (201 M cells)
    "c4_mixed_learned": dict(compare=True, base="io_1024x384x512"),
    # the same comparison on the heated 384x192x192 channel
    "c2_mixed_learned": dict(compare=True, base="io_384x192x192"),
    # the coupled TG + IO configuration: the TG section feeds the IO section's
    # inlet (BCX_io = 2, 1: Neumann inlet, Dirichlet outlet, convective outflow)
    "c1_tg_io": dict(pair=True, tg="tg_256x192x256", io="io_512x192x256", bcx=(2, 1)),
    # IO section of the coupled configuration (alone: x-periodic): constant-property
    # passive heat (rho = mu = k = cp = 1, T = h), wall heat flux 1, Pr 0.71
    "io_512x192x256": dict(io=True, nx=512, ny=192, nz=256, lx=8 * math.pi, lz=4 * math.pi / 3, ren=2800.0,
                           dt=1e-3, seed=1, thermal=1, prt=0.71, qw=1.0, table="constant"),
}
METRIC = "cell-steps/s"

# Algorithmic HBM bytes per launch of each phase kernel, FP64 form, in units
# of 8-byte values per cell (spectral phases: per complex spectral value).
PHASE_VALUES_PER_CELL = {"rhs": 13, "adix": 6, "adiz": 6, "adiy": 9, "fftx": 4, "corr": 10}
PHASE_SPECTRAL_PASSES = {"fftx": 1, "fftz": 2, "ysolve": 2, "ifftz": 2, "ifftx": 1}
PHASE_KERNEL = {"rhs": "k_rhs_tma", "adix": "k_adixz_row", "adiz": "k_adixz_row", "adiy": "k_adiy_band",
                "fftx": "k_fftx", "fftz": "k_fftz", "ysolve": "k_ysolve_line", "ifftz": "k_fftz", "ifftx": "k_ifftx",
                "corr": "k_corr"}


# IO substep phases (the library's IO timer slots, in execution order) and
# their algorithmic 8-byte values per cell (thermal form): energy RHS reads
# h, T, k, G, G0, rho h, R0 and writes rho h, R0; the property update reads
# rho h, rho, mu and writes mu0, rho0, rho, h, T, mu, k, mu0 + mu; prep reads G, G0,
# rho, rho0 and writes u, v, w, DrhoDtP; the momentum RHS reads u, v, w, G,
# mu, mu0, p, EXPLT0 and writes EXPLT0 and G*; the x-transform reads G* and
# DrhoDtP and writes RHSLLPHI; the correction reads G*, phi, p and writes G, p.
IO_PHASES = ["eng_rhs", "eng_props", "prep", "mom_rhs", "fftx", "fftz", "ysolve", "ifftz", "ifftx", "corr"]
IO_VALUES_PER_CELL = {"eng_rhs": 13, "eng_props": 11, "prep": 12, "mom_rhs": 17, "fftx": 5, "corr": 9}
IO_KERNEL = {"eng_rhs": "k_io_eng_rhs", "eng_props": "k_io_eng_props", "prep": "k_io_prep",
             "mom_rhs": "k_io_rhs_tma", "fftx": "k_fftx", "fftz": "k_fftz", "ysolve": "k_ysolve_line",
             "ifftz": "k_fftz", "ifftx": "k_ifftx", "corr": "k_io_corr"}


# Semi-implicit scheme: the momentum phase is k_io_rhs_si (u, v, w, p, G x3,
# mu, mu0, DRHOI x3 read; EXPLT0 x3 read and written; RHS x3 written: 21
# values) and the nine MOMFA line solves (per component and direction RHS in
# and out plus the four property fields of the coefficients; the y solves
# also read G and write G*): 78 values per cell with the energy equation on.
IO_SI_MOM_VALUES = {1: 78, 0: 37}
IO_SI_KERNEL = "k_si_stg + k_io_rhs_si + MOMFA solves (k_si_x, k_si_zy)"


# End-to-end transfers of an IO step.  Its inputs are the mass flux G, the
# pressure and rho h (with the device-resident properties and old-substep
# terms); u, v, w are results: VELOCITY_CALC_io rebuilds them from G and the
# density at every cell before each substep's momentum stage
# (src/SOLVE.f90:131-132), and the energy stage does not read them.
IO_INPUT_FIELDS = ("gx", "gy", "gz", "p", "rhoh")
IO_RESULT_FIELDS = ("u", "v", "w", "p", "gx", "gy", "gz", "rhoh")


def io_phase_bytes(ph, nx, ny, nz, real_bytes=8, visc=0, thermal=1):
    cells = nx * ny * nz
    spec = (nx // 2 + 1) * ny * nz
    vals = IO_SI_MOM_VALUES[1 if thermal else 0] if (visc and ph == "mom_rhs") else IO_VALUES_PER_CELL.get(ph, 0)
    b = vals * real_bytes * cells
    if ph == "ifftx":
        b += real_bytes * cells
    b += PHASE_SPECTRAL_PASSES.get(ph, 0) * 2 * real_bytes * spec
    return b


def io_table(kind):
    import numpy as np
    if kind == "constant":
        H = np.linspace(-1.0, 1.0, 4096)
        one = np.ones_like(H)
        return H, H.copy(), one, one.copy(), one.copy()
    from chapsim1ww_b200 import synthetic_table
    return synthetic_table(4096)[:5]


def phase_bytes(ph, nx, ny, nz, real_bytes=8):
    cells = nx * ny * nz
    spec = (nx // 2 + 1) * ny * nz
    b = PHASE_VALUES_PER_CELL.get(ph, 0) * real_bytes * cells
    if ph == "ifftx":
        b += real_bytes * cells  # phi written
    b += PHASE_SPECTRAL_PASSES.get(ph, 0) * 2 * real_bytes * spec
    return b


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_bf16_peak():
    """Dense BF16 TFLOP/s: the burst figure (a kernel that runs at the full SM
    clock; the sustained figure is a GEMM held at the power cap)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured (bf16 burst)"
    except Exception:
        return 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws):
    """NCCL process group of the replicas (None on one GPU); the timeout
    bounds any rank that waits for a rank that died."""
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist


def dist_done(pg):
    if pg is not None:
        pg.destroy_process_group()


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, local, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def load_traffic(workload, kernel):
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d.get(workload, {}).get(kernel)
    except Exception:
        return None


def bench_learned(cells, device):
    """THERM_PROP_UPDATE on one field of the workload's size: the table
    splines against the learned model (MLP 1->64->64->5, trained on the GPU on
    65,536 samples of the synthetic 4096-point table, seed 2; BF16 tensor-core
    inference), with the error gate at 1e-4 relative."""
    import torch

    from chapsim1ww_b200 import PropertyEngine, synthetic_table
    eng = PropertyEngine(*synthetic_table(4096), device=device)
    t0 = time.perf_counter()
    loss = eng.train(65536, 2, 8000, 3e-3)
    t_train = time.perf_counter() - t0
    g = torch.Generator(device=f"cuda:{device}").manual_seed(5)
    h = torch.rand(cells, dtype=torch.float64, device=f"cuda:{device}", generator=g) * 1.998 - 0.999
    outs = [torch.zeros(cells, dtype=torch.float64, device=f"cuda:{device}") for _ in range(5)]

    def timed(mode, reps=10):
        eng.update(h, *outs[:4], cp=outs[4], mode=mode)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            eng.update(h, *outs[:4], cp=outs[4], mode=mode)
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / reps

    table_ms = timed(0)
    eng.gate(1e9, 256)
    mlp_ms = timed(1)
    nbins, worst = eng.gate(1e-4, 256)
    gated_ms = timed(1)
    eng.close()
    return {"train_loss": loss, "train_s": t_train, "train_steps": 8000, "gate_tol": 1e-4,
            "mlp_bins": nbins, "bins": 256, "mlp_max_rel_err": worst,
            "table_update_ms": table_ms, "mlp_update_ms": mlp_ms, "gated_update_ms": gated_ms,
            "cells": cells}


def cpu_baseline_io(wl, steps):
    """FP64 IO oracle port on the host cores: init + projection, then `steps` timed steps."""
    from oracle.pyoracle import OracleIO, get_threads
    nz = wl.get("cpu_nz", wl["nz"])  # z-slab of the workload (same cell size) when set
    o = OracleIO(wl["nx"], wl["ny"], nz, lx=wl["lx"], lz=wl["lz"] * nz / wl["nz"], ren=wl["ren"], dt=wl["dt"],
                 thermal=wl["thermal"], prt=wl["prt"], qw=(wl["qw"], wl["qw"]), table=io_table(wl["table"]),
                 visc_scheme=wl.get("visc_scheme", 0))
    o.init_random(wl["seed"], 0.1)
    t0 = time.perf_counter()
    o.step(steps)
    t = time.perf_counter() - t0
    cells = wl["nx"] * wl["ny"] * nz
    return cells * steps / t, t, get_threads()


def run_io(args, wl, ws, rank, local):
    """IO channel section: one step = NS 1, 2, 3 of SOLVERRK3_ENG_IO + SOLVERRK3_MOM_IO."""
    import torch

    from chapsim1ww_b200 import IOChannel

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    s = IOChannel(wl["nx"], wl["ny"], wl["nz"], lx=wl["lx"], lz=wl["lz"], ren=wl["ren"], dt=wl["dt"],
                  thermal=wl["thermal"], prt=wl["prt"], qw=(wl["qw"], wl["qw"]), table=io_table(wl["table"]),
                  device=local, visc_scheme=wl.get("visc_scheme", 0))
    s.random_fl_theml_fld_io(wl["seed"] + rank, 0.1)
    cells = wl["nx"] * wl["ny"] * wl["nz"]
    stream = torch.cuda.ExternalStream(s.stream(), device=local)

    def barrier():
        if pg is not None:
            pg.barrier()

    def max_over_ranks(x):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    s.step(args.warmup)
    s.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = s.launch_count()
    e0.record(stream)
    s.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    launches = s.launch_count() - n0
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = cells * ws * args.steps / (ms / 1000.0)
    divmax = s.divgck_io()
    bad = s.bad_cells()

    s.phase_timing(True)
    s.phase_reset()
    s.step(max(1, min(args.steps, 10)))
    ph, nsub = s.phase_times()
    s.phase_timing(False)
    per_launch = {IO_PHASES[i]: v / max(nsub, 1) for i, v in enumerate(ph.values())}
    dom = max(per_launch, key=per_launch.get)
    peak, peak_kind = measured_peak()
    nx, ny, nz = wl["nx"], wl["ny"], wl["nz"]
    visc = wl.get("visc_scheme", 0)
    kernel_dom = IO_SI_KERNEL if (visc and dom == "mom_rhs") else IO_KERNEL[dom]
    bytes_dom = io_phase_bytes(dom, nx, ny, nz, visc=visc, thermal=wl["thermal"])
    achieved = bytes_dom / (per_launch[dom] / 1000.0) / 1e9
    total_bytes = sum(io_phase_bytes(p, nx, ny, nz, visc=visc, thermal=wl["thermal"]) for p in IO_PHASES)
    traffic = None if visc else load_traffic(args.workload, IO_KERNEL[dom])

    names, inputs = IO_RESULT_FIELDS, IO_INPUT_FIELDS
    host = {}
    for n in names:
        t = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
        host[n] = t.numpy()
        s.get_field(n, out=host[n])
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 10))
    e2.record(stream)
    for _ in range(e2e_steps):
        for n in inputs:
            s.set_field_async(n, host[n])
        s.step(1)
        for n in names:
            s.get_field_async(n, out=host[n])
        _ = s.divgck_io()
    e3.record(stream)
    e3.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3))
    e2e_value = cells * ws * e2e_steps / (ms_e2e / 1000.0)
    h2d = len(inputs) * s.n * 8
    nbytes = len(names) * s.n * 8

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            v, t, cores = cpu_baseline_io(wl, args.cpu_steps)
            slab = (f" (a {wl['cpu_nz']}-plane z-slab, same cell size)" if wl.get("cpu_nz") else "")
            cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
                   "sample": f"{args.cpu_steps} full RK3 steps of the {args.workload} channel{slab} after init, "
                             f"FP64 oracle port, OpenMP {cores} threads, {t:.1f} s"}
        except Exception as ex:
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded splitmix64 velocity, h = 0, table properties, NS=0 projection)",
            "config": workload_config(args, wl),
            "arm": {"parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                    "l2": "working set (>2 GB) larger than the 126 MB L2"},
            "max_div_g_plus_drho": divmax, "out_of_table_cells": bad,
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": nbytes + 8, "steps": e2e_steps,
                    "uploaded": list(inputs), "downloaded": list(names)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kernel_dom, "phase": dom,
                         "algorithmic_bytes_per_launch": bytes_dom, "avg_launch_ms": per_launch[dom],
                         "peak_source": peak_kind},
            "phases_ms_per_launch": per_launch,
            "step_roofline": {"algorithmic_bytes_per_step": 3 * total_bytes,
                              "achieved_gbs": 3 * total_bytes / (ms / args.steps / 1000.0) / 1e9,
                              "frac": 3 * total_bytes / (ms / args.steps / 1000.0) / 1e9 / peak,
                              "phase_sum_ms": 3 * sum(per_launch.values())},
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def run_compare(args, wl, ws, rank, local):
    """The metric's comparison: the same IO channel advanced by the plain FP64
    form (table splines) and by the learned form (the property model on the
    tensor cores in place of the splines; FP64 Poisson spectra, or FP32
    spectra with an FP64-residual refinement sweep when args.spectra is
    "fp32"), K graph-replayed steps each after W warm-up steps, both from
    the same seeded state.  value = the learned form's cell-steps/s; the
    FP64 form's figure, their ratio, the property model's gate and the
    learned form's error against the FP64 form at full size (u, p, T,
    max |div|) ride along."""
    import torch

    import chapsim1ww_b200 as cs
    from chapsim1ww_b200 import IOChannel, PropertyEngine

    b = WORKLOADS[wl["base"]]
    torch.cuda.set_device(local)
    pg = dist_init(ws)
    nx, ny, nz = b["nx"], b["ny"], b["nz"]
    cells = nx * ny * nz
    table = io_table(b["table"])

    def make(precision):
        ch = IOChannel(nx, ny, nz, lx=b["lx"], lz=b["lz"], ren=b["ren"], dt=b["dt"], thermal=1, prt=b["prt"],
                       qw=(b["qw"], b["qw"]), table=table, device=local, precision=precision)
        return ch

    def timed_steps(ch, n):
        stream = torch.cuda.ExternalStream(ch.stream(), device=local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ch.step(n)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    # ---- the plain FP64 form (table splines)
    ref = make(cs.FP64)
    ref.random_fl_theml_fld_io(b["seed"] + rank, 0.1)
    ref.step(args.warmup)
    ref.sync()
    barrier(pg)
    torch.cuda.synchronize()
    ms64 = max_over_ranks(pg, local, timed_steps(ref, args.steps))
    div64 = ref.divgck_io()

    # ---- the learned property model: trained on the GPU, gated at 1e-4
    t0 = time.perf_counter()
    eng = PropertyEngine(*synthetic_table_cols(table), device=local)
    loss = eng.train(65536, 2, 20000, 3e-3)
    t_train = time.perf_counter() - t0
    nbins, worst = eng.gate(1e-4, 256)
    out_bins, out_err = eng.gate_outputs()

    # ---- the mixed form with the learned properties
    mix = make(cs.MIXED if args.spectra == "fp32" else cs.FP64)
    mix.set_refinement(args.refine)
    mix.set_props_mode(1, eng)
    mix.random_fl_theml_fld_io(b["seed"] + rank, 0.1)
    mix.step(args.warmup)
    mix.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    torch.cuda.synchronize()
    n0 = mix.launch_count()
    ms = max_over_ranks(pg, local, timed_steps(mix, args.steps))
    torch.cuda.synchronize()
    barrier(pg)
    launches = mix.launch_count() - n0
    clk = clocks.stop()
    value = cells * ws * args.steps / (ms / 1000.0)
    value64 = cells * ws * args.steps / (ms64 / 1000.0)
    divmix = mix.divgck_io()
    bad = mix.bad_cells()
    again = mix.model_again_tiles()

    # error of the learned form against the FP64 form after the same
    # W + K steps from the same state (on the device)
    def field(ch, name):
        t = torch.empty(ch.shape, dtype=torch.float64, device=f"cuda:{local}")
        ch.get_field_device(name, t.data_ptr())
        ch.sync()  # the copy is ordered on the context's stream, not torch's
        return t

    errors = {}
    for name in ("u", "v", "w", "p", "gx", "t", "rho", "mu"):
        a, r = field(mix, name), field(ref, name)
        errors[name] = float((a - r).abs().max() / r.abs().max())
        del a, r
    torch.cuda.empty_cache()
    # per-phase kernel times of the FP64 form (after the error comparison:
    # these steps advance it past the learned form)
    ref.phase_timing(True)
    ref.phase_reset()
    ref.step(max(1, min(args.steps, 5)))
    ph64, nsub64 = ref.phase_times()
    ref.phase_timing(False)
    phases64 = {IO_PHASES[i]: v / max(nsub64, 1) for i, v in enumerate(ph64.values())}
    ref.close()
    del ref

    # per-phase kernel times of the learned form
    mix.phase_timing(True)
    mix.phase_reset()
    mix.step(max(1, min(args.steps, 5)))
    ph, nsub = mix.phase_times()
    mix.phase_timing(False)
    per_launch = {IO_PHASES[i]: v / max(nsub, 1) for i, v in enumerate(ph.values())}
    dom = max(per_launch, key=per_launch.get)
    peak, peak_kind = measured_peak()
    bytes_dom = io_phase_bytes(dom, nx, ny, nz)
    if args.spectra == "fp32" and (dom in PHASE_SPECTRAL_PASSES or dom == "fftx"):
        bytes_dom -= PHASE_SPECTRAL_PASSES.get(dom, 0) * 2 * 4 * (nx // 2 + 1) * ny * nz  # FP32 spectra
    achieved = bytes_dom / (per_launch[dom] / 1000.0) / 1e9
    kern = IO_KERNEL[dom] if dom != "eng_props" else "k_io_eng_props_mlp"
    # the learned-property kernel: one model evaluation per cell with its
    # forward-mode derivative; per 128-cell tile three BF16 hi/lo MMA chains
    # plus one derivative chain for layer 2 (128 x 64 x 64) and for layer 3
    # (128 x 16 x 64); a tile that evaluates the model a second time adds
    # three chains per layer and 128 more tanh per cell
    ntiles = (nx * (ny + 2) * nz + 127) // 128
    again_frac = again / max(1, 3 * (args.warmup + args.steps + 1) * ntiles)
    mlp_flops = ntiles * 128 * 2 * 64 * (64 + 16) * (4 + 3 * again_frac)
    mlp = {"kernel": "k_io_eng_props_mlp", "avg_launch_ms": per_launch["eng_props"],
           "mma_tflops": mlp_flops / (per_launch["eng_props"] / 1000.0) / 1e12,
           "tanh_per_cell": 128 * (1 + again_frac),
           "note": "bound by instruction issue and tensor-memory round trips (the tanh, BF16 hi/lo splits and "
                   "derivative factors between the layers), not by HBM bytes or the tensor pipe"}
    traffic = load_traffic(args.workload, kern)
    hbm_view = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": kern, "phase": dom, "algorithmic_bytes_per_launch": bytes_dom,
                "avg_launch_ms": per_launch[dom], "peak_source": peak_kind}
    if dom == "eng_props":
        # the learned-property kernel sits above the ridge point (its issued
        # MMA flops per HBM byte exceed peak TFLOP/s / peak GB/s): its
        # roofline is the tensor pipe, with the HBM view beside it
        tpk, tpk_kind = measured_bf16_peak()
        roofline = {"bound": "tensor", "achieved": mlp["mma_tflops"], "peak": tpk, "unit": "TFLOP/s",
                    "frac": mlp["mma_tflops"] / tpk, "traffic": traffic, "kernel": kern, "phase": dom,
                    "algorithmic_flops_per_launch": mlp_flops, "avg_launch_ms": per_launch[dom],
                    "peak_source": tpk_kind, "flops": "issued BF16 MMA flops: 3 hi/lo chains + 1 derivative chain "
                    "per layer per 128-cell tile", "hbm_view": hbm_view}
    else:
        roofline = hbm_view

    # ---- end to end through the public API with host buffers
    names, inputs = IO_RESULT_FIELDS, IO_INPUT_FIELDS
    host = {}
    for n in names:
        host[n] = torch.empty(mix.shape, dtype=torch.float64, pin_memory=True).numpy()
        mix.get_field(n, out=host[n])
    barrier(pg)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(mix.stream(), device=local)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 5))
    e2.record(stream)
    for _ in range(e2e_steps):
        for n in inputs:
            mix.set_field_async(n, host[n])
        mix.step(1)
        for n in names:
            mix.get_field_async(n, out=host[n])
        _ = mix.divgck_io()
    e3.record(stream)
    e3.synchronize()
    barrier(pg)
    ms_e2e = max_over_ranks(pg, local, e2.elapsed_time(e3))
    e2e_value = cells * ws * e2e_steps / (ms_e2e / 1000.0)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            v, t, cores = cpu_baseline_io(b, args.cpu_steps)
            slab = f" (a {b['cpu_nz']}-plane z-slab, same cell size)" if b.get("cpu_nz") else ""
            cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
                   "sample": f"{args.cpu_steps} full RK3 steps of the {wl['base']} channel{slab} after init, FP64 "
                             f"oracle port (table splines), OpenMP {cores} threads, {t:.1f} s"}
        except Exception as ex:
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": (f"f64 fields, {args.spectra} Poisson spectra, bf16 hi/lo tensor-core property model "
                      "(f32 accumulate)"),
            "data": "synthetic (seeded splitmix64 velocity, h = 0, synthetic 4096-point table, NS=0 projection)",
            "config": workload_config(args, wl),
            "arm": {"parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                    "l2": "working set (>40 GB) larger than the 126 MB L2"},
            "fp64": {"value": value64, "ms_per_step": ms64 / args.steps, "max_div_g_plus_drho": div64,
                     "form": "plain FP64, table splines", "phases_ms_per_launch": phases64},
            "mixed_form": {"poisson_spectra": args.spectra,
                           "fp64_residual_refinement_sweeps": args.refine if args.spectra == "fp32" else 0},
            "ratio_vs_fp64": value / value64,
            "max_div_g_plus_drho": divmix, "out_of_table_cells": bad,
            "model_second_evaluations": {"tiles": again, "of": 3 * (args.warmup + args.steps + 1) *
                                         ((nx * (ny + 2) * nz + 127) // 128)},
            "error_vs_fp64": {"after_steps": args.warmup + args.steps, "relative_max": errors},
            "property_model": {"train_s": t_train, "train_loss": loss, "gate_tol": 1e-4, "bins": 256,
                               "bins_cleared_T_rho_mu_k": nbins, "max_rel_err_T_rho_mu_k": worst,
                               "bins_cleared_per_output": dict(zip(("T", "rho", "mu", "k", "cp"), out_bins)),
                               "max_rel_err_per_output": dict(zip(("T", "rho", "mu", "k", "cp"), out_err))},
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": len(inputs) * mix.n * 8,
                    "d2h_bytes_per_step": len(names) * mix.n * 8 + 8, "steps": e2e_steps,
                    "uploaded": list(inputs), "downloaded": list(names)},
            "roofline": roofline,
            "learned_property_kernel": mlp,
            "phases_ms_per_launch": per_launch,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    mix.close()
    eng.close()
    dist_done(pg)
    return 0


def synthetic_table_cols(table5):
    """Columns H, T, D, M, K, CP for a property engine: the workload's table
    plus cp = dh/dT of the synthetic table."""
    from chapsim1ww_b200 import synthetic_table
    full = synthetic_table(len(table5[0]))
    return list(table5[:5]) + [full[5]]


# Coupled IO section (x ghost columns, the non-periodic Poisson transforms):
# its phase kernels and algorithmic 8-byte values per cell.  The divergence
# reads G and DrhoDtP and writes RHSLLPHI, which the forward x transform reads
# and writes as nx real modes per row, two to a complex line; the z transforms
# and y-lines pass over nx / 2 complex values per row.
IO_KERNEL_COUPLED = dict(IO_KERNEL, mom_rhs="k_io_rhs_tma (coupled layout)", fftx="k_np_divg + k_xnp_qfwd",
                         ysolve="k_ysolve_pair", ifftx="k_xnp_qbwd")
IO_COUPLED_VALUES = dict(IO_VALUES_PER_CELL, fftx=7, fftz=2, ysolve=2, ifftz=2, ifftx=2)


def io_phase_bytes_coupled(ph, nx, ny, nz):
    return IO_COUPLED_VALUES.get(ph, 0) * 8 * nx * ny * nz


class CoupledOracle:
    """The TG oracle feeding the coupled IO oracle in SOLVE's order (per
    substep: SOLVERRK3_MOM_tg, then the IO section, whose BC_TINLET_FLOW reads
    the TG fields), on z-slabs of nz planes with the sections' mesh spacing."""

    def __init__(self, wt, wi, bcx, nz):
        from oracle.pyoracle import OracleIO
        self.t = make_oracle("tg", wt, nz)
        self.o = OracleIO(wi["nx"], wi["ny"], nz, lx=wi["lx"], lz=wi["lz"] * nz / wi["nz"], ren=wi["ren"],
                          dt=wi["dt"], thermal=wi["thermal"], prt=wi["prt"], qw=(wi["qw"], wi["qw"]),
                          table=io_table(wi["table"]))
        self.o.set_bcx(*bcx)
        self._feed()
        self.o.init_random(wi["seed"], 0.1)

    def _feed(self):
        self.o.set_inlet(*[self.t.get(f) for f in ("u", "v", "w", "p")])

    def step(self, n=1):
        for _ in range(n):
            for ns in (1, 2, 3):
                self.t.substep(ns)
                self._feed()
                self.o.substep(ns)


def run_pair(args, wl, ws, rank, local):
    """Configuration 1: the TG section feeds the inlet of the IO section
    (chapsim_io_set_inlet; BCX_io = 2, 1, convective outlet) and both advance
    by chapsim_step_coupled (SOLVE's substep loop: per substep the TG
    momentum, the IO energy and the IO momentum; one captured graph per step
    on the TG's stream).  value = (TG cells + IO cells) x steps / time."""
    import torch

    import chapsim1ww_b200 as cs
    from chapsim1ww_b200 import IOChannel, TGChannel

    wt, wi = WORKLOADS[wl["tg"]], WORKLOADS[wl["io"]]
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    prec = cs.MIXED if args.precision == "mixed" else cs.FP64
    tg = TGChannel(wt["nx"], wt["ny"], wt["nz"], lx=wt["lx"], lz=wt["lz"], ren=wt["ren"], dt=wt["dt"],
                   precision=prec, device=local)
    io = IOChannel(wi["nx"], wi["ny"], wi["nz"], lx=wi["lx"], lz=wi["lz"], ren=wi["ren"], dt=wi["dt"],
                   thermal=wi["thermal"], prt=wi["prt"], qw=(wi["qw"], wi["qw"]), table=io_table(wi["table"]),
                   device=local, bcx=wl["bcx"])
    io.set_inlet(tg)
    tg.random_fl_fld_tg(wt["seed"] + rank, 0.1, project=True)
    io.random_fl_theml_fld_io(wi["seed"] + rank, 0.1)
    ct, ci = wt["nx"] * wt["ny"] * wt["nz"], wi["nx"] * wi["ny"] * wi["nz"]
    st = torch.cuda.ExternalStream(io.stream(), device=local)  # the TG's stream, shared

    def barrier():
        if pg is not None:
            pg.barrier()

    def max_over_ranks(x):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    def timed(fn, steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn(steps)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def both(n):
        io.step_coupled(tg, n)

    both(args.warmup)
    io.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    n0 = tg.launch_count() + io.launch_count()
    ms = max_over_ranks(timed(both, args.steps))
    torch.cuda.synchronize()
    barrier()
    launches = tg.launch_count() + io.launch_count() - n0
    clk = clocks.stop()
    cells = ct + ci
    value = cells * ws * args.steps / (ms / 1000.0)
    # each section alone (the IO one with its inflow as it stands)
    ms_tg = timed(tg.step, args.steps) / args.steps
    ms_io = timed(io.step, args.steps) / args.steps

    # per-phase kernel times of both sections
    nph = max(1, min(args.steps, 10))
    tg.phase_timing(True)
    tg.phase_reset()
    tg.step(nph)
    ph_t, n_t = tg.phase_times()
    tg.phase_timing(False)
    io.phase_timing(True)
    io.phase_reset()
    io.step(nph)
    ph_i, n_i = io.phase_times()
    io.phase_timing(False)
    per_tg = {k: v / max(n_t, 1) for k, v in ph_t.items()}
    per_io = {IO_PHASES[q]: v / max(n_i, 1) for q, v in enumerate(ph_i.values())}
    cand = [("tg", k, v) for k, v in per_tg.items()] + [("io", k, v) for k, v in per_io.items()]
    sec, dom, dom_ms = max(cand, key=lambda x: x[2])
    peak, peak_kind = measured_peak()
    if sec == "tg":
        bytes_dom = phase_bytes(dom, wt["nx"], wt["ny"], wt["nz"])
        kern = PHASE_KERNEL[dom]
        traffic = load_traffic(wl["tg"], kern)
    else:
        bytes_dom = io_phase_bytes_coupled(dom, wi["nx"], wi["ny"], wi["nz"])
        kern = IO_KERNEL_COUPLED[dom]
        traffic = load_traffic("c1_io_coupled", kern)
    achieved = bytes_dom / (dom_ms / 1000.0) / 1e9
    step_bytes = 3 * (sum(phase_bytes(p, wt["nx"], wt["ny"], wt["nz"]) for p in per_tg) +
                      sum(io_phase_bytes_coupled(p, wi["nx"], wi["ny"], wi["nz"]) for p in IO_PHASES))

    # end to end through the C ABI with host buffers (both sections): uploads,
    # one coupled step and downloads, stream-ordered on the shared stream
    tg_names, io_names = ("u", "v", "w", "p"), IO_RESULT_FIELDS
    host_t = {n: torch.empty(tg.shape, dtype=torch.float64, pin_memory=True).numpy() for n in tg_names}
    host_i = {n: torch.empty(io.shape, dtype=torch.float64, pin_memory=True).numpy() for n in io_names}
    for n in tg_names:
        tg.get_field(n, out=host_t[n])
    for n in io_names:
        io.get_field(n, out=host_i[n])
    barrier()
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, 10))

    def e2e(steps):
        for _ in range(steps):
            for n in tg_names:
                tg.set_field_async(n, host_t[n])
            for n in IO_INPUT_FIELDS:
                io.set_field_async(n, host_i[n])
            io.step_coupled(tg, 1)
            for n in tg_names:
                tg.get_field_async(n, out=host_t[n])
            for n in io_names:
                io.get_field_async(n, out=host_i[n])
            _ = tg.divgck_tg() + io.divgck_io()

    ms_e2e = max_over_ranks(timed(e2e, e2e_steps))
    e2e_value = cells * ws * e2e_steps / (ms_e2e / 1000.0)
    h2d = (len(tg_names) * tg.n + len(IO_INPUT_FIELDS) * io.n) * 8
    nbytes = (len(tg_names) * tg.n + len(io_names) * io.n) * 8
    bcs = io.bc_scalars()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            from oracle.pyoracle import get_threads
            nzc = 32  # a z-slab of both sections with their mesh spacing
            co = CoupledOracle(wt, wi, wl["bcx"], nzc)
            t0 = time.perf_counter()
            co.step(args.cpu_steps)
            t1 = time.perf_counter() - t0
            v = (wt["nx"] + wi["nx"]) * wt["ny"] * nzc * args.cpu_steps / t1
            cores = get_threads()
            cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
                   "sample": f"{args.cpu_steps} full coupled RK3 steps of {nzc}-plane z-slabs of both sections "
                             f"(same cell size) after init, {t1:.1f} s, FP64 oracle port, OpenMP {cores} threads"}
        except Exception as ex:
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == cs.FP64 else "TG f64 state / f32 temporaries, IO f64",
            "data": "synthetic (seeded splitmix64 velocity, NS=0 projection; IO h = 0, constant properties)",
            "config": workload_config(args, wl),
            "arm": {"parallelism": f"replicas x{ws}" if ws > 1 else "single GPU, both sections on one stream",
                    "l2": "working set (>4 GB) larger than the 126 MB L2"},
            "sections_ms_per_step": {"tg": ms_tg, "io": ms_io, "both": ms / args.steps},
            "max_div_u_tg": tg.divgck_tg(), "max_div_g_plus_drho_io": io.divgck_io(),
            "io_boundary": {"u_outlet": bcs["u_outlet"], "mass_scaling": bcs["scaling"],
                            "inflow": bcs["inflow"], "outflow": bcs["outflow"]},
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": nbytes + 16, "steps": e2e_steps,
                    "uploaded": {"tg": list(tg_names), "io": list(IO_INPUT_FIELDS)},
                    "downloaded": {"tg": list(tg_names), "io": list(io_names)}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kern, "phase": f"{sec}:{dom}",
                         "algorithmic_bytes_per_launch": bytes_dom, "avg_launch_ms": dom_ms,
                         "peak_source": peak_kind},
            "phases_ms_per_launch": {"tg": per_tg, "io": per_io},
            "step_roofline": {"algorithmic_bytes_per_step": step_bytes,
                              "achieved_gbs": step_bytes / (ms / args.steps / 1000.0) / 1e9,
                              "frac": step_bytes / (ms / args.steps / 1000.0) / 1e9 / peak},
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    io.close()
    tg.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def cpu_baseline_oracle(wl, steps):
    """FP64 oracle port on the host cores: init + NS=0, then `steps` timed steps."""
    from oracle.pyoracle import OracleTG, get_threads
    o = OracleTG(wl["nx"], wl["ny"], wl["nz"], lx=wl["lx"], lz=wl["lz"], ren=wl["ren"], dt=wl["dt"])
    o.init_random(wl["seed"], 0.1)
    o.substep(0)
    t0 = time.perf_counter()
    o.step(steps)
    t = time.perf_counter() - t0
    cells = wl["nx"] * wl["ny"] * wl["nz"]
    return cells * steps / t, t, get_threads()


def section_specs(wl):
    """(kind, spec) of every section a workload advances per step."""
    if wl.get("compare"):
        return [("io", WORKLOADS[wl["base"]])]
    if wl.get("pair"):
        # both sections as one coupled object (equal ny, nz): nx counts both
        wt, wi = WORKLOADS[wl["tg"]], WORKLOADS[wl["io"]]
        return [("pair", dict(nx=wt["nx"] + wi["nx"], ny=wt["ny"], nz=wt["nz"], tg=wt, io=wi, bcx=wl["bcx"]))]
    if wl.get("batch"):
        from chapsim1ww_b200 import batch64_configs
        return [("tg", dict(c, seed=wl["seed"] + i)) for i, c in enumerate(batch64_configs(seed=wl["seed"]))]
    return [("io" if wl.get("io") else "tg", wl)]


def make_oracle(kind, spec, nz):
    """FP64 oracle of one section on a z-slab of nz planes (the same mesh
    spacing as the full section: Lz scaled by nz / Nz), initialised as the
    GPU arm is (seeded field, NS=0 projection)."""
    from oracle.pyoracle import OracleIO, OracleTG
    if kind == "pair":
        return CoupledOracle(spec["tg"], spec["io"], spec["bcx"], nz)
    lz = spec["lz"] * nz / spec["nz"]
    if kind == "tg":
        o = OracleTG(spec["nx"], spec["ny"], nz, lx=spec["lx"], lz=lz, ren=spec["ren"], dt=spec["dt"])
        o.init_random(spec["seed"], 0.1)
        o.substep(0)
    else:
        o = OracleIO(spec["nx"], spec["ny"], nz, lx=spec["lx"], lz=lz, ren=spec["ren"], dt=spec["dt"],
                     thermal=spec["thermal"], prt=spec["prt"], qw=(spec["qw"], spec["qw"]),
                     table=io_table(spec["table"]), visc_scheme=spec.get("visc_scheme", 0))
        o.init_random(spec["seed"], 0.1)
    return o


def reference_sample(wl, steps, warmup, budget_s):
    """Pick the bounded sample of the workload the reference arm times: every
    section (or channel) as a z-slab of the same mesh spacing, sized from one
    calibration step of 8-plane slabs so that warmup + steps full RK3 steps
    take about budget_s seconds.  Returns [(kind, spec, nz_sample)]."""
    secs = section_specs(wl)
    if wl.get("batch"):
        secs = secs[:8]  # the first 8 channels, each a slab
    cal_nz = 8
    cells_cal = sum(sp["nx"] * sp["ny"] * min(cal_nz, sp["nz"]) for _, sp in secs)
    objs = [make_oracle(k, sp, min(cal_nz, sp["nz"])) for k, sp in secs]
    t0 = time.perf_counter()
    for o in objs:
        o.step(1)
    rate = cells_cal / max(time.perf_counter() - t0, 1e-6)  # cell-steps/s of the sample mix
    del objs
    cells_target = rate * budget_s / max(steps + warmup, 1)
    frac = cells_target / sum(sp["nx"] * sp["ny"] * sp["nz"] for _, sp in secs)
    out = []
    for k, sp in secs:
        nz = int(sp["nz"] * min(frac, 1.0)) // 8 * 8
        out.append((k, sp, max(8, min(nz, sp["nz"]))))
    return out


def run_reference(args, wl, ws, rank):
    """The reference algorithm's CPU path (the FP64 oracle port, all host
    threads) on rank 0: W warm-up and K timed full RK3 steps of a bounded
    sample of the workload (z-slabs with the workload's mesh spacing)."""
    if rank != 0:
        return 0
    from oracle.pyoracle import get_threads
    sample = reference_sample(wl, args.steps, args.warmup, args.ref_budget)
    objs = [make_oracle(k, sp, nz) for k, sp, nz in sample]
    for _ in range(args.warmup):
        for o in objs:
            o.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for o in objs:
            o.step(1)
    t = time.perf_counter() - t0
    cells = sum(sp["nx"] * sp["ny"] * nz for _, sp, nz in sample)
    v = cells * args.steps / t
    cores = get_threads()
    desc = ", ".join(f"{k} {sp['nx']}x{sp['ny']}x{nz} of {sp['nz']} planes" for k, sp, nz in sample)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
        "scaling": workload_scaling(wl), "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded splitmix64 field, NS=0 projection)",
        "config": workload_config(args, wl),
        "arm": {"impl": "FP64 oracle port (restatement of the Fortran path), OpenMP", "threads": cores},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
                         "sample": f"{args.warmup} warm-up + {args.steps} timed full RK3 steps of z-slabs with the "
                                   f"workload's mesh spacing ({desc}; {cells} cells per step, sized to about "
                                   f"{args.ref_budget:.0f} s of host work), FP64 oracle, OpenMP {cores} threads"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_scaling(wl):
    # the 64-channel batch is split across ranks (total work fixed); every
    # other workload runs one independent replica per rank
    return "strong" if wl.get("batch") else "weak"


def workload_config(args, wl):
    """The config block both arms print for a workload."""
    if wl.get("compare"):
        b = WORKLOADS[wl["base"]]
        return {"workload": args.workload, **{k: b[k] for k in ("nx", "ny", "nz", "ren", "dt", "prt")},
                "cells": b["nx"] * b["ny"] * b["nz"], "wall_heat_flux": b["qw"], "table": b["table"],
                "lx": b["lx"], "lz": b["lz"], "seed": b["seed"],
                "forms": "mixed precision + learned properties (value) against plain FP64 + table splines",
                "property_model": "degree-5 polynomial + MLP 1-64-64-5 tanh residual, 65,536 samples, seed 2, "
                                  "gate 1e-4 over 256 h-bins"}
    if wl.get("batch"):
        return {"workload": args.workload, "channels": 64, "seed": wl["seed"], "precision": args.precision,
                "steps_unit": "one RK3 step of every channel"}
    if wl.get("pair"):
        wt, wi = WORKLOADS[wl["tg"]], WORKLOADS[wl["io"]]
        return {"workload": args.workload,
                "tg": {k: wt[k] for k in ("nx", "ny", "nz", "ren", "dt")},
                "io": {**{k: wi[k] for k in ("nx", "ny", "nz", "ren", "dt", "prt")},
                       "table": wi["table"], "wall_heat_flux": wi["qw"],
                       "x": "inflow from the TG section, convective outflow", "bcx_io": list(wl["bcx"])},
                "cells": wt["nx"] * wt["ny"] * wt["nz"] + wi["nx"] * wi["ny"] * wi["nz"],
                "precision": args.precision}
    cfg = {"workload": args.workload, **{k: wl[k] for k in ("nx", "ny", "nz", "ren", "dt")},
           "cells": wl["nx"] * wl["ny"] * wl["nz"], "precision": args.precision}
    if wl.get("io"):
        cfg.update(prt=wl["prt"], wall_heat_flux=wl["qw"], table=wl["table"],
                   viscous_scheme="semi-implicit (MOMFA_io)" if wl.get("visc_scheme") else "explicit")
    return cfg


def shard_channels(cells, ws, rank):
    """Channel indices of one rank: channels dealt largest first to the rank
    with the fewest cells so far (ties to the lower rank), so every rank gets
    a near-equal share of the work; deterministic and identical on all ranks."""
    load = [0] * ws
    own = [[] for _ in range(ws)]
    for i in sorted(range(len(cells)), key=lambda q: (-cells[q], q)):
        r = min(range(ws), key=lambda q: (load[q], q))
        load[r] += cells[i]
        own[r].append(i)
    return sorted(own[rank])


def run_batch(args, wl, ws, rank, local):
    """The 64 uneven channels split across the ranks (shard_channels; no
    data-path collective), each rank advancing its share by one graph launch
    per step.  value = all 64 channels' cells x steps / max-over-ranks time."""
    import torch

    import chapsim1ww_b200 as cs
    from chapsim1ww_b200 import ChannelBatch, batch64_configs

    torch.cuda.set_device(local)
    pg = dist_init(ws)
    prec = cs.FP64 if args.precision == "fp64" else cs.MIXED
    all_cfgs = batch64_configs(seed=wl["seed"])
    mine = shard_channels([c["nx"] * c["ny"] * c["nz"] for c in all_cfgs], ws, rank)
    cfgs = [all_cfgs[i] for i in mine]
    b = ChannelBatch(cfgs, precision=prec, device=local)
    t0 = time.perf_counter()
    b.autotune(reps=3)
    t_tune = time.perf_counter() - t0
    b.init_random(seed=wl["seed"], amp=0.1, project=True)
    b.step(args.warmup)
    b.sync()
    stream = torch.cuda.ExternalStream(b.stream(), device=local)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop()
    ms = max_over_ranks(pg, local, e0.elapsed_time(e1))
    divmax = max_over_ranks(pg, local, max(ch.divgck_tg() for ch in b.channels))
    total_cells = sum(c["nx"] * c["ny"] * c["nz"] for c in all_cfgs)
    value = total_cells * args.steps / (ms / 1000.0)
    launches = int(max_over_ranks(pg, local, float(b.kernels_per_step() * args.steps)))
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": workload_scaling(wl),
        "vs_baseline": None, "dtype": "f64" if prec == cs.FP64 else "f64 state / f32 temporaries",
        "data": "synthetic (64 channels, sizes and Re drawn from seed 3)",
        "config": workload_config(args, wl),
        "arm": {"graph": "one CUDA graph launch per step, channels as parallel branches",
                "channels_per_rank": len(cfgs), "cells_rank0": b.cells, "autotune_s": t_tune},
        "max_div_u": divmax, "gpu_launches": launches, "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    dist_done(pg)
    return 0


def run_ours(args, wl, ws, rank, local):
    import numpy as np
    import torch

    import chapsim1ww_b200 as cs
    from chapsim1ww_b200 import TGChannel

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    prec = cs.MIXED if args.precision == "mixed" else cs.FP64
    s = TGChannel(wl["nx"], wl["ny"], wl["nz"], lx=wl["lx"], lz=wl["lz"], ren=wl["ren"], dt=wl["dt"],
                  precision=prec, device=local)
    s.random_fl_fld_tg(wl["seed"] + rank, 0.1, project=True)
    cells = wl["nx"] * wl["ny"] * wl["nz"]
    stream = torch.cuda.ExternalStream(s.stream(), device=local)

    def barrier():
        if pg is not None:
            pg.barrier()

    def max_over_ranks(x):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    # ---- resident timing (graph replay)
    s.step(args.warmup)
    s.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = s.launch_count()
    e0.record(stream)
    s.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    launches = s.launch_count() - n0
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = cells * ws * args.steps / (ms / 1000.0)
    divmax = s.divgck_tg()

    # ---- per-phase kernel times (eager launches, CUDA events between phases)
    s.phase_timing(True)
    s.phase_reset()
    s.step(args.steps)
    ph, nsub = s.phase_times()
    s.phase_timing(False)
    per_launch = {k: v / max(nsub, 1) for k, v in ph.items()}
    dom = max(per_launch, key=per_launch.get)
    peak, peak_kind = measured_peak()
    bytes_dom = phase_bytes(dom, wl["nx"], wl["ny"], wl["nz"])
    achieved = bytes_dom / (per_launch[dom] / 1000.0) / 1e9
    total_bytes = sum(phase_bytes(p, wl["nx"], wl["ny"], wl["nz"]) for p in ph)
    step_ms_phases = 3 * sum(per_launch.values())
    traffic = load_traffic(args.workload, PHASE_KERNEL[dom])

    # ---- end to end through the public API with host buffers
    names = ("u", "v", "w", "p")
    host = {}
    for n in names:
        t = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
        host[n] = t.numpy()
        s.get_field(n, out=host[n])
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 20))
    e2.record(stream)
    for _ in range(e2e_steps):
        for n in names:
            s.set_field_async(n, host[n])
        s.step(1)
        for n in names:
            s.get_field_async(n, out=host[n])
        _ = s.divgck_tg()
    e3.record(stream)
    e3.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3))
    e2e_value = cells * ws * e2e_steps / (ms_e2e / 1000.0)
    nbytes = 4 * s.n * 8

    learned = None
    if rank == 0 and not args.no_props:
        learned = bench_learned(cells, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            v, t, cores = cpu_baseline_oracle(wl, args.cpu_steps)
            slab = (f" (a {wl['cpu_nz']}-plane z-slab, same cell size)" if wl.get("cpu_nz") else "")
            cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
                   "sample": f"{args.cpu_steps} full RK3 steps of the {args.workload} channel{slab} after init, "
                             f"FP64 oracle port, OpenMP {cores} threads, {t:.1f} s"}
        except Exception as ex:  # the checker is optional for the GPU arm
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == cs.FP64 else "f64 state / f32 temporaries",
            "data": "synthetic (seeded splitmix64 initial field, NS=0 projection)",
            "config": workload_config(args, wl),
            "arm": {"parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                    "l2": "working set (>1 GB) larger than the 126 MB L2"},
            "max_div_u": divmax,
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes + 8, "steps": e2e_steps},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": PHASE_KERNEL[dom],
                         "phase": dom, "algorithmic_bytes_per_launch": bytes_dom,
                         "avg_launch_ms": per_launch[dom], "peak_source": peak_kind},
            "phases_ms_per_launch": per_launch,
            "step_roofline": {"algorithmic_bytes_per_step": 3 * total_bytes,
                              "achieved_gbs": 3 * total_bytes / (ms / args.steps / 1000.0) / 1e9,
                              "frac": 3 * total_bytes / (ms / args.steps / 1000.0) / 1e9 / peak,
                              "phase_sum_ms": step_ms_phases},
            "clocks": clk,
            "learned": learned,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def profile_case(spec, precision, spectra="fp64", refine=1):
    import chapsim1ww_b200 as cs
    from chapsim1ww_b200 import TGChannel
    if spec.lower().startswith("iolearn"):
        # the IO form with the learned property model, Poisson spectra as in
        # the comparison workload (model trained briefly: the kernels' work
        # does not depend on its accuracy)
        from chapsim1ww_b200 import IOChannel, PropertyEngine, synthetic_table
        nx, ny, nz = (int(x) for x in spec.lower()[7:].split("x"))
        eng = PropertyEngine(*synthetic_table(4096))
        eng.train(65536, 2, 300, 3e-3)
        eng.gate(1e9, 256)
        c = IOChannel(nx, ny, nz, table=io_table("synthetic"), precision=cs.MIXED if spectra == "fp32" else cs.FP64)
        c.set_refinement(refine)
        c.set_props_mode(1, eng)
        c.random_fl_theml_fld_io(2, 0.1)
        for _ in range(2):
            for ns in (1, 2, 3):
                c.solverrk3_eng_io(ns)
                c.solverrk3_mom_io(ns)
        c.sync()
        print("profile case ok", spec, "max|div G + drho| =", c.divgck_io())
        return 0
    if spec.lower().startswith("cpl"):
        # the coupled pair: TG nx/2 x ny x nz feeding the IO section nx x ny x
        # nz (BCX_io = 2, 1, constant properties), eager substeps in SOLVE's order
        from chapsim1ww_b200 import IOChannel
        nx, ny, nz = (int(x) for x in spec.lower()[3:].split("x"))
        t = TGChannel(nx // 2, ny, nz)
        c = IOChannel(nx, ny, nz, table=io_table("constant"), bcx=(2, 1))
        c.set_inlet(t)
        t.random_fl_fld_tg(1, 0.1, project=True)
        c.random_fl_theml_fld_io(1, 0.1)
        for _ in range(2):
            for ns in (1, 2, 3):
                t.solverrk3_mom_tg(ns)
                c.solverrk3_eng_io(ns)
                c.solverrk3_mom_io(ns)
        c.sync()
        print("profile case ok", spec, "max|div G + drho| =", c.divgck_io())
        c.close()
        t.close()
        return 0
    if spec.lower().startswith("io"):
        from chapsim1ww_b200 import IOChannel
        si = spec.lower().startswith("iosi")  # the semi-implicit viscous scheme
        nx, ny, nz = (int(x) for x in spec.lower()[4 if si else 2:].split("x"))
        c = IOChannel(nx, ny, nz, table=io_table("synthetic"), visc_scheme=1 if si else 0)
        c.random_fl_theml_fld_io(2, 0.1)
        for _ in range(2):
            for ns in (1, 2, 3):
                c.solverrk3_eng_io(ns)
                c.solverrk3_mom_io(ns)
        c.sync()
        print("profile case ok", spec, "max|div G + drho| =", c.divgck_io())
        return 0
    nx, ny, nz = (int(x) for x in spec.lower().split("x"))
    s = TGChannel(nx, ny, nz, precision=cs.MIXED if precision == "mixed" else cs.FP64)
    s.random_fl_fld_tg(1, 0.1, project=True)
    for _ in range(2):
        for ns in (1, 2, 3):
            s.solverrk3_mom_tg(ns)
    s.sync()
    print("profile case ok", spec, precision, "max|div u| =", s.divgck_tg())
    return 0


def launch_ranks(n):
    """Run this same command as n ranks, one per GPU, under
    torch.distributed.run on 127.0.0.1 (used when --gpus N > 1 is given
    without an outside launcher); returns the launcher's exit code."""
    import socket
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c4_mixed_learned")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--ref-budget", type=float, default=100.0,
                    help="seconds of host work the reference arm's W + K steps are sized to")
    ap.add_argument("--refine", type=int, choices=[0, 1], default=1,
                    help="FP64-residual refinement sweeps of the mixed IO form's Poisson solve")
    ap.add_argument("--spectra", choices=["fp32", "fp64"], default="fp64",
                    help="precision of the Poisson spectra of the learned-property IO form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-props", action="store_true", help="skip the learned-property measurement")
    ap.add_argument("--profile-case", default=None, metavar="NXxNYxNZ",
                    help="run init + NS=0 + 2 eager RK3 steps of a channel of this size and exit "
                         "(the small case for ncu captures; no timing); prefix io for an IO channel, "
                         "iosi for an IO channel with the semi-implicit viscous scheme")
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args.profile_case, args.precision, args.spectra, args.refine)
    args.warmup = max(args.warmup, 3)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus)
    wl = WORKLOADS[args.workload]
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, wl, ws, rank)
    if wl.get("batch"):
        return run_batch(args, wl, ws, rank, local)
    if wl.get("compare"):
        return run_compare(args, wl, ws, rank, local)
    if wl.get("pair"):
        return run_pair(args, wl, ws, rank, local)
    if wl.get("io"):
        return run_io(args, wl, ws, rank, local)
    return run_ours(args, wl, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
