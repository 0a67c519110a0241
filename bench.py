#!/usr/bin/env python
"""Benchmark: grid-point updates per second of the FP64 Teukolsky step.

Workload (default, the size the HBM-roofline target is quoted at): FP64
plunge-driven ringdown, s=-2, m=2, a=0.9, M=1, grid coordinate in
[-200, 600] with N_r=16384, N_theta=256, dt = 0.25 min(dx, r_min dtheta),
source from a prograde equatorial plunge worldline sampled at dt/2 (a
seeded synthetic stand-in for GenOT output: no GenOT inputs exist here).
`--workload plunge` runs the same at 8192 x 128, `--workload grid16k` the
16384 x 256 grid source-free.

A step is one full time step (source patch, three SSP-RK3 stages,
extraction) over the whole grid.  When the three states (96 B per point)
exceed the 126 MB L2, the K timed steps run back to back between one pair
of CUDA events on the solver's stream; otherwise L2 is flushed by writing
a 256 MB buffer before each step and each step is timed alone.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N>1 (torchrun, one process per GPU) every rank advances its own
independent solve (replicas: solves share nothing), timing is the max over
ranks and value is the sum of all ranks' updates over that time.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys
import time

import numpy as np

from bh_ringdown_b200 import replicas

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt updates/s (%HBM roofline); solves/s, p99 latency vs FP64 plain @1e-6"
UNIT = "grid-pt updates/s"
WORKLOADS = {
    # plunge-driven ringdown at the size the HBM-roofline target is quoted at (the default)
    "plunge16k": dict(N=16384, M=256, Xmin=-200.0, Xmax=600.0, a=0.9, m=2.0, T=1000.0, courant=0.25, source=True),
    # the same physics at the plunge configuration's own grid, 8192 x 128
    "plunge": dict(N=8192, M=128, Xmin=-200.0, Xmax=600.0, a=0.9, m=2.0, T=1000.0, courant=0.25, source=True),
    # 16384 x 256, source-free (Gaussian pulse initial data)
    "grid16k": dict(N=16384, M=256, Xmin=-200.0, Xmax=600.0, a=0.9, m=2.0, T=1000.0, courant=0.25, source=False),
}
DEFAULT_WORKLOAD = "plunge16k"
WORKLOAD = WORKLOADS[DEFAULT_WORKLOAD]
# The reference's own kernels on host cores (oracle/_ref, built by
# oracle/build_ref.py with the grid fixed at compile time), per workload.
REFERENCE_LIBS = {"plunge16k": "libref_p16k.so", "plunge": "libref_cfg2.so"}
L2_BYTES = 126 * 1024 * 1024
BYTES_PER_PT = 256.0  # FP64 SSP-RK3 algorithmic bytes per point per step (coefficients recomputed)
# Mixed precision: stage 1 reads u^n and writes u1 (FP64) and delta1 (FP32),
# stage 2 reads delta1 and writes eps2 (FP32), stage 3 reads eps2 and u1 and
# writes u^{n+1}: 80 + 32 + 80 bytes per point.
BYTES_PER_PT_MIXED = 192.0
# Classical RK4 (--integrator rk4): stage 1 reads u^n, writes y1 (64 B);
# stage 2 reads y1 and u^n, writes y2 and z (128 B); stage 3 reads y2 and
# u^n, writes y3 (96 B); stage 4 reads y3 and z, writes u^{n+1} (96 B).
BYTES_PER_PT_RK4 = 384.0
INTEGRATOR = "ssprk3"
PRECISION = "fp64"


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(workload):
    """DRAM bytes per grid point of one step's three stage launches, from the
    committed ncu summary of this workload (line
    'dram_bytes_per_point_per_step: X'), or None."""
    name = {("plunge", "ssprk3"): "stage_kernel_plunge8192x128.txt",
            ("plunge16k", "ssprk3"): "stage_dram_plunge16384x256.txt",
            ("grid16k", "ssprk3"): "stage_dram_grid16384x256.txt",
            ("grid16k", "rk4"): "stage_dram_rk4_grid16384x256.txt"}.get((workload, INTEGRATOR))
    if name is None:
        return None
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith("dram_bytes_per_point_per_step:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every few ms while
    the timed region runs (read-only queries)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, cuda_device):
        self.dev = cuda_device
        self.samples = []
        self.stop = None
        self.thread = None
        self.max_mhz = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.dev)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def sample(self):
        """One sample now (also called at fixed points of the timed region,
        so a starved sampling thread still leaves a record)."""
        if getattr(self, "h", None) is None:
            return
        try:
            import pynvml
            mhz = pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            rs = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
            self.samples.append((mhz, rs))
        except Exception:
            pass

    def __enter__(self):
        import threading
        self.h = None
        try:
            import pynvml
            self.h = self._handle()
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.stop = threading.Event()

            def run():
                while not self.stop.is_set():
                    self.sample()
                    time.sleep(0.001)
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return None
        mhz = [m for m, _ in self.samples]
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": float(self.max_mhz or max(mhz)),
                "reasons": reasons, "samples": len(mhz), "source": "NVML during the timed region"}


def source_available():
    import bh_ringdown_b200 as bhr
    try:
        bhr.source_coefficients(bhr.Particle(rp=6.0, tp=np.pi / 2, E=0.9, lz=3.0), 0.5, 1.0, 2.0)
        return True
    except bhr.BhrError:
        return False


def make_params(device=0, dt=None):
    import bh_ringdown_b200 as bhr
    w = WORKLOAD
    return bhr.Params(N=w["N"], M=w["M"], Xmin=w["Xmin"], Xmax=w["Xmax"], a=w["a"], m=w["m"], T=w["T"],
                      dt=0.0 if dt is None else dt, courant=w["courant"], Fr=50, out_start=0.0, device=device,
                      init_kind=bhr.BHR_INIT_ZERO, precision=bhr.BHR_MIXED if PRECISION == "mixed" else bhr.BHR_FP64,
                      integrator=bhr.BHR_RK4 if INTEGRATOR == "rk4" else bhr.BHR_SSPRK3)


# The plunge workloads' source: GenOT's transition-to-plunge worldline for
# mass ratio 1e-3 from the ISCO, rows every dt/2 (the reference's step reads
# two rows), 60 M of it (more than any timed or e2e run reaches).
PLUNGE_ETA, PLUNGE_DURATION = 1e-3, 60.0


def plunge_rows(a, dt):
    from bh_ringdown_b200.genot import transition_plunge
    return transition_plunge(a, PLUNGE_ETA, dt / 2.0, PLUNGE_DURATION)


def workload_inputs(with_source, device=0):
    """(params, trajectory rows or None).  Without a source the run starts
    from a Gaussian pulse instead (psi = exp(-(x-20)^2/8) swsh(2,2))."""
    import bh_ringdown_b200 as bhr
    prm = make_params(device)
    x, r, th = bhr.grid(prm)
    dx = (prm.Xmax - prm.Xmin) / prm.N
    dt = prm.courant * min(dx, r[0] * np.pi / prm.M)
    prm.dt = dt
    if with_source:
        return prm, plunge_rows(prm.a, dt)
    prm.init_kind = bhr.BHR_INIT_GAUSSIAN
    prm.init_center, prm.init_width, prm.init_ell = 20.0, 2.0, 2.0
    return prm, None


def workload_config(name, N, M, dt, with_source, world):
    """The `config` dict of a single-solve workload; both arms (ours and
    --impl reference) print exactly this dict for the same workload."""
    w = WORKLOADS[name]
    prec = "FP64" if PRECISION == "fp64" else "mixed FP64/FP32"
    return {"workload": f"{name}: {prec} s=-2 m={w['m']:g} a={w['a']:g}, {N}x{M} on "
                        f"[{w['Xmin']:g},{w['Xmax']:g}], "
                        + ("plunge source" if with_source else "source-free (Gaussian pulse initial data)"),
            "N_r": N, "N_theta": M, "dt": dt,
            "integrator": "classical RK4" if INTEGRATOR == "rk4" else "SSP-RK3",
            "precision": PRECISION,
            "source": (f"GenOT transition-to-plunge worldline (prograde equatorial, eta={PLUNGE_ETA:g}, from the "
                       "ISCO; stand-in inspiral table), rows every dt/2") if with_source else "none",
            "parallelism": f"replicas x{world}"}


def run_ours(args, rank, local_rank, world):
    import torch
    import bh_ringdown_b200 as bhr

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    with_source = WORKLOAD["source"]
    if with_source and not source_available():
        raise SystemExit("the particle source coefficients are unavailable in libbhr.so")
    prm, rows = workload_inputs(with_source, device=local_rank)
    N, M = prm.N, prm.M
    solver = bhr.Solver(prm)
    if rows is not None:
        solver.set_trajectory(rows)
    tiling, ahead = solver.info()["tiling"], solver.info()["prefetch_ahead"]
    # Three states of 32 B per point larger than L2: the timed steps run back
    # to back (each reads what the previous one wrote from HBM); otherwise L2
    # is flushed before each step and each step is timed alone.
    resident = 3 * 32 * N * M <= L2_BYTES
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") if resident else None

    def flush_l2():
        flush.zero_()
        torch.cuda.synchronize()

    # clocks are sampled from the first warm-up step to the end of the
    # per-kernel breakdown pass
    with ClockSampler(local_rank) as clk:
        for _ in range(args.warmup):
            if resident:
                flush_l2()
            solver.time_steps(1)
            clk.sample()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        total_ms = 0.0
        if resident:
            for _ in range(args.steps):
                flush_l2()
                total_ms += solver.time_steps(1)
                clk.sample()
        else:
            total_ms = solver.time_steps(args.steps)
            clk.sample()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            total_ms = replicas.max_over_ranks(total_ms, dist, device="cuda")
        # per-kernel breakdown (eager launches, events around each kernel): not
        # the timed figure, which is the graph-launched step above
        nprof = min(args.steps, 20)
        per_kernel = np.zeros(5)
        for _ in range(nprof):
            if resident:
                flush_l2()
            avg, _tot = solver.profile(1)
            per_kernel += avg
            clk.sample()
        torch.cuda.synchronize()
    clocks = clk.summary()
    solver.close()

    value = world * N * M * args.steps / (total_ms / 1e3)
    ms_per_step = total_ms / args.steps
    peak, peak_kind = measured_peak()
    bytes_pt = (BYTES_PER_PT_MIXED if PRECISION == "mixed" else
                BYTES_PER_PT_RK4 if INTEGRATOR == "rk4" else BYTES_PER_PT)
    # The stage kernels carry the step (the launch lists in profiles/ give
    # their share); achieved = the step's algorithmic bytes over the device
    # time of the graph-launched step, so it can only understate the kernels.
    achieved = bytes_pt * N * M / (ms_per_step / 1e3) / 1e9
    traffic_pp = profile_traffic(args.workload) if PRECISION == "fp64" else None

    # End to end through the public API: host params + host trajectory in,
    # solver set-up (grid, tables, initial data uploaded), n steps, waveform
    # rows copied back, solver destroyed; wall clock.
    n_e2e = args.e2e_steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2 = bhr.Solver(prm)
    if rows is not None:
        s2.set_trajectory(rows)
    s2.step(n_e2e)
    tw, hw, ew = s2.waveform()
    info = s2.info()
    s2.close()
    t_e2e = time.perf_counter() - t0
    if dist is not None:  # every rank ran its own e2e solve: the job takes the slowest
        t_e2e = replicas.max_over_ranks(t_e2e, dist, device="cuda")
    # bytes the API copies host -> device: column (14) and row (4) tables, r_c and
    # theta, projection and dE/dt weights, the separable initial-data factors
    # (Gaussian data), and one 128-byte source record per step of the run
    # (sourced; built and uploaded chunk by chunk while the device steps)
    h2d = ((14 * N + 4 * M) + (N + M) + (7 * M + M)) * 8
    if prm.init_kind == bhr.BHR_INIT_GAUSSIAN:
        h2d += (N + M) * 8
    if rows is not None:
        h2d += info["nt"] * 128
    d2h = len(tw) * 16 * 8
    e2e = {"value": N * M * n_e2e / t_e2e * world, "unit": UNIT, "h2d_bytes_per_step": int(h2d / n_e2e),
           "d2h_bytes_per_step": int(d2h / n_e2e), "steps": n_e2e,
           "note": "wall clock of create + trajectory upload + steps + waveform readback + destroy"}

    cpu = ref_gpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(prm, rows, args.cpu_seconds)
        ref_gpu = reference_gpu_baseline(args.workload, prm)

    if rank == 0:
        kernel_label = ("FP64 stage 1 + FP32 mixed_stage_kernel<2,3> (192 B/pt algorithmic)"
                        if PRECISION == "mixed" else
                        "stage kernels <1,4,4,5> (one classical RK4 step, 384 B/pt algorithmic)"
                        if INTEGRATOR == "rk4" else
                        "stage kernels <1,2,3> (one SSP-RK3 step, 256 B/pt algorithmic)")
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if PRECISION == "fp64" else "f64+f32", "data": "synthetic",
            "config": workload_config(args.workload, N, M, prm.dt, with_source, world),
            "timing": {"l2": ("flushed (256 MB write) before each timed step, each step timed alone" if resident else
                              f"working set {3 * 32 * N * M / 2**20:.0f} MiB > L2 (126 MiB): "
                              f"{args.steps} steps back to back, no flush"),
                       "events": "CUDA events on the solver stream around graph-launched steps",
                       "stage_tiling": tiling, "prefetch_ahead_blocks": ahead},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": None if traffic_pp is None else traffic_pp * N * M,
                         "kernel": kernel_label,
                         "basis": f"{bytes_pt:g} B/pt x {N}x{M} points per step / ms_per_step"},
            "kernel_ms": {"source": per_kernel[0] / nprof, "stage1": per_kernel[1] / nprof,
                          "stage2": per_kernel[2] / nprof,
                          "stage3+4" if INTEGRATOR == "rk4" else "stage3": per_kernel[3] / nprof,
                          "extract": per_kernel[4] / nprof,
                          "note": "breakdown only: eager launches each timed alone (no programmatic overlap "
                                  "between kernels); source and extract run on a side stream beside stages 1 "
                                  "and 2, timed from the side stream's fork to the kernel's end"},
            # per step: the stages, the step-clock kernel, the extraction (of the
            # previous step, beside stage 2) and the source when there is one
            "gpu_launches": args.steps * ((6 if with_source else 5) + (1 if INTEGRATOR == "rk4" else 0)),
            "e2e": e2e,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
        }
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


# The reference's own GPU code (HighOrder/body.cu + kern.cu compiled unchanged
# by nvcc for sm_100a, oracle/build_ref.py), per workload: its grid and final
# time are fixed at compile time.
REFERENCE_GPU_EXES = {"plunge16k": "refgpu_gp16k"}


def reference_gpu_baseline(workload, prm):
    """Wall clock of the reference's body() run on this GPU for the
    workload's grid, spin, m and dt with the same synthetic plunge (its
    whole loop: set-up, the sourced SSP-RK3 steps with a host sync after
    every kernel, the per-step D2H copy and host projections), as grid-point
    updates per second; None when the build is absent."""
    import subprocess
    import tempfile
    exe = REFERENCE_GPU_EXES.get(workload)
    if exe is None or PRECISION != "fp64" or INTEGRATOR != "ssprk3":
        return None
    path = os.path.join(ROOT, "oracle", "_ref", exe)
    if not os.path.exists(path):
        return {"unavailable": f"oracle/_ref/{exe} was not built (the reference tree was absent at build time)"}
    rows = plunge_rows(prm.a, prm.dt)
    with tempfile.TemporaryDirectory() as work:
        os.makedirs(os.path.join(work, "Trajectories"))
        os.makedirs(os.path.join(work, "run"))
        np.savetxt(os.path.join(work, "Trajectories", "a0.0_thi000_thf090.0_n.traj"), rows, fmt="%.17g")
        out = subprocess.run([path, work, "%.17g" % prm.a, "%.17g" % prm.m, "%.17g" % prm.dt], capture_output=True,
                             text=True, timeout=600)
    if out.returncode != 0:
        return {"unavailable": f"{exe} exited {out.returncode}: {out.stderr.strip()[-300:]}"}
    info = json.loads(out.stdout.strip().splitlines()[-1])
    if info["nt"] <= 0:
        return {"unavailable": f"{exe} ran no steps: {info}"}
    return {"value": info["N"] * info["M"] * info["nt"] / info["seconds"], "unit": UNIT, "steps": info["nt"],
            "seconds": info["seconds"], "kind": "reference",
            "note": "the reference's body() (HighOrder/body.cu + kern.cu, compiled unchanged for sm_100a) on this "
                    "GPU, wall clock of the whole call: set-up, sourced SSP-RK3 steps with a sync after each of "
                    "its 14 kernels, per-step D2H copy and host projections"}


def cpu_baseline(prm, rows, seconds):
    """The FP64 oracle on this host's cores, a bounded sample of the same
    workload (steps of the full grid until about `seconds` elapse)."""
    from oracle import pyoracle
    import bh_ringdown_b200 as bhr
    o = pyoracle.Oracle(prm.N, prm.M, prm.Xmin, prm.Xmax, prm.a, prm.m, prm.dt, T=prm.T, Fr=50, out_start=0.0,
                        integrator=prm.integrator)
    coef = None
    if rows is None:
        o.init_gaussian(prm.init_center, prm.init_width, prm.init_ell)
    else:
        lib = bhr.load_library()

        def _coef(pt, a, mass, m, cr, ci):
            p = bhr.Particle(*[getattr(pt.contents, n) for n, _ in pyoracle.OrcParticle._fields_])
            import ctypes
            lib.bhr_source_coefficients(ctypes.byref(p), a, mass, m, cr, ci)
        coef = pyoracle.COEF_FN(_coef)
    t0 = time.perf_counter()
    n = 0
    chunk = 5
    while time.perf_counter() - t0 < seconds:
        if rows is None:
            o.step(chunk)
        else:
            o.run(traj=rows, coef_fn=coef, nsteps=chunk, max_rows=10)
        n += chunk
    el = time.perf_counter() - t0
    return {"value": prm.N * prm.M * n / el, "unit": UNIT, "cores": pyoracle.num_threads(), "kind": "port",
            "sample": f"{n} steps of the full {prm.M}x{prm.N} grid in {el:.1f} s (FP64 oracle, OpenMP over theta rows)"}


def run_reference(args, rank, world):
    """The reference's own HighOrder kernels compiled for and run on this
    host's cores (oracle/_ref/libref_<tag>.so, its grid fixed at compile
    time), on the same workload, config and metric as our arm."""
    if rank != 0:
        return
    lib_name = REFERENCE_LIBS.get(args.workload)
    if lib_name is None or PRECISION != "fp64" or INTEGRATOR != "ssprk3":
        print(json.dumps({"impl": "reference", "unavailable": "the reference integrates FP64 SSP-RK3 with a source; "
                                                               f"oracle/_ref holds builds for {sorted(REFERENCE_LIBS)}"}))
        return
    import ctypes as C
    lib_path = os.path.join(ROOT, "oracle", "_ref", lib_name)
    if not os.path.exists(lib_path):
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/{lib_name} was not built "
                                                               "(the reference tree was absent at build time)"}))
        return
    from oracle import pyoracle
    D = C.c_double
    L = C.CDLL(lib_path)
    # All of the host's threads, whatever OMP_NUM_THREADS the launcher set
    # (torchrun sets 1): the library's OpenMP runtime, found by its soname.
    threads = os.cpu_count() or 1
    try:
        gomp = C.CDLL("libgomp.so.1")
        gomp.omp_set_num_threads(threads)
        threads = int(gomp.omp_get_max_threads())
    except (OSError, AttributeError):
        threads = int(os.environ.get("OMP_NUM_THREADS", threads))
    L.ref_source.argtypes = [D] * 16
    N, M = L.ref_N(), L.ref_M()
    w = WORKLOAD
    assert (N, M) == (w["N"], w["M"]), (lib_name, N, M)
    o = pyoracle.Oracle(N, M, w["Xmin"], w["Xmax"], w["a"], w["m"], 0.01)
    # the reference's grid(), except that the radii it leaves NaN near the horizon are floored at
    # nextafter(r+), as the library does
    x, r, th = o.grid()
    o.close()
    dx = (w["Xmax"] - w["Xmin"]) / N
    dt = w["courant"] * min(dx, r[0] * np.pi / M)
    L.ref_init(D(1.0), D(w["a"]), D(w["m"]), D(dt), th.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p))
    rows = plunge_rows(w["a"], dt)
    er, ei = np.zeros(M), np.zeros(M)

    # body.cu:97-124 consumption of the trajectory rows, restated.
    cur = [2]
    state = {"rp": rows[1, 1], "t11": 0.0, "t22": 0.0, "t33": 0.0, "row": rows[1]}

    def one_step(k, timer):
        for _ in range(2):
            if cur[0] < len(rows):
                state["row"] = rows[cur[0]]
                state["rp"] = state["row"][1]
                cur[0] += 1
        row = state["row"]
        state["rp"] += 1e-6
        L.ref_source(D(0.0), D(timer), D(state["rp"]), D(row[6]), D(row[2]), D(row[7]), D(row[8]), D(row[9]),
                     D(row[3]), D((row[3] - state["t11"]) / dt), D(0.0), D(row[4]), D((row[4] - state["t22"]) / dt),
                     D(0.0), D(row[5]), D((row[5] - state["t33"]) / dt))
        state["t11"], state["t22"], state["t33"] = row[3], row[4], row[5]
        L.ref_step(er.ctypes.data_as(C.c_void_p), ei.ctypes.data_as(C.c_void_p))

    timer = 0.0
    for k in range(args.warmup):
        one_step(k, timer)
        timer += dt
    t0 = time.perf_counter()
    for k in range(args.steps):
        one_step(args.warmup + k, timer)
        timer += dt
    el = time.perf_counter() - t0
    value = N * M * args.steps / el
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(args.workload, N, M, dt, True, world),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                            "sample": f"{args.steps} full step{'s' if args.steps != 1 else ''} (reference sourced + "
                                      f"12 step kernels, HighOrder/body.cu:108-165 order, source from the "
                                      f"reference's Maple block) on the {M}x{N} grid, host cores"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def _solve_steps(prm):
    """Step count of a solve (the solver's own dt rule) without creating it."""
    import bh_ringdown_b200 as bhr
    if prm.dt > 0:
        dt = prm.dt
    else:
        _, r, _ = bhr.grid(prm)
        dt = prm.courant * min((prm.Xmax - prm.Xmin) / prm.N, r[0] * np.pi / prm.M)
        if prm.out_every > 0:
            dt = prm.out_every / np.ceil(prm.out_every / dt)
    return int(prm.T / dt)


def _dist_init(world, local_rank):
    """Process group for the replica bookkeeping (N > 1), else None."""
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist


def run_batch(args):
    """Batched form: 64 seeded source-free solves of mixed size resident on
    one GPU, advanced together by the engine (one launch per RK stage over
    the (solve, tile) work-list, graph-captured), against the same solves
    run one at a time through bhr_solver (each with its autotuned tile).

    Throughput is device time (CUDA events) over `--steps` batch steps with
    all 64 resident; the working set (GBs) is far above L2.  The plain
    figure weights each solve's measured per-step time by its full step
    count, so the ratio is the ratio of solves/s at equal work."""
    import torch
    import bh_ringdown_b200 as bhr
    from bh_ringdown_b200.workloads import batch_requests
    rank, local_rank, world = env_rank()
    torch.cuda.set_device(local_rank)
    dist = _dist_init(world, local_rank)
    all_reqs = batch_requests(64, precision=bhr.BHR_MIXED if PRECISION == "mixed" else bhr.BHR_FP64)
    # replicas: this rank's share of the 64 solves (work-balanced, no collective on the data path)
    mine = replicas.run_shard(all_reqs, rank, world, lambda r: replicas.request_work(r.params))
    reqs = [all_reqs[i] for i in mine]
    for r in reqs:
        r.params.device = local_rank
    nts = [_solve_steps(r.params) for r in reqs]
    work = [nt * r.points() for nt, r in zip(nts, reqs)]
    with bhr.Engine(device=local_rank, hbm_budget_bytes=150 << 30) as e:
        for r in reqs:
            e.submit(r.params, r.traj)
        while e.stats()["queued"] > 0:  # requests are prepared off the stepping thread
            e.step(0)
        e.step(args.warmup)
        st0 = e.stats()
        assert st0["running"] == len(reqs), st0
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        with ClockSampler(local_rank) as clk:
            e.step(args.steps)
        wall = replicas.max_over_ranks(time.perf_counter() - t0, dist, device="cuda")
        st1 = e.stats()
    dev_ms = replicas.max_over_ranks(st1["device_ms"] - st0["device_ms"], dist, device="cuda")
    pts = sum(replicas.gather_objects(st1["point_updates"] - st0["point_updates"], dist))
    value = pts / (dev_ms / 1e3)
    # one at a time, each solve alone
    plain_ms = []
    for r in reqs:
        with bhr.Solver(dataclasses.replace(r.params, precision=bhr.BHR_FP64)) as s:
            s.time_steps(args.warmup)
            plain_ms.append(s.time_steps(args.steps) / args.steps)
    # each GPU runs its share one solve at a time; the job takes the slowest share
    plain_s = replicas.max_over_ranks(sum(nt * ms for nt, ms in zip(nts, plain_ms)) / 1e3, dist, device="cuda")
    all_work = [w for ws in replicas.gather_objects(work, dist) for w in ws]
    plain_value = sum(all_work) / plain_s
    mean_work = float(np.mean(all_work))
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if PRECISION == "fp64" else "f64+f32", "data": "synthetic",
        "config": {"workload": f"batch64 ({PRECISION}): 64 seeded source-free solves, a~U[0,0.99], m~U{{1..4}}, "
                               "N_r~{2048,4096,8192,16384}, N_theta~{64,128,256}, x in [-100,300], T=500",
                   "points_per_batch_step": pts / args.steps, "l2": "working set > L2 (GBs)",
                   "parallelism": f"replicas x{world} (solves sharded by work)"},
        "solves_per_s": value / mean_work, "plain_value": plain_value, "plain_solves_per_s": plain_value / mean_work,
        "speedup_vs_plain": value / plain_value,
        "e2e": {"value": pts / wall, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "wall clock around bhr_engine_step (host sync included)"},
        "gpu_launches": args.steps * 4, "clocks": clk.summary(),
    }
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def run_serve(args):
    """Served form: a seeded Poisson stream of solves (70 % source-free
    2048-4096 x 64-128, 30 % plunge-driven 8192 x 128) submitted to the
    engine as they arrive, at `--load` times the engine's measured capacity,
    with a 150 GB admission budget.  Reports solves/s and p50/p99
    time-to-waveform (submit -> waveform ready), beside the plain path that
    serves the same stream one solve at a time (measured service times,
    first-come first-served queue).  Final times are scaled by
    `--time-scale` to bound the run."""
    import threading
    import torch
    import bh_ringdown_b200 as bhr
    from bh_ringdown_b200.workloads import serve_requests, with_arrivals
    rank, local_rank, world = env_rank()
    torch.cuda.set_device(local_rank)
    dist = _dist_init(world, local_rank)
    reqs = serve_requests(args.requests, 1.0, time_scale=args.time_scale,
                          precision=bhr.BHR_MIXED if PRECISION == "mixed" else bhr.BHR_FP64)
    nts = [_solve_steps(r.params) for r in reqs]
    work = np.array([nt * r.points() for nt, r in zip(nts, reqs)], dtype=np.float64)
    budget = 150 << 30

    # capacity: a saturated engine on the first requests, device throughput
    ncal = min(len(reqs), 48)
    with bhr.Engine(device=local_rank, hbm_budget_bytes=budget) as e:
        for r in reqs[:ncal]:
            e.submit(r.params, r.traj)
        while e.stats()["queued"] > 0:
            e.step(0)
        e.step(20)
        st0 = e.stats()
        t0 = time.perf_counter()
        while e.stats()["running"] == ncal and time.perf_counter() - t0 < 2.0:
            e.step(50)
        st1 = e.stats()
    cal_rate = (st1["point_updates"] - st0["point_updates"]) / ((st1["device_ms"] - st0["device_ms"]) / 1e3)
    # per-GPU capacity (the slowest GPU's when several serve), the stream's
    # rate is `load` times all GPUs' capacity
    capacity = -replicas.max_over_ranks(-cal_rate / float(np.mean(work)), dist, device="cuda")
    rate = args.load * capacity * world
    with_arrivals(reqs, rate)
    all_reqs = reqs
    # replicas: each GPU serves its share of the stream (work-balanced), one engine per GPU
    reqs = [all_reqs[i] for i in replicas.run_shard(all_reqs, rank, world,
                                                    lambda r: replicas.request_work(r.params))]
    for r in reqs:
        r.params.device = local_rank

    # the stream through the engine
    with bhr.Engine(device=local_rank, hbm_budget_bytes=budget) as e:
        ids = [None] * len(reqs)
        if dist is not None:
            dist.barrier()
        start = time.perf_counter()

        stop = threading.Event()

        def submitter():
            for i, r in enumerate(reqs):
                delay = r.arrival_s - (time.perf_counter() - start)
                if delay > 0 and stop.wait(delay):
                    return
                if stop.is_set():
                    return
                ids[i] = e.submit(r.params, r.traj)

        th = threading.Thread(target=submitter)
        th.start()
        try:
            with ClockSampler(local_rank) as clk:
                while True:
                    running = e.step(args.chunk)
                    if running == 0:
                        st_now = e.stats()
                        if not th.is_alive() and st_now["queued"] == 0 and st_now["running"] == 0:
                            break
                        time.sleep(0.0005)
        finally:
            # the engine must outlive the submitting thread
            stop.set()
            th.join()
        makespan = replicas.max_over_ranks(time.perf_counter() - start, dist, device="cuda")
        lat, fails = [], 0
        for rid in ids:
            info = e.poll(rid)
            if info["state"] != bhr.Engine.DONE:
                fails += 1
                continue
            lat.append(info["finish_s"] - info["submit_s"])
        st = e.stats()
    lat = np.array([x for part in replicas.gather_objects(lat, dist) for x in part])
    fails = sum(replicas.gather_objects(fails, dist))
    dev_pts = sum(replicas.gather_objects(st["point_updates"], dist))
    dev_ms = replicas.max_over_ranks(st["device_ms"], dist, device="cuda")

    # the plain path: the same requests one at a time through bhr_solver (one per GPU);
    # each grid shape's one-time autotuning is done first, untimed, as a
    # long-running plain server would have done it long before
    nplain = min(len(reqs), max(1, args.plain_requests // world))
    for shape in sorted({(r.params.N, r.params.M) for r in reqs[:nplain]}):
        warm = next(r for r in reqs[:nplain] if (r.params.N, r.params.M) == shape)
        with bhr.Solver(dataclasses.replace(warm.params, precision=bhr.BHR_FP64)):
            pass
    service = []
    for r in reqs[:nplain]:
        t0 = time.perf_counter()
        with bhr.Solver(dataclasses.replace(r.params, precision=bhr.BHR_FP64)) as s:
            if r.traj is not None:
                s.set_trajectory(r.traj)
            s.run()
            s.waveform()
        service.append(time.perf_counter() - t0)
    service = np.array(service)
    # first-come first-served single server over the same arrivals; requests
    # past the measured subset reuse the subset's service times in turn
    svc = np.resize(service, len(reqs))
    fin, plat = 0.0, []
    for r, sv in zip(reqs, svc):
        fin = max(fin, r.arrival_s) + sv
        plat.append(fin - r.arrival_s)
    plat = np.array([x for part in replicas.gather_objects(list(plat), dist) for x in part])
    service = np.array([x for part in replicas.gather_objects(list(service), dist) for x in part])
    plain_capacity = world / float(np.mean(service))
    engine_capacity = capacity * world
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    out = {
        "metric": METRIC, "value": len(lat) / makespan, "unit": "solves/s", "n_gpus": world,
        "steps": int(st["batch_steps"]), "warmup": 0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if PRECISION == "fp64" else "f64+f32", "data": "synthetic",
        "config": {"workload": f"serve ({PRECISION}): {len(all_reqs)} seeded Poisson arrivals at {args.load:.0%} of measured capacity, "
                               f"70% source-free (N_r 2048/4096, N_theta 64-128), 30% plunge (8192x128); "
                               f"final times x{args.time_scale}", "hbm_budget_gb": budget / 2**30,
                   "chunk_steps": args.chunk, "arrival_rate_per_s": rate,
                   "parallelism": f"replicas x{world} (requests sharded by work, one engine per GPU)"},
        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)), "failed": fails,
        "capacity_solves_per_s": engine_capacity,
        "device_pt_updates_per_s": dev_pts / (dev_ms / 1e3),
        "plain": {"capacity_solves_per_s": plain_capacity, "p50_s": float(np.percentile(plat, 50)),
                  "p99_s": float(np.percentile(plat, 99)), "measured_requests": nplain,
                  "note": "bhr_solver one request at a time, wall-clock service times (each grid shape "
                          "autotuned beforehand, untimed), FCFS queue"},
        "capacity_vs_plain": engine_capacity / plain_capacity,
        "e2e": {"value": len(lat) / makespan, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "wall clock of the whole stream through bhr_engine_submit/step/poll"},
        "clocks": clk.summary(),
    }
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=2000)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batch64", "serve"], default=DEFAULT_WORKLOAD)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="fp64, or mixed: FP64 state and stage 1, FP32 corrections in stages 2 and 3")
    ap.add_argument("--integrator", choices=["ssprk3", "rk4"], default="ssprk3",
                    help="single-solve workloads: SSP-RK3 (the reference's) or classical RK4 (FP64 only)")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the stream")
    ap.add_argument("--time-scale", type=float, default=0.01, help="serve: factor on every request's final time")
    ap.add_argument("--load", type=float, default=0.8, help="serve: arrival rate / measured capacity")
    ap.add_argument("--chunk", type=int, default=64, help="serve: steps per engine call")
    ap.add_argument("--plain-requests", type=int, default=60, help="serve: requests timed on the plain path")
    args = ap.parse_args()
    global PRECISION, INTEGRATOR
    PRECISION = args.precision
    INTEGRATOR = args.integrator
    if INTEGRATOR == "rk4" and PRECISION == "mixed":
        ap.error("--integrator rk4 runs in FP64 only")
    if args.warmup < 3:
        args.warmup = 3
    rank, local_rank, world = env_rank()
    if args.impl == "reference" and args.workload in ("batch64", "serve"):
        run_reference(args, rank, world)
        return
    if args.workload in ("batch64", "serve"):
        (run_batch if args.workload == "batch64" else run_serve)(args)
        return
    global WORKLOAD
    WORKLOAD = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, local_rank, world)


if __name__ == "__main__":
    main()
