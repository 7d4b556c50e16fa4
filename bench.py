#!/usr/bin/env python3
"""Benchmark of the grand-potential time step (cell-updates/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cfg4|cfg2|cfg1|cfg3|cfg5] [--no-cpu-baseline]
                    [--no-extras] [--precision-steps S] [--slab]

Default workload (cfg4, the precision configuration the HBM-roofline target is
stated on): 4096x4096 grid, 3 phases, ternary alloy (2 chemical potentials),
isotropic, Neumann boundaries, 256 seeds (uniform centres, r ~ U[4,12], random
solid phase, seed 0), liquid diffusivity diag(1, 0.5), solid 0, FP64 -- the
plain drop-in step, bit-identical to the reference's.  Synthetic data: the seed
layout comes from a splitmix64 generator, the physical constants are fixed in
eshwar_dipan_b200/workloads.py.

The line's `value` is K steps of that grid in FP64, device-resident, timed with
CUDA events around one CUDA graph of exactly K steps (captured before the
warm-up, with the launch-shape autotuning), with no statistics step inside.
Beside it the line carries:
  fp32        the FP32 storage form on the same grid, same timing, and its
              max|dphi| and solute-mass difference against FP64 at every 1000
              steps of a 10^4-step run (--precision-steps);
  cfg2        the plain FP64 drop-in configuration (2048^2, anisotropic,
              periodic), same timing;
  cfg3        the batched ensemble (256 binary sims, sides 128..1024) in FP32
              and the same ensemble in FP64, and the FP32 speed-up;
  roofline    algorithmic bytes 2(N+K)*8 per cell over the kf_step launch time,
              and the DRAM bytes ncu counted for that launch;
  e2e         the same steps through the C ABI with host buffers;
  cpu_baseline  the reference's serial C step timed on this host's cores.

A step is one explicit time step of the whole grid (phase-field pass +
concentration pass + boundary handling).  Cell-updates count interior cells
x steps.  With N>1 (torchrun) every rank runs its own replica of the grid;
value is the sum over ranks, timed as the max over ranks.  With --slab the
grid is instead split along x over the ranks (eshwar_dipan_b200/slab.py), one
halo exchange per step, and value is the one grid's cell-updates per second.
"""
import argparse
import concurrent.futures
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

from eshwar_dipan_b200.workloads import ensemble, filling_text, input_text, workload, write_workload  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "gp_ref_harness")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one kf_step
# launch in FP64, from ncu captures of the step at these workloads (the
# summaries are under profiles/; cfg4: an early step, as the timed ones are)
NCU_TRAFFIC = {"cfg2": 116.6e6, "cfg4": 638.8e6}

# steps run untimed before the warm-up: the launch-shape autotuner times one
# 100-step chunk per candidate shape (at most five), then the chosen shape's
# 100-step graph is captured
PREP_STEPS = 600


def cpu_info():
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    return {"model": model, "logical_cpus": os.cpu_count(), "usable_cpus": usable}


def nvml_handle(local):
    """NVML handle of the CUDA device this rank uses (matched by PCI bus id,
    since NVML ignores CUDA_VISIBLE_DEVICES), or None."""
    try:
        import pynvml
        pynvml.nvmlInit()
    except Exception:
        return None
    try:
        import torch
        pr = torch.cuda.get_device_properties(local)
        bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
    except Exception:
        try:
            return pynvml.nvmlDeviceGetHandleByIndex(local)
        except Exception:
            return None


_REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}


class NvmlSampler:
    """SM clock and clock-event reasons read through NVML in a tight loop on a
    host thread while the timed region runs (the main thread waits inside a
    libgp call, which releases the GIL)."""

    def __init__(self, handle):
        self.h = handle
        self.samples = []
        self.stop = threading.Event()

    def _run(self):
        import pynvml
        get_r = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                self.samples.append((pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM), get_r(self.h)))
            except Exception:
                return
            time.sleep(0.0002)

    def __enter__(self):
        if self.h is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
            time.sleep(0.002)
        return self

    def __exit__(self, *a):
        if self.h is not None:
            self.stop.set()
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "samples": 0, "reasons": ["unsampled"], "source": "nvml"}
        import pynvml
        reasons = sorted(n for n, bit in _REASONS.items() if any(r & bit for _, r in self.samples))
        try:
            mx = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            mx = None
        return {"sm_mhz": statistics.median(c for c, _ in self.samples), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples), "source": "nvml, polled during the timed region"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 100 ms in the background
    (for windows of a second or more)."""
    Q = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, handle):
        self.sel = None
        if handle is not None:
            try:
                import pynvml
                self.sel = pynvml.nvmlDeviceGetPciInfo(handle).busId
                self.sel = self.sel.decode() if isinstance(self.sel, bytes) else self.sel
            except Exception:
                self.sel = None
        self.proc = None
        self.lines = []

    def __enter__(self):
        if shutil.which("nvidia-smi") and self.sel:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.sel, "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, pw, reasons = [], None, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                pw.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(pw) if pw else None, "source": "nvidia-smi every 100 ms"}


def reduce_over_ranks(dist, value, op="max"):
    """max (or sum) of a float over the ranks of the process group; the
    value itself without one.  NCCL reduces a CUDA tensor, gloo a CPU one."""
    if not dist:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def ensemble_shard(rank):
    """The simulations of one rank: rank r steps the 256-member ensemble
    drawn with seed r, its own shard of a 256*N-member ensemble (rank 0's is
    the cfg3 ensemble)."""
    return ensemble(seed=rank)


def measured_peaks():
    try:
        return json.load(open(PEAKS))
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# CPU baselines: the reference's own serial C step (oracle/_ref), else the
# oracle's restatement of it
# ---------------------------------------------------------------------------

def run_reference(ip, fp, nsteps):
    """The reference's own serial C implementation (built from its sources into
    oracle/_ref): device-free, single thread.  Returns seconds of the time loop."""
    with tempfile.TemporaryDirectory() as d:
        for _ in range(4):   # the reference crashes at random at start-up; retry
            r = subprocess.run([HARNESS, ip, fp, "time", str(nsteps)], capture_output=True, text=True, cwd=d)
            if r.returncode == 0:
                return float(r.stdout.strip().splitlines()[-1])
    raise RuntimeError("reference harness failed: " + r.stderr[-400:])


def run_oracle_port(ip, fp, nsteps):
    """CPU restatement (oracle/liboracle.so), single thread; seconds of the steps."""
    import eshwar_dipan_b200 as gp
    from oracle_py import Oracle
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=0)
    o.set(phi, mu)
    o.smooth(max(0, p.nsmooth - 1))
    t0 = time.perf_counter()
    o.step(nsteps)
    return time.perf_counter() - t0


def cpu_baseline(name, target_s=15.0):
    """Reference timed on a bounded sample: the same configuration shrunk 4x per
    axis (same seed density), enough steps for ~target_s of CPU time, on one
    core (the reference's solver is serial)."""
    scale = 4
    with tempfile.TemporaryDirectory() as d:
        ip, fp, desc, kw = write_workload(d, name, scale)
        cells = kw["mesh"][0] * kw["mesh"][1]
        kind = "reference" if os.path.exists(HARNESS) else "port"
        runner = run_reference if kind == "reference" else run_oracle_port
        t1 = runner(ip, fp, 2)
        steps = max(2, min(400, int(target_s / max(t1 / 2, 1e-3))))
        t = runner(ip, fp, steps)
    return {"value": cells * steps / t, "unit": "cell-updates/s", "cores": 1, "kind": kind, "cpu": cpu_info(),
            "sample": "%s, %d time steps (after the NSMOOTH-1 smoothing sweeps, untimed), %.1f s on one core "
                      "(the reference's GP solver is serial)" % (desc, steps, t)}


def cpu_baseline_ensemble(target_s=12.0):
    """The ensemble on the host: one reference process per usable core, each
    stepping a different member for about target_s; aggregate cell-updates/s of
    the processes running side by side."""
    info = cpu_info()
    ncores = max(1, info["usable_cpus"])
    kind = "reference" if os.path.exists(HARNESS) else "port"
    runner = run_reference if kind == "reference" else run_oracle_port
    members = ensemble()[:ncores]
    d = tempfile.mkdtemp(prefix="gpcpu")
    jobs = []
    for i, (kw, seeds) in enumerate(members):
        ip, fp = os.path.join(d, "m%d.in" % i), os.path.join(d, "m%d_fill.in" % i)
        open(ip, "w").write(input_text(**kw))
        open(fp, "w").write(filling_text(seeds))
        cells = kw["mesh"][0] * kw["mesh"][1]
        # about 4e6 binary cell-updates per second per core
        steps = max(2, min(4000, int(target_s * 4e6 / cells)))
        jobs.append((ip, fp, cells, steps))
    with concurrent.futures.ThreadPoolExecutor(ncores) as pool:
        times = list(pool.map(lambda j: runner(j[0], j[1], j[3]), jobs))
    shutil.rmtree(d, ignore_errors=True)
    rate = sum(c * s / t for (_, _, c, s), t in zip(jobs, times))
    return {"value": rate, "unit": "cell-updates/s", "cores": ncores, "kind": kind, "cpu": info,
            "sample": "ensemble members 0..%d (sides %s), one serial reference process per core side by side, "
                      "%.0f-%.0f s each" % (ncores - 1, sorted({m[0]["mesh"][0] for m in members}),
                                            min(times), max(times))}


def reference_arm(args, rank, world):
    """--impl reference: the reference's own serial C step on this host (rank 0
    only), on a bounded sample of this arm's configuration."""
    if rank != 0:
        return 0
    name = args.workload
    if name == "cfg3":
        base = cpu_baseline_ensemble()
    else:
        base = cpu_baseline(name, target_s=min(60.0, 3.0 * max(1, args.steps)))
    out = {"metric": "cell-updates/s", "value": base["value"], "unit": "cell-updates/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
           "dtype": "f64", "data": "synthetic", "scaling": "weak", "vs_baseline": None,
           "config": {"workload": workload(name)[2]},
           "cpu_baseline": base,
           "e2e": {"value": base["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU measurements
# ---------------------------------------------------------------------------

def _barrier(dist):
    if dist:
        dist.barrier()


def measure_grid(gp, p, phi0, mu0, prec, K, W, handle, dist=None, sample_window=True):
    """One grid: smoothing, untimed preparation (autotuning, graph capture),
    a ~1.5 s clock window of the same steps, back to the smoothed state, W
    warm-up steps, then K steps timed with CUDA events (one K-step graph).
    Returns a dict of timings and the context (left open)."""
    sim = gp.Simulation(p, phi0, mu0, precision=prec)
    sim.smooth(p.nsmooth - 1)
    phs, mus = sim.get()
    # untimed preparation: tuning and 100-step graphs, then the K- and W-step
    # graphs for both ping-pong parities
    sim.step(PREP_STEPS, stats=False)
    for _ in range(2):
        sim.step(K, stats=False)
        sim.step(W, stats=False)
        sim.step(1, stats=False)
    win = None
    if sample_window:
        ms100 = sim.step_timed(100)[0]
        nwin = 100 * max(1, int(1500.0 / max(ms100, 1e-3)))
        with ClockSampler(handle) as clk:
            ms_win = sim.step_timed(nwin)[0]
        win = {"steps": nwin, "ms_per_step": ms_win / nwin, "clocks": clk.summary()}
    sim.set(phs, mus)
    sim.step(W, stats=False)
    _barrier(dist)
    with NvmlSampler(handle) as nv:
        tot_ms = sim.step_timed(K)[0]
    _barrier(dist)
    tot_ms = reduce_over_ranks(dist, tot_ms)
    kt = sim.kernel_times(20)
    return {"sim": sim, "ms": tot_ms, "ms_per_step": tot_ms / K, "clocks": nv.summary(), "window": win,
            "kernels": kt}


def measure_batch(gp, params, fields, prec, K, W, dist=None):
    """The ensemble as one batch: smoothing, untimed preparation, W warm-up
    steps, K steps timed with CUDA events."""
    b = gp.Batch(params, fields, precision=prec)
    b.smooth(params[0].nsmooth - 1)
    b.step(PREP_STEPS, stats=False)
    for _ in range(2):
        b.step(K, stats=False)
        b.step(W, stats=False)
        b.step(1, stats=False)
    b.step(W, stats=False)
    _barrier(dist)
    ms, _ = b.step_timed(K)
    _barrier(dist)
    ms = reduce_over_ranks(dist, ms)
    st = b.step(1)
    b.close()
    return ms, st


def load_ensemble(gp, rank, work):
    params, fields = [], []
    for i, (kw, seeds) in enumerate(ensemble_shard(rank)):
        ip, fp = os.path.join(work, "e%d.in" % i), os.path.join(work, "e%d_fill.in" % i)
        open(ip, "w").write(input_text(**kw))
        open(fp, "w").write(filling_text(seeds))
        p = gp.load_params(ip)
        params.append(p)
        fields.append(gp.fill(p, fp))
    return params, fields


def precision_run(gp, p, phi0, mu0, nsteps, every=1000):
    """FP32 storage form against the FP64 step from the same smoothed state:
    max|dphi|, RMS dphi and the relative solute-mass difference at every
    `every` steps up to nsteps."""
    s64 = gp.Simulation(p, phi0, mu0, precision=gp.GP_FP64)
    s32 = gp.Simulation(p, phi0, mu0, precision=gp.GP_FP32)
    for s in (s64, s32):
        s.smooth(p.nsmooth - 1)
    cps = []
    done = 0
    while done < nsteps:
        n = min(every, nsteps - done)
        st64 = s64.step(n)
        st32 = s32.step(n)
        done += n
        a, b = s32.get()[0], s64.get()[0]
        d = np.abs(a - b)
        cps.append({"step": done, "max_abs_dphi": float(d.max()), "rms_dphi": float(np.sqrt((d * d).mean())),
                    "cells_over_1e-4": int((d > 1e-4).sum()),
                    "mass_rel_diff": [abs(x - y) / abs(y) for x, y in zip(st32["comp_sum"], st64["comp_sum"])]})
    s64.close()
    s32.close()
    return {"steps": nsteps, "every": every, "checkpoints": cps,
            "max_abs_dphi_over_run": max(c["max_abs_dphi"] for c in cps),
            "max_mass_rel_diff_over_run": max(max(c["mass_rel_diff"]) for c in cps)}


def vtk_overlap(gp, p, phi0, mu0, work, steps=3000, every=1000):
    """`steps` steps with a binary VTK of the state every `every` steps,
    written (a) after gp_get, stopping the steps, as the reference's time loop
    does, and (b) by gp_vtk_write_async while the next steps run; wall clock
    of each, and of the steps alone."""
    out = {"steps": steps, "every": every, "format": "binary"}
    with gp.Simulation(p, phi0, mu0) as s:
        s.step(102, stats=False)
        t0 = time.perf_counter()
        s.step(steps, stats=False)
        s.get()
        out["steps_only_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        for i in range(steps // every):
            s.step(every, stats=False)
            ph, m = s.get()
            gp.vtk_write(p, os.path.join(work, "sync_%d.vtk" % i), ph, m, ascii=0)
        out["sync_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        for i in range(steps // every):
            s.step(every, stats=False)
            s.vtk_write_async(os.path.join(work, "async_%d.vtk" % i), ascii=0)
        s.vtk_wait()
        out["async_s"] = time.perf_counter() - t0
    out["bytes_per_file"] = os.path.getsize(os.path.join(work, "async_0.vtk"))
    return out


def e2e_run(gp, p, phi0, mu0, K, W, dist, savet=1000):
    """End to end through the C ABI with host buffers: gp_init uploads the host
    state, gp_smooth and gp_step run, and every SAVET steps (and after the
    last) the step statistics are returned and the state is read back to the
    host, as the CLI does before its progress line and VTK file; wall clock
    around the whole sequence."""
    import ctypes
    L = gp._abi.lib()
    prog = gp.Stats()
    # the caller's arrays for the read-backs exist before the timed region,
    # pages touched (a caller keeps its arrays; the first-touch page faults
    # of fresh memory belong to the allocation, not to the copy)
    phi_h = np.empty_like(phi0)
    mu_h = np.empty_like(mu0)
    phi_h.fill(0.0)
    mu_h.fill(0.0)
    _barrier(dist)
    t0 = time.perf_counter()
    h = ctypes.c_void_p()
    gp._abi.check(L.gp_init(ctypes.byref(h), ctypes.byref(p), phi0.ctypes.data_as(ctypes.c_void_p),
                            mu0.ctypes.data_as(ctypes.c_void_p), gp.GP_FP64))
    gp._abi.check(L.gp_smooth(h, p.nsmooth - 1), h)
    total, done, ngets = W + K, 0, 0
    while done < total:
        n = min(savet, total - done)
        gp._abi.check(L.gp_step(h, n, ctypes.byref(prog)), h)
        gp._abi.check(L.gp_get(h, phi_h.ctypes.data_as(ctypes.c_void_p), mu_h.ctypes.data_as(ctypes.c_void_p)), h)
        done += n
        ngets += 1
    t = time.perf_counter() - t0
    L.gp_destroy(h)
    _barrier(dist)
    return reduce_over_ranks(dist, t), total, ngets


def roofline(kt, cells, bpc, traffic, hbm, peak_src, step_ms):
    """Roofline of the dominant kernel (kf_step, fused shape; else the
    bulk/interface pair) from its average launch time over kt's 20 steps."""
    nk = 20
    if kt["fused"]:
        launch_ms = kt["step_ms"] / nk
        kname = "kf_step"
    else:
        launch_ms = (kt["bulk_ms"] + kt["iface_ms"]) / nk
        kname = "kf_classify+kf_bulk+kf_general"
    achieved = bpc * cells / (launch_ms / 1e3) / 1e9
    out = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
           "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_src,
           "bytes_per_cell": bpc, "algorithmic_bytes": bpc * cells, "launch_ms": launch_ms,
           "step_frac": bpc * cells / (step_ms / 1e3) / 1e9 / hbm,
           "note": "achieved = 2(N+K)*s algorithmic bytes per cell x cells / average %s launch (CUDA events "
                   "around each launch, 20 steps launched one by one); step_frac uses the whole step "
                   "(classification included) of the timed graph" % kname}
    if traffic:
        out["dram_gbs"] = traffic / (launch_ms / 1e3) / 1e9
        out["dram_frac"] = out["dram_gbs"] / hbm
        out["traffic_unit"] = "bytes per kf_step launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)"
    return out


def run_grid(args, rank, world, local, dist):
    """cfg1 / cfg2 / cfg4: one grid per rank (replicas for N>1)."""
    import eshwar_dipan_b200 as gp
    K, W = args.steps, args.warmup
    handle = nvml_handle(local)
    work = tempfile.mkdtemp(prefix="gpbench")
    ip, fp, desc, kw = write_workload(work, args.workload)
    p = gp.load_params(ip)
    phi0, mu0 = gp.fill(p, fp)
    N, K2 = p.numphases, p.numcomponents - 1
    cells = p.mesh_x * p.mesh_y
    state_bytes = (N + K2) * cells * 8
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    bpc = 2 * (N + K2) * 8

    # ---- FP64 headline ------------------------------------------------------
    m64 = measure_grid(gp, p, phi0, mu0, gp.GP_FP64, K, W, handle, dist, sample_window=not args.no_clock_window)
    st = m64["sim"].step(1)   # progress record after the timed steps (untimed)
    m64["sim"].close()
    value = world * cells * K / (m64["ms"] / 1e3)

    # ---- FP32 storage form, same grid and timing ------------------------------
    m32 = None
    if not args.no_fp32:
        m32 = measure_grid(gp, p, phi0, mu0, gp.GP_FP32, K, W, handle, dist, sample_window=not args.no_clock_window)
        m32["sim"].close()
    prec = None
    if m32 is not None and args.precision_steps > 0 and rank == 0:
        prec = precision_run(gp, p, phi0, mu0, args.precision_steps)

    # ---- the other configurations of the metric --------------------------------
    extras = {}
    if not args.no_extras:
        Kx = max(K, 200)
        if args.workload != "cfg2":
            ip2, fp2, desc2, _ = write_workload(work, "cfg2")
            p2 = gp.load_params(ip2)
            f2 = gp.fill(p2, fp2)
            m = measure_grid(gp, p2, f2[0], f2[1], gp.GP_FP64, Kx, W, handle, dist, sample_window=False)
            c2 = p2.mesh_x * p2.mesh_y
            extras["cfg2"] = {"workload": "cfg2: " + desc2, "dtype": "f64", "steps": Kx, "warmup": W,
                              "value": world * c2 * Kx / (m["ms"] / 1e3), "unit": "cell-updates/s",
                              "ms_per_step": m["ms_per_step"], "clocks": m["clocks"],
                              "roofline": roofline(m["kernels"], c2, 80, NCU_TRAFFIC.get("cfg2"), hbm, peak_src,
                                                   m["ms_per_step"])}
            m["sim"].close()
        params, fields = load_ensemble(gp, rank, work)
        ecells = sum(q.mesh_x * q.mesh_y for q in params)
        ms32, st32 = measure_batch(gp, params, fields, gp.GP_FP32, Kx, W, dist)
        ms64, _ = measure_batch(gp, params, fields, gp.GP_FP64, Kx, W, dist)
        all_cells = reduce_over_ranks(dist, ecells, op="sum")
        v32 = all_cells * Kx / (ms32 / 1e3)
        v64 = all_cells * Kx / (ms64 / 1e3)
        extras["cfg3"] = {
            "workload": "cfg3: 256 binary 2-phase simulations, sides log-uniform [128,1024] x32, c0~U[0.40,0.48], "
                        "delta~U[0,0.05], 1-8 seeds; one persistent launch per step over all of them",
            "simulations": len(params), "cells": ecells, "steps": Kx, "warmup": W,
            "untimed_before": "smoothing, %d preparation steps" % (PREP_STEPS + 2 * (Kx + W + 1)),
            "fp32": {"value": v32, "unit": "cell-updates/s", "ms_per_step": ms32 / Kx,
                     "roofline_frac": 24 * ecells / (ms32 / Kx / 1e3) / 1e9 / hbm,
                     "nonfinite": sum(x["nonfinite"] for x in st32)},
            "fp64": {"value": v64, "unit": "cell-updates/s", "ms_per_step": ms64 / Kx,
                     "roofline_frac": 48 * ecells / (ms64 / Kx / 1e3) / 1e9 / hbm},
            "fp32_speedup_vs_fp64": ms64 / ms32,
        }
        if not args.no_cpu_baseline and rank == 0:
            extras["cfg3"]["cpu_baseline"] = cpu_baseline_ensemble()

    # ---- end to end through the C ABI with host buffers: seven runs (wall
    # clock, host-side work included; a shared host makes single runs noisy),
    # the median reported ----------------------------------------------------
    runs = [e2e_run(gp, p, phi0, mu0, K, W, dist) for _ in range(7)]
    t_runs = sorted(r[0] for r in runs)
    t_e2e, e2e_steps, ngets = t_runs[len(t_runs) // 2], runs[0][1], runs[0][2]

    if rank == 0:
        kt = m64["kernels"]
        out = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": m64["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (splitmix64 seed layout, seed 0)",
            "config": {"workload": args.workload + ": " + desc, "grid": [p.mesh_x, p.mesh_y], "phases": N,
                       "components": K2, "precision": "fp64 plain (bit-identical to the reference step)",
                       "state_bytes": state_bytes,
                       "l2": "inputs larger than L2: %.0f MB of state read and written per step"
                             % (2 * state_bytes / 1e6),
                       "timed": "K steps as one CUDA graph of K steps (captured untimed before the warm-up), "
                                "no statistics step inside; CUDA events on the context's stream",
                       "untimed_before": "smoothing, %d preparation steps (launch-shape tuning, graph capture), "
                                         "a clock window of %d steps, then back to the smoothed state"
                                         % (PREP_STEPS + 2 * (K + W + 1),
                                            m64["window"]["steps"] if m64["window"] else 0),
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": roofline(kt, cells, bpc, NCU_TRAFFIC.get(args.workload), hbm, peak_src, m64["ms_per_step"]),
            "e2e": {"value": world * cells * e2e_steps / t_e2e, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": state_bytes / e2e_steps,
                    "d2h_bytes_per_step": state_bytes * ngets / e2e_steps,
                    "includes": "gp_init upload of the host state, %d smoothing sweeps, %d steps, statistics and a "
                                "state read-back every 1000 steps and after the last, into host arrays allocated "
                                "(and touched) before the timed region; the median of seven runs" %
                                (p.nsmooth - 1, e2e_steps),
                    "runs_s": t_runs},
            "gpu_launches": K * kt["launches_per_step"],
            "clocks": m64["clocks"],
            "clock_window": m64["window"],
            "kernels_ms_per_launch": {k: v / 20 for k, v in kt.items() if k.endswith("_ms") and v},
            "stats_last_step": st,
        }
        if m32 is not None:
            v32 = world * cells * K / (m32["ms"] / 1e3)
            a32 = (N + K2) * 2 * 4 * cells / (m32["ms_per_step"] / 1e3) / 1e9
            out["fp32"] = {"value": v32, "unit": "cell-updates/s", "ms_per_step": m32["ms_per_step"],
                           "speedup_vs_fp64": v32 / value,
                           "roofline": roofline(m32["kernels"], cells, (N + K2) * 2 * 4, None, hbm, peak_src,
                                                m32["ms_per_step"]),
                           "clocks": m32["clocks"], "clock_window": m32["window"],
                           "form": "fields stored and stepped in FP32, stochastic rounding of each commit; "
                                   "interface dc/dmu inversion, anisotropy and all sums in FP64"}
            if prec:
                out["fp32"]["error_vs_fp64"] = prec
            out["gpu_launches"] += K * m32["kernels"]["launches_per_step"]
            out["roofline"]["fp32_frac"] = a32 / hbm
        out.update(extras)
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(args.workload)
        if world == 1 and args.vtk:
            out["vtk_output"] = vtk_overlap(gp, p, phi0, mu0, work)
        print(json.dumps(out), flush=True)
    shutil.rmtree(work, ignore_errors=True)
    return 0


def run_ensemble(args, rank, world, local, dist):
    """cfg3 alone: the batched ensemble through gp_batch_* (FP32 storage), with
    the same ensemble in FP64 beside it."""
    import eshwar_dipan_b200 as gp
    K, W = args.steps, args.warmup
    work = tempfile.mkdtemp(prefix="gpens")
    params, fields = load_ensemble(gp, rank, work)
    cells = sum(p.mesh_x * p.mesh_y for p in params)
    N, K2 = 2, 1
    handle = nvml_handle(local)
    with NvmlSampler(handle) as nv:
        tot_ms, st = measure_batch(gp, params, fields, gp.GP_FP32, K, W, dist)
    ms64, _ = measure_batch(gp, params, fields, gp.GP_FP64, K, W, dist)

    # end to end: upload of every simulation, smoothing, steps, read-back of all
    _barrier(dist)
    t0 = time.perf_counter()
    b = gp.Batch(params, fields, precision=gp.GP_FP32)
    b.smooth(params[0].nsmooth - 1)
    b.step(W + K, stats=False)
    for i in range(len(params)):
        b.get(i)
    t_e2e = time.perf_counter() - t0
    b.close()
    _barrier(dist)
    t_e2e = reduce_over_ranks(dist, t_e2e)
    all_cells = reduce_over_ranks(dist, cells, op="sum")   # every rank's shard
    shutil.rmtree(work, ignore_errors=True)
    if rank != 0:
        return 0
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs") or 6650.0
    bpc = 2 * (N + K2) * 4
    value = all_cells * K / (tot_ms / 1e3)
    achieved = bpc * cells * K / (tot_ms / 1e3) / 1e9
    e2e_steps = W + K
    host_bytes = cells * (N + K2) * 8
    out = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": tot_ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (splitmix64 ensemble, seed 0)",
        "config": {"workload": "cfg3: 256 binary 2-phase simulations, sides log-uniform [128,1024] x32, "
                               "c0~U[0.40,0.48], delta~U[0,0.05], 1-8 seeds; FP32 storage, FP64 dc/dmu and sums",
                   "simulations": len(params), "cells": cells,
                   "l2": "inputs larger than L2: %.0f MB state per step" % (2 * cells * (N + K2) * 4 / 1e6),
                   "timed": "K steps as one CUDA graph after smoothing, %d preparation steps and W warm-up steps"
                            % (PREP_STEPS + 2 * (K + W + 1)),
                   "parallelism": "ensemble shards (rank r: the 256 simulations of seed r)" if world > 1 else "single"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "bytes_per_cell": bpc,
                     "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback"},
        "e2e": {"value": all_cells * e2e_steps / t_e2e, "unit": "cell-updates/s",
                "h2d_bytes_per_step": host_bytes / e2e_steps, "d2h_bytes_per_step": host_bytes / e2e_steps,
                "includes": "gp_batch_create upload of 256 simulations, %d smoothing sweeps, %d steps, "
                            "read-back of every simulation" % (params[0].nsmooth - 1, e2e_steps)},
        "gpu_launches": 2 * K,
        "clocks": nv.summary(),
        "nonfinite": sum(x["nonfinite"] for x in st),
        "fp64_same_ensemble": {"value": all_cells * K / (ms64 / 1e3), "unit": "cell-updates/s",
                               "ms_per_step": ms64 / K, "fp32_speedup": ms64 / tot_ms},
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_ensemble()
    print(json.dumps(out), flush=True)
    return 0


def run_adjoint(args, rank, world, local, dist):
    """cfg5: gradients of the L2 mismatch of the final phi (target from a run with
    Tau, dab, epsilon, GAMMA 5% larger) through the FP64 steps, by gp_adjoint."""
    import ctypes
    import eshwar_dipan_b200 as gp
    work = tempfile.mkdtemp(prefix="gpadj")
    ip, fp, desc, kw = write_workload(work, "cfg5")
    p = gp.load_params(ip)
    phi0, mu0 = gp.fill(p, fp)
    with gp.Simulation(p, phi0, mu0) as s:
        s.smooth(p.nsmooth - 1)
        phi, mu = s.get()
    nsteps = args.steps
    q = gp.Params()
    ctypes.memmove(ctypes.byref(q), ctypes.byref(p), ctypes.sizeof(p))
    q.tau_ab[0][1] = q.tau_ab[1][0] = 1.05 * p.tau_ab[0][1]
    q.dab[0][1] = q.dab[1][0] = 1.05 * p.dab[0][1]
    q.epsilon = 1.05 * p.epsilon
    q.gamma[0][1] = q.gamma[1][0] = 1.05 * p.gamma[0][1]
    with gp.Simulation(q, phi, mu) as s:
        s.step(nsteps, stats=False)
        target = s.get()[0]
    with gp.Simulation(p, phi, mu) as s:
        s.step(args.warmup, stats=False)
    with gp.Simulation(p, phi, mu) as s:
        s.step(nsteps, stats=False)     # graphs of this length captured
        s.set(phi, mu)
        fwd_ms, _, _, _ = s.step_timed(nsteps)
    handle = nvml_handle(local)
    with NvmlSampler(handle) as nv:
        with gp.Simulation(p, phi, mu) as s:
            g = s.adjoint(nsteps, target_phi=target)
    cells = p.mesh_x * p.mesh_y
    adj_ms = g["ms_forward"] + g["ms_reverse"]
    if rank == 0:
        out = {"metric": "cell-updates/s", "value": world * cells * nsteps / (adj_ms / 1e3), "unit": "cell-updates/s",
               "n_gpus": world, "steps": nsteps, "warmup": args.warmup, "ms_per_step": adj_ms / nsteps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (one seed at the centre)",
               "config": {"workload": "cfg5: " + desc, "grid": [p.mesh_x, p.mesh_y], "phases": 2, "components": 1,
                          "loss": "1/2 sum (phi_T - target)^2, target from Tau, dab, epsilon, GAMMA x 1.05",
                          "states_kept": g["snapshots"], "steps_recomputed": g["recomputed"],
                          "parallelism": "single"},
               "adjoint": {"loss": g["loss"], "d_tau": g["d_tau"], "d_mobility": -g["d_tau"] * p.tau_ab[0][1] ** 2,
                           "d_dab": g["d_dab"], "d_epsilon": g["d_epsilon"], "d_gamma": g["d_gamma"],
                           "max_abs_dphi0": float(np.abs(g["phi0_bar"]).max()),
                           "ms_forward_pass": g["ms_forward"], "ms_reverse_pass": g["ms_reverse"],
                           "ms_plain_forward": fwd_ms, "cost_vs_forward": adj_ms / fwd_ms},
               # forward: kf_classify + kf_step per step, recomputed steps too; reverse: four
               # kernels per step, and two more per step whose delta-phi is not on the tape
               "gpu_launches": 2 * (nsteps + g["recomputed"]) + 4 * nsteps
                               + (2 * nsteps if g["snapshots"] < nsteps - 1 else 0),
               "clocks": nv.summary(),
               "note": "value = cell-updates of the differentiated steps per second of forward + reverse"}
        print(json.dumps(out), flush=True)
    shutil.rmtree(work, ignore_errors=True)
    return 0


def run_slab(args, rank, world, local, dist):
    """--slab: one grid of the workload split along x over the ranks (one
    slab per GPU, 3 halo rows each side, the halo rows exchanged after every
    step by NCCL point-to-point messages on the context's stream).  Strong
    scaling: value is the grid's cell-updates per second, timed as the max
    over ranks of K steps with their exchanges."""
    import torch

    import eshwar_dipan_b200 as gp
    from eshwar_dipan_b200.slab import GpuSlab, SlabPlan, SlabRunner, TorchTransport, reduce_stats
    K, W = args.steps, args.warmup
    work = tempfile.mkdtemp(prefix="gpbench")
    ip, fp, desc, kw = write_workload(work, args.workload)
    p = gp.load_params(ip)
    phi0, mu0 = gp.fill(p, fp)
    plan = SlabPlan(p, world, rank)
    slab = GpuSlab(plan, phi0, mu0)
    run = SlabRunner(plan, slab, TorchTransport(dist, stream=slab.stream) if dist else None)
    run.smooth(p.nsmooth - 1)
    run.step(W)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    _barrier(dist)
    ev0.record(slab.stream)
    run.step(K)
    ev1.record(slab.stream)
    torch.cuda.synchronize()
    _barrier(dist)
    ms = reduce_over_ranks(dist, ev0.elapsed_time(ev1))
    slab.step_stats(1)
    run.exchange()

    def allreduce(a, op):
        if not dist:
            return a
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        dist.all_reduce(t, op={"max": dist.ReduceOp.MAX, "min": dist.ReduceOp.MIN, "sum": dist.ReduceOp.SUM}[op])
        return t.cpu().numpy()
    st = reduce_stats(slab.stats(), allreduce)
    slab.close()
    cells = p.mesh_x * p.mesh_y
    if rank == 0:
        print(json.dumps({
            "metric": "cell-updates/s", "value": cells * K / (ms / 1e3), "unit": "cell-updates/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload + ": " + desc, "grid": [p.mesh_x, p.mesh_y],
                       "slabs": world, "halo_rows": plan.halo, "rows_per_rank": [plan.bounds[r + 1] - plan.bounds[r]
                                                                             for r in range(world)],
                       "inputs_vs_l2": "larger than L2" if 2 * (p.numphases + p.numcomponents - 1) * cells * 8
                       > 126e6 else "smaller than L2"},
            "stats": {"phi_max": list(st["phi_max"]), "mu_max": list(st["mu_max"]), "nonfinite": st["nonfinite"]},
            "e2e": None,
            "note": "one grid split over the ranks; the halo rows cross NVLink once per step"}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg4", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32 form beside the FP64 headline")
    ap.add_argument("--no-extras", action="store_true", help="skip the cfg2 and cfg3 lines beside the headline")
    ap.add_argument("--precision-steps", type=int, default=None,
                    help="steps of the FP32-vs-FP64 error run (default 10000 for cfg4, else 0)")
    ap.add_argument("--vtk", action="store_true", help="also time VTK output in the loop vs in the background")
    ap.add_argument("--slab", action="store_true",
                    help="split the grid along x over the ranks (strong scaling) instead of one replica per rank")
    ap.add_argument("--no-clock-window", action="store_true",
                    help="skip the ~1.5 s nvidia-smi clock window (short runs under a profiler)")
    args = ap.parse_args()
    if args.warmup < 1 or args.steps < 1:
        raise SystemExit("--steps and --warmup must be >= 1")
    if args.precision_steps is None:
        args.precision_steps = 10000 if args.workload == "cfg4" else 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    if args.impl == "reference":
        rc = reference_arm(args, rank, world)
    elif args.workload == "cfg3":
        rc = run_ensemble(args, rank, world, local, dist)
    elif args.workload == "cfg5":
        rc = run_adjoint(args, rank, world, local, dist)
    elif args.slab:
        rc = run_slab(args, rank, world, local, dist)
    else:
        rc = run_grid(args, rank, world, local, dist)
    if dist:
        dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
