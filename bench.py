#!/usr/bin/env python
"""Throughput of the B200 space-charge kick and element push.

Workload (one step = one space-charge step: deposit, open-boundary field
solve, fused gather/kick/push pass): 4e6 protons at 2.5 MeV, 30 mA,
402.5 MHz, uncorrelated 6D Gaussian (Philox-seeded), 64x64x128 grid, the
FODO lattice with 10 steps per 0.1 m element, FP32-convolution form.
`value` = particle-steps/s with the particles resident in HBM, timed with
CUDA events on the bunch's own stream; `e2e` = the same through the C ABI
with the particles uploaded from and downloaded to pinned host memory and
the per-step lattice table and moment records crossing PCIe, wall clock.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N>1 runs one replica per GPU under torchrun (weak scaling, no collective on
the data path); rank 0 prints one JSON line.
"""
import argparse
import ctypes
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
N_PARTICLES = 4_000_000
GRID = (64, 64, 128)
METRIC = "particle-steps/s at <=1e-5 moment error vs plain FP64 GPU"
UNIT = "particle-steps/s"
# the FP32-convolution form: FP64 particles, maps, Green function and moments,
# int64 fixed-point charge, FP32 convolution and field gather
DTYPE = "f64+i64+f32conv"


def load(name, path, pkg_dir=None):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, path, submodule_search_locations=[pkg_dir] if pkg_dir else None)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def impz_pkg():
    pkg = os.path.join(ROOT, "impact-z_b200")
    return load("impz_b200", os.path.join(pkg, "__init__.py"), pkg)


def oracle_pkg():
    return load("impz_oracle", os.path.join(ROOT, "oracle", "oracle.py"))


def workload_config(steps, n=N_PARTICLES):
    return {"workload": "proton FODO: %d protons 2.5 MeV 30 mA 402.5 MHz, "
                        "6D Gaussian, grid %dx%dx%d, 10 steps per 0.1 m element" % ((n,) + GRID),
            "particles": n, "grid": list(GRID), "steps": steps, "form": "fp32-convolution",
            "l2": "no flush: 384 MB resident particle state per step exceeds the 126 MB L2",
            "parallelism": "replicas"}


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# ---------------------------------------------------------------------------
def cpu_baseline_port(n, threads, steps, max_seconds=None):
    """The oracle (C restatement of the reference's Fortran) on the host: a
    bounded sample of the same workload.  Returns (value, seconds, steps)."""
    impz = impz_pkg()
    orc = oracle_pkg()
    from impz_b200 import beams
    pts, ref = beams.gaussian_bunch(n)
    orc.set_threads(threads)
    done = 0
    t_total = 0.0
    p = pts
    refc = ref.copy()
    z = 0.0
    chunk = 1
    while done < steps:
        lat = _steps_slice(beams, done, chunk)
        t0 = time.perf_counter()
        rows, p, beam = orc.run(lat, p, 0.030, beams.PROTON_MASS_EV, 1.0, 402.5e6, refc, GRID, z)
        t_total += time.perf_counter() - t0
        refc = np.array(beam.refptcl[:])
        z = beam.z
        done += chunk
        if max_seconds is not None and t_total > max_seconds:
            break
    orc.set_threads(1)
    return n * done / t_total, t_total, done


def _steps_slice(beams, start, count):
    """Elements covering steps [start, start+count) of the 4e6-particle FODO lattice."""
    from impz_b200 import elem
    full = beams.fodo_steps(start + count)
    out, pos = [], 0
    for e in full:
        lo, hi = pos, pos + e.nseg
        a, b = max(lo, start), min(hi, start + count)
        if a < b:
            k = b - a
            vals = [e.val[i] for i in range(24)]
            out.append(elem(e.type, e.length * k / e.nseg, k, e.mapstp, vals))
        pos = hi
    return out


def run_reference(args):
    """Reference arm: the oracle port of the reference's CPU path, all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n = N_PARTICLES
    # W untimed warm-up steps (at least one), then as many of the K timed
    # steps as fit in about two minutes
    v0, t0, w = cpu_baseline_port(n, threads, max(1, args.warmup), max_seconds=60.0)
    per_step = t0 / max(w, 1)
    budget = max(1, min(args.steps, int(120.0 / max(per_step, 1e-3))))
    value, secs, done = cpu_baseline_port(n, threads, budget)
    sample = "%d of %d steps of the %d-particle %dx%dx%d workload (oracle port, %d threads)" % (
        done, args.steps, n, *GRID, threads)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": done, "warmup": w,
            "ms_per_step": 1e3 * secs / done, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (Philox-seeded Gaussian)",
            "config": workload_config(done),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(dist, t, device):
    """The largest of the ranks' times (each rank's own when not distributed):
    every multi-GPU number is the slowest replica's."""
    if dist is None:
        return t
    import torch
    tt = torch.tensor([t], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="impz", choices=["impz", "reference"])
    ap.add_argument("--particles", type=int, default=N_PARTICLES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes (fewer launches before the timed run, "
                         "for profiling a chosen launch)")
    ap.add_argument("--workload", default="fodo",
                    choices=["fodo", "small", "chicane", "scan", "serve"],
                    help="fodo: the headline 4e6-proton line; small: 1e5 protons, 32x32x64, "
                         "160 steps, plain FP64; chicane: 5e7 electrons, 64x64x2048; scan: 256 "
                         "bunches batched; serve: Poisson job stream")
    ap.add_argument("--jobs", type=int, default=0, help="scan/serve: number of bunches or jobs")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: arrivals per second")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "small":
        return run_small(args)
    if args.workload == "chicane":
        return run_chicane(args)
    if args.workload == "scan":
        return run_scan(args)
    if args.workload == "serve":
        return run_serve(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    impz = impz_pkg()
    from impz_b200 import beams
    if impz.lib().impz_set_device(local) != 0:
        raise SystemExit("no CUDA device")
    n = args.particles
    K, W = args.steps, args.warmup
    pts, ref = beams.gaussian_bunch(n, seed=beams.SEED0 + rank)
    lat = beams.fodo_steps(K)
    warm = beams.fodo_steps(W)

    b = impz.Bunch(pts, 0.030, beams.PROTON_MASS_EV, 1.0, 402.5e6, ref, GRID,
                   form=impz.FORM_FP32CONV, track_ids=False)
    tuned = None if args.no_tune else b.autotune(8)  # launch shapes picked by timing
    b.run(warm)                          # W warm-up steps (untimed): the step graphs of the
    b.upload(pts, 0.030, ref)            # tuned launch shapes are captured here
    stream = torch.cuda.ExternalStream(b.stream())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    # ---- device-timed region: K steps, state resident in HBM
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.2)
    l0 = impz.kernel_launches()
    ev0.record(stream)
    b.run_async(lat)
    ev1.record(stream)
    recs32, zs = b.run_fetch()
    torch.cuda.synchronize()
    l1 = impz.kernel_launches()
    clk = clocks.stop()
    t = max_over_ranks(dist, ev0.elapsed_time(ev1) / 1e3, "cuda")
    value = world * n * K / t

    # ---- per-kernel CUDA-event times: the same K steps again, every kernel
    # group bracketed by events on the bunch stream (graphs off)
    b.upload(pts, 0.030, ref)
    b.profile_enable(True)
    b.run(lat)
    prof = b.profile_fetch()
    b.profile_enable(False)

    # ---- the plain FP64 GPU form on the same bunch and steps: its own
    # device-timed throughput, and the reference for the moment errors
    moment_err, plain = None, None
    if not args.no_check:
        b64 = impz.Bunch(pts, 0.030, beams.PROTON_MASS_EV, 1.0, 402.5e6, ref, GRID,
                         form=impz.FORM_FP64, track_ids=False)
        b64.run(warm)
        b64.upload(pts, 0.030, ref)
        s64 = torch.cuda.ExternalStream(b64.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s64)
        b64.run_async(lat)
        e1.record(s64)
        recs64, _ = b64.run_fetch()
        torch.cuda.synchronize()
        t64 = max_over_ranks(dist, e0.elapsed_time(e1) / 1e3, "cuda")
        b64.close()
        plain = {"value": world * n * K / t64, "ms_per_step": 1e3 * t64 / K,
                 "fp32conv_over_fp64": t64 / t}
        moment_err = moment_error(impz, recs32, recs64, zs, ref)
        moment_err["per_step_fields"] = field_errors(impz, beams, pts, ref, min(K, 10))

    # ---- e2e through the C ABI with pinned host buffers
    hp = torch.empty((n, 9), dtype=torch.float64, pin_memory=True).numpy()
    hp[:] = pts
    hout = torch.empty((n, 9), dtype=torch.float64, pin_memory=True).numpy()
    arr = impz.elem_array(lat)
    nrec = ctypes.c_int()
    recs = np.zeros((K + 1, impz.MOMREC))
    zz = np.zeros(K + 1)
    L = impz.lib()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L.impz_bunch_upload(b.h, hp.ctypes.data_as(impz._D), n, 0.030, ref.ctypes.data_as(impz._D))
    L.impz_run(b.h, arr, len(lat), recs.ctypes.data_as(impz._D), zz.ctypes.data_as(impz._D),
               K + 1, ctypes.byref(nrec))
    nout = ctypes.c_longlong()
    L.impz_bunch_download(b.h, hout.ctypes.data_as(impz._D), n, ctypes.byref(nout))
    te = max_over_ranks(dist, time.perf_counter() - t0, "cuda")
    step_table_bytes = impz.lib().impz_step_params_size() * (K + 2)
    e2e = {"value": world * n * K / te, "unit": UNIT,
           "h2d_bytes_per_step": int((72 * n + step_table_bytes) / K),
           "d2h_bytes_per_step": int((72 * n + 8 * impz.MOMREC * (K + 1)) / K),
           "scope": "per job of K steps: Pts1 upload from pinned memory, lattice step table, "
                    "K steps, moment records and Pts1 download"}
    b.close()

    # ---- roofline of the dominant kernel group
    peak, peak_kind = measured_peak()
    G = GRID[0] * GRID[1] * GRID[2]
    # algorithmic bytes per step: the deposit reads the three conv1st-frame
    # columns the push stored; the Green build writes and reads the FP64
    # corners and writes Ĝ (FP32) once per plane pass
    alg = {"deposit": 24 * n + 16 * G, "scan": 12 * G, "green": 24 * G, "convolve": 76 * G,
           "efield": 4 * G + 16 * G, "push": 96 * n + 16 * G}
    kernels = {}
    total_ms = sum(v[0] for v in prof.values())
    for k, (ms, scopes) in prof.items():
        if scopes:
            per_step = ms / K / 1e3
            kernels[k] = {"scopes": scopes, "ms_total": round(ms, 3),
                          "us_per_step": round(per_step * 1e6, 2),
                          "share": round(ms / total_ms, 4),
                          "gbs": round(alg[k] / per_step / 1e9, 1)}
    dom = max(kernels, key=lambda k: kernels[k]["ms_total"])
    traffic = committed_traffic().get(dom)
    achieved = kernels[dom]["gbs"]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": alg[dom],
                "timing": "CUDA events around each kernel group on the bunch stream over a "
                          "second pass of the same K steps"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, secs, done = cpu_baseline_port(n, 1, 6, max_seconds=30.0)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "%d steps of the %d-particle %dx%dx%d workload, oracle port, 1 thread "
                         "(%.1f s)" % (done, n, *GRID, secs)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
                "warmup": W, "ms_per_step": 1e3 * t / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": DTYPE,
                "data": "synthetic (Philox-seeded 6D Gaussian protons)",
                "config": dict(workload_config(K, n), launch=tuned), "clocks": clk, "e2e": e2e,
                "gpu_launches": int(l1 - l0), "roofline": roofline, "cpu_baseline": cpu,
                "kernels": kernels, "plain_fp64": plain,
                "moment_rel_err_vs_fp64": moment_err["max"] if moment_err else None,
                "errors_vs_fp64": moment_err}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


CHICANE_N = 50_000_000
CHICANE_GRID = (64, 64, 2048)


def run_chicane(args):
    """The large-bunch line: 5e7 electrons at 250 MeV with a 1 % density
    modulation at 10 µm (flat top, 1 mm), 20 m of drift and a 4-dipole
    chicane (R56 about -20 mm), grid 64x64x2048, FP32-convolution form.
    Prints particle-steps/s of the device-timed run and the bunching factor
    at 10 µm before and after (one GPU; a bunch does not shard here)."""
    import torch
    impz = impz_pkg()
    from impz_b200 import beams
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    impz.lib().impz_set_device(local)
    n = args.particles if args.particles != N_PARTICLES else CHICANE_N
    pts, ref = beams.flat_top_bunch(n)
    lat = beams.chicane()
    K = impz.count_steps(lat)
    b = impz.Bunch(pts, 100.0, beams.ELECTRON_MASS_EV, -1.0, 1.3e9, ref, CHICANE_GRID,
                   form=impz.FORM_FP32CONV, track_ids=False)
    k = 2 * math.pi / 10e-6
    b0 = abs(b.bunching(k))
    b.run(beams.chicane(ldrift_in=0.5, drift_steps_in=args.warmup))  # warm-up steps
    b.upload(pts, 100.0, ref)
    del pts
    stream = torch.cuda.ExternalStream(b.stream())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.2)
    ev0.record(stream)
    b.run_async(lat)
    ev1.record(stream)
    recs, zs = b.run_fetch()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = ev0.elapsed_time(ev1) / 1e3
    b1 = abs(b.bunching(k))
    info = b.info()
    b.close()
    line = {"metric": METRIC, "value": n * K / t, "unit": UNIT, "n_gpus": 1, "steps": K,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE,
            "data": "synthetic (Philox-seeded flat-top electrons)",
            "config": {"workload": "electron chicane: %d electrons 250 MeV 100 A 1.3 GHz, "
                                   "1 mm flat top with 1%% modulation at 10 um, grid %dx%dx%d, "
                                   "20 m drift + 4 bends of 3 deg" % ((n,) + CHICANE_GRID),
                       "particles": n, "grid": list(CHICANE_GRID), "steps": K,
                       "form": "fp32-convolution"},
            "clocks": clk, "bunching_10um": {"before": b0, "after": b1},
            "spectral_gain_10um": b1 / b0 if b0 > 0 else None,
            "live_particles": info["nlocal"]}
    print(json.dumps(line), flush=True)
    return 0


def run_small(args):
    """The CPU-runnable configuration: 1e5 protons, 32x32x64,
    ten FODO periods with four steps per element (160 steps), plain FP64.
    The GPU run is timed with CUDA events on the bunch's stream after W
    warm-up runs; the oracle port runs the same 160 steps on all host cores
    beside it.  A launch-bound size: reported, not the headline."""
    import torch
    impz = impz_pkg()
    orc = oracle_pkg()
    from impz_b200 import beams
    torch.cuda.set_device(0)
    impz.lib().impz_set_device(0)
    cfg = beams.fodo_1e5()
    lat = cfg["lattice"]
    K = impz.count_steps(lat)
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    for _ in range(max(1, args.warmup // 3)):
        b.run(lat)
        b.upload(cfg["pts"], cfg["current"], cfg["refptcl"])
    stream = torch.cuda.ExternalStream(b.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    b.run_async(lat)
    e1.record(stream)
    b.run_fetch()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    b.close()
    n = cfg["pts"].shape[0]
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    t0 = time.perf_counter()
    orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
            cfg["refptcl"], cfg["grid"])
    tc = time.perf_counter() - t0
    orc.set_threads(1)
    line = {"metric": METRIC, "value": n * K / t, "unit": UNIT, "n_gpus": 1, "steps": K,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+i64",
            "data": "synthetic (Philox-seeded 6D Gaussian protons)",
            "config": {"workload": "proton FODO: 100000 protons, grid 32x32x64, 160 steps",
                       "form": "fp64"},
            "cpu_baseline": {"value": n * K / tc, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "the same 160 steps, oracle port (%.1f s)" % tc}}
    print(json.dumps(line), flush=True)
    return 0


def run_scan(args):
    """The batched parameter scan: 256 independent proton bunches
    (N log-uniform in [1e4, 2e6], grids 16^3 / 32x32x64 / 64x64x128, gradient
    and current drawn per bunch, 25 FODO periods = 400 steps), all advanced
    together by impz_run_batch in the FP32-convolution form (one packed launch
    per particle kernel and one per field-solve kernel and grid size, each step
    pair a CUDA graph), against the same 256 runs done one by one in the plain
    FP64 form, and one by one in the FP32 form.  Wall clock around each (the
    calls are synchronous), bunches uploaded before the clock starts."""
    import torch
    impz = impz_pkg()
    from impz_b200 import beams
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    impz.lib().impz_set_device(local)
    jobs = beams.scan_jobs(nbunch=args.jobs or 256)
    data = [beams.make_scan_bunch(j) for j in jobs]
    lats = [j["lattice"] for j in jobs]
    work = sum(j["n"] * impz.count_steps(j["lattice"]) for j in jobs)
    warm = [beams.fodo_steps(args.warmup, nseg=4)] * len(jobs)

    def make(form):
        return [impz.Bunch(p, j["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, r, j["grid"],
                           form=form, track_ids=False) for j, (p, r) in zip(jobs, data)]

    def reload(bunches):
        for b, j, (p, r) in zip(bunches, jobs, data):
            b.upload(p, j["current"], r)
        torch.cuda.synchronize()

    def one_by_one(bunches):
        for b in bunches:
            b.run(beams.fodo_steps(args.warmup, nseg=4))
        reload(bunches)
        t0 = time.perf_counter()
        for b, lat in zip(bunches, lats):
            b.run(lat)
        return time.perf_counter() - t0

    bunches = make(impz.FORM_FP32CONV)
    impz.run_batch(bunches, warm)
    reload(bunches)
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    impz.run_batch(bunches, lats)
    tb = time.perf_counter() - t0
    clk = clocks.stop()
    ts32 = one_by_one(bunches)
    for b in bunches:
        b.close()
    b64 = make(impz.FORM_FP64)
    ts64 = one_by_one(b64)
    for b in b64:
        b.close()
    line = {"metric": METRIC, "value": work / tb, "unit": UNIT, "n_gpus": 1,
            "steps": int(sum(impz.count_steps(l) for l in lats)), "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE, "data": "synthetic (Philox-seeded Gaussian)",
            "config": {"workload": "batched scan: %d proton bunches, %d particles in all, "
                                   "400 steps each" % (len(jobs), sum(j["n"] for j in jobs)),
                       "form": "fp32-convolution", "timing": "wall clock, synchronous calls"},
            "clocks": clk, "batched_s": tb,
            "one_by_one_fp64": {"seconds": ts64, "value": work / ts64},
            "one_by_one_fp32conv": {"seconds": ts32, "value": work / ts32},
            "batched_over_fp64_one_by_one": ts64 / tb}
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """The served stream: jobs arrive as a Poisson process (`--rate` per s),
    N log-uniform in [1e4, 4e6], grids 32^3 / 64^3 / 64x64x128, 100-2000
    FODO steps; the serving loop admits them under a 160 GB HBM budget.
    Reports the particle-steps/s over the whole stream and the p50/p99 job
    latency from submission to completion."""
    import threading as th
    import torch
    impz = impz_pkg()
    from impz_b200 import beams
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    impz.lib().impz_set_device(local)
    jobs = beams.serve_jobs(args.jobs or 100, args.rate)
    data = [beams.gaussian_bunch(j["n"], seed=j["seed"]) for j in jobs]
    work = sum(j["n"] * impz.count_steps(j["lattice"]) for j in jobs)
    budget = 160e9
    with impz.Server(budget_bytes=budget, max_active=64) as srv:
        # warm-up job (kernels loaded, graphs instantiated once)
        p, r = beams.gaussian_bunch(20_000)
        srv.wait(srv.submit(p, 0.03, beams.PROTON_MASS_EV, 1.0, 402.5e6, r, (32, 32, 32),
                            beams.fodo_steps(args.warmup, nseg=4)))
        ids = [None] * len(jobs)
        t0 = time.perf_counter()

        def feeder():
            for i, (j, (pp, rr)) in enumerate(zip(jobs, data)):
                delay = t0 + j["arrival"] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                ids[i] = srv.submit(pp, 0.03, beams.PROTON_MASS_EV, 1.0, 402.5e6, rr, j["grid"],
                                    j["lattice"])

        f = th.Thread(target=feeder)
        f.start()
        lat = []
        for i in range(len(jobs)):
            while ids[i] is None:
                time.sleep(0.001)
            recs, latency, queued, measured = srv.wait(ids[i])
            lat.append(latency)
        f.join()
        span = time.perf_counter() - t0
        st = srv.stats()
    lat = np.array(lat)
    line = {"metric": METRIC, "value": work / span, "unit": UNIT, "n_gpus": 1,
            "steps": int(sum(impz.count_steps(j["lattice"]) for j in jobs)),
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE,
            "data": "synthetic (Philox-seeded Gaussian)",
            "config": {"workload": "served stream: %d proton jobs, Poisson arrivals at %g/s, "
                                   "160 GB budget" % (len(jobs), args.rate),
                       "form": "fp32-convolution", "timing": "wall clock from the first arrival"},
            "latency_s": {"p50": float(np.percentile(lat, 50)),
                          "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "span_s": span, "peak_admitted_bytes": st["peak_admitted_bytes"],
            "completed": st["completed"], "failed": st["failed"]}
    print(json.dumps(line), flush=True)
    return 0


# fort.24/25/26 columns of a diagnostic row (impz_diag_row): rms sizes and
# spreads, emittances; Twiss alpha; centroids, each against the rms of its
# coordinate (a centroid near zero has no scale of its own)
RMS_COLS = {7: "x_rms", 9: "px_rms", 11: "x_emit", 13: "y_rms", 15: "py_rms", 17: "y_emit",
            19: "phase_rms", 21: "dE_rms", 23: "z_emit"}
ALPHA_COLS = {10: "x_alpha", 16: "y_alpha", 22: "z_alpha"}
CENTROID_COLS = {6: ("x_mean", 7), 8: ("px_mean", 9), 12: ("y_mean", 13), 14: ("py_mean", 15),
                 18: ("phase_mean", 19), 20: ("dE_mean", 21)}


def moment_error(impz, recs_a, recs_b, zs, ref):
    """Largest difference over all records of every reported moment column:
    rms sizes and emittances relative to their value, Twiss alpha relative to
    its largest magnitude, centroids relative to the rms of the coordinate."""
    from impz_b200 import beams
    ra = np.array([impz.diag_row(zs[i], recs_a[i], ref, beams.PROTON_MASS_EV, 402.5e6)
                   for i in range(len(recs_a))])
    rb = np.array([impz.diag_row(zs[i], recs_b[i], ref, beams.PROTON_MASS_EV, 402.5e6)
                   for i in range(len(recs_b))])
    cols = {}
    for c, name in RMS_COLS.items():
        cols[name] = float(np.max(np.abs(ra[:, c] - rb[:, c]) / np.maximum(np.abs(rb[:, c]),
                                                                          1e-300)))
    for c, name in ALPHA_COLS.items():
        cols[name] = float(np.max(np.abs(ra[:, c] - rb[:, c])) / max(np.max(np.abs(rb[:, c])),
                                                                     1e-300))
    for c, (name, s) in CENTROID_COLS.items():
        cols[name] = float(np.max(np.abs(ra[:, c] - rb[:, c])) / max(np.max(np.abs(rb[:, s])),
                                                                     1e-300))
    return {"max": max(cols.values()), "columns": cols, "records": int(len(ra))}


def field_errors(impz, beams, pts, ref, nsteps):
    """Per-step relative L2 of the potential and of the field (Ex, Ey, Ez)
    of the FP32-convolution form against the plain FP64 form, both through
    the per-step calls (drift1/quadrupole half map, conv1st, deposit,
    openBC3D, kick1 + scatter1, half map) on the first `nsteps` steps."""
    out = {"steps": nsteps, "phi_rel_l2": [], "e_rel_l2": []}
    runs = []
    for form in (impz.FORM_FP32CONV, impz.FORM_FP64):
        b = impz.Bunch(pts, 0.030, beams.PROTON_MASS_EV, 1.0, 402.5e6, ref, GRID, form=form,
                       track_ids=False)
        phis, egs, z, done = [], [], 0.0, 0
        try:
            for e in beams.fodo_steps(nsteps):
                zedge, tau, ih = z, e.length / e.nseg, 0
                rad = e.val[0] if e.type == 0 else e.val[2]
                for j in range(1, e.nseg + 1):
                    z, ih = b.map_half(e, zedge, z, tau / 2, j, ih)
                    b.sc_prepare(rad, rad)
                    b.deposit(want_rho=False, want_counts=False)
                    phis.append(b.poisson())
                    egs.append(b.kick(tau, want_e=True))
                    z, ih = b.map_half(e, zedge, z, tau / 2, j, ih)
        finally:
            b.close()
        runs.append((phis, egs))
    (p32, e32), (p64, e64) = runs
    for s in range(len(p32)):
        out["phi_rel_l2"].append(float(np.linalg.norm(p32[s] - p64[s]) / np.linalg.norm(p64[s])))
        out["e_rel_l2"].append(float(np.linalg.norm(e32[s] - e64[s]) / np.linalg.norm(e64[s])))
    return out


if __name__ == "__main__":
    sys.exit(main())
