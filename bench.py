#!/usr/bin/env python
"""Benchmark of the unsplit Godunov update on the 2D shear-layer workload.

Workload (the headline configuration): 2D unsplit CTU hydro, Kelvin-Helmholtz
shear layer on a 1024 x 1024 periodic unit square, gamma = 5/3, HLLC,
MUSCL-Hancock with the van Leer limiter, CFL 0.3, FP64 (bit-faithful path).
A step is one CFL-limited unsplit step of the whole grid (ghost fill, CFL dt,
fused update). Metric: cell-updates/s (interior cells x steps / time).

  value      device time of K steps with the state resident in HBM, L2 flushed
             before every step (the 84 MB double-buffered state fits in L2);
  e2e        the same steps through the C ABI with the state uploaded from
             pinned host memory and downloaded back every step, eight grids
             in flight on their own streams so copies overlap steps
             (one_grid_value: a single grid, nothing overlapped);
  roofline   the fused step kernel's algorithmic HBM bytes (80 B per cell
             update: 5 FP64 fields read + written) over its CUDA-event time;
  roofline_fp64  the same kernel's executed FP64 operations per cell update
             (ncu counters, profiles/step2d_hydro_kh.json) over its time, against
             a cuBLAS DGEMM measured in the run: the bound that applies;
  cpu_baseline  the DRAGON reference itself (oracle/_ref, DistGrid2D with
             core_count = host threads) on a bounded number of full steps;
  mixed      the mixed FP32/FP64 path on the same workload, with its relative
             L1 difference per field from the FP64 state;
  learned_guess  the exact solver's Newton iterations per solve on a 3D blast
             with the reference's mean guess, the analytic guess and the
             GPU-trained network's guess (training included);
  batch      2048 1D hydro + 256 2D MHD grids of uneven sizes advanced by the
             persistent work-queue kernel, against the same grids one by one,
             in mixed FP32/FP64 (with its L1 per field from FP64) and FP64;
  mhd        2D MHD Orszag-Tang 1024^2, FP64 and mixed, with the mixed path's
             L1 per field and max |div B| of both;
  stated_length  the mixed path against the FP64 path at the stated lengths of
             the two 2D configurations: the shear layer 1024^2 for 2000 steps
             and Orszag-Tang 1024^2 to t = 0.5 (relative L1 per field).

stdout carries one JSON line: the contract keys and a compact "summary" of
the sections above, last so a tail of the line keeps it; the full sections
go to stderr as one JSON line prefixed "detail: ".

``--impl reference`` times only the reference on the host cores and prints its
own line. Multi-GPU (torchrun): every rank advances its own 1024^2 grid
(replicas, weak scaling; the headline), timing is the max over ranks; then one
4096^2 grid sharded across the ranks in x slabs (DistGrid2D: halo exchange,
CFL all-reduce, all-or-nothing commit over NCCL) is timed the same way
("dist", strong scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 1024  # grid extent per axis (--grid overrides it, e.g. for profiling captures)
CELL_BYTES = 80  # 5 FP64 primitive fields read + written per cell update
METRIC = "cell-updates/s (2D unsplit CTU hydro, FP64)"
WORKLOAD = "kelvin_helmholtz_2d_1024sq_hllc_vanleer_cfl0.3_periodic"
L2_RULE = "84 MB double-buffered state < 126 MB L2: the device arm writes 256 MB before every timed step"


def config_line():
    """The workload both arms report (same keys and values)."""
    return {"workload": WORKLOAD, "grid": [N, N], "solver": "HLLC", "limiter": "vanLeer", "precision": "fp64",
            "l2": L2_RULE}


def sig(x, digits=4):
    """x with every float rounded to `digits` significant digits (lists and
    dicts recursively): the compact summary of the bench line."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}") if math.isfinite(x) else x
    if isinstance(x, dict):
        return {k: sig(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [sig(v, digits) for v in x]
    return x


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


E2E_INFLIGHT = 8  # grids whose upload / step / download overlap on separate streams (4: 1.00e9, 6: 1.07e9, 8: 1.08e9)


def e2e_run(G0, grids, dev, steps, barrier):
    """Device time (ms) of `steps` end-to-end steps on each grid in `grids`
    through the C ABI: upload of the padded state from pinned host memory,
    one CFL step, download of the result into pinned host memory. Each grid
    runs on its own stream from its own host thread (the ABI calls release
    the GIL), so one grid's copies overlap another's step; the time runs from
    an event every stream waits on to the last stream's final event."""
    import torch
    from dragon_b200 import _lib
    L = G0._lib
    streams = [torch.cuda.ExternalStream(L.dragon_gpu_stream(g._h), device=dev) for g in grids]
    pins = []
    for g in grids:
        host_in = torch.from_numpy(g.w.copy()).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        pins.append((host_in, host_out))
    barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    start.record(streams[0])
    for s in streams[1:]:
        s.wait_event(start)
    ends = [torch.cuda.Event(enable_timing=True) for _ in grids]
    errors = []

    def worker(k):
        try:
            g, (hin, hout) = grids[k], pins[k]
            pin_in = hin.numpy().ctypes.data_as(_lib.c_double_p)
            pin_out = hout.numpy().ctypes.data_as(_lib.c_double_p)
            for _ in range(steps):
                _lib.check(L.dragon_gpu_upload_prim(g._h, pin_in))
                _lib.check(L.dragon_gpu_advance_steps(g._h, 1, None))
                _lib.check(L.dragon_gpu_download_prim(g._h, pin_out))
            ends[k].record(streams[k])
        except Exception as e:  # reported after the join
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(grids))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    torch.cuda.synchronize()
    for g in grids:  # the device now holds the downloaded results; the host mirrors are stale
        g._host_dirty = False
        g._device_ran()
    return max(start.elapsed_time(e) for e in ends)


def copy_bound(dev, nbytes, cells, reps=8):
    """The host-link ceiling of the end-to-end step: `reps` pinned uploads and
    `reps` pinned downloads of one step's state, each direction on its own
    stream, alone and both at once (the two copy directions overlap), timed
    with CUDA events. Returns the per-direction bandwidths, the duplex time per
    step and the cell-updates/s a step could reach if the copies were its only
    cost."""
    import torch
    host_in = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    host_out = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d_in = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d_out = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def timed(streams_ops):
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record(torch.cuda.current_stream(dev))
        ends = []
        for s, op in streams_ops:
            s.wait_event(start)
            with torch.cuda.stream(s):
                for _ in range(reps):
                    op()
                e = torch.cuda.Event(enable_timing=True)
                e.record(s)
                ends.append(e)
        torch.cuda.synchronize()
        return max(start.elapsed_time(e) for e in ends) / reps

    def h2d():
        d_in.copy_(host_in, non_blocking=True)

    def d2h():
        host_out.copy_(d_out, non_blocking=True)

    timed([(up, h2d), (down, d2h)])  # warm-up
    h2d_ms = timed([(up, h2d)])
    d2h_ms = timed([(down, d2h)])
    duplex_ms = timed([(up, h2d), (down, d2h)])
    return {"h2d_gbs": nbytes / (h2d_ms / 1e3) / 1e9, "d2h_gbs": nbytes / (d2h_ms / 1e3) / 1e9,
            "duplex_ms_per_step": duplex_ms, "value": cells / (duplex_ms / 1e3), "unit": "cell-updates/s"}


def roofline_fp64(k_avg_ms, dev):
    """The fused FP64 step against FP64 throughput: it is bound by FP64 issue, not
    by HBM, so this is the roofline that explains it."""
    fpc = fp64_flops_per_cell()
    if not fpc or not k_avg_ms:
        return None
    peak = fp64_peak_tflops(dev)
    achieved = fpc * N * N / (k_avg_ms / 1e3) / 1e12
    return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "flops_per_cell": fpc, "kernel": "k_step2d_hydro",
            "peak_source": "cuBLAS DGEMM 4096^3 measured in this run (no FP64 figure in MEASURED_PEAKS.json)"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def traffic_from_profile():
    p = os.path.join(ROOT, "profiles", "step2d_hydro_kh.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch_full")
    return None


def fp64_flops_per_cell():
    """FP64 operations the fused step executes per cell update (ncu instruction
    counters dadd + dmul + 2 dfma of one launch over its cells)."""
    p = os.path.join(ROOT, "profiles", "step2d_hydro_kh.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get("fp64_flops_per_cell_update")
    return None


def fp64_peak_tflops(dev):
    """FP64 throughput of a cuBLAS DGEMM (4096^3, best of 5, CUDA events) on this
    GPU: the denominator of the FP64 compute roofline."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region by polling
    NVML every 2 ms from a background thread (read-only queries)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.stop = threading.Event()
        self.nv = None
        self.h = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        self.nv = pynvml
        try:
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.device.index or 0)

    def _poll(self):
        nv, h = self.nv, self.h
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), int(get_reasons(h))))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        try:
            self.h = self._handle()
            self.max_mhz = self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception as e:  # no NVML: report without clocks
            self.h = None
            self.err = str(e)
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.h is not None:
            self.t.join(timeout=1)

    def summary(self):
        if self.h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "error": getattr(self, "err", "")}
        sm = sorted(x[0] for x in self.samples)
        reasons = sorted({k for _, r in self.samples for k, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "source": "nvml 2 ms polling"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reference_baseline(steps: int, warmup: int, budget_s: float | None = None):
    """Times the DRAGON reference (oracle/_ref) on the host: DistGrid2D with
    core_count = host threads, full 1024^2 steps. With budget_s, runs as many
    steps as fit (at least one)."""
    from dragon_b200 import problems
    from oracle import refgrid
    if not refgrid.available("hydro"):
        return None, "reference library not built"
    cores = os.cpu_count() or 1
    w0, dx, dy = problems.kelvin_helmholtz_2d(N, ghosts=3)
    R = refgrid.RefGrid(2, (N, N), (dx, dy), ghosts=3, dist=True, riemann=2, limiter=2, cfl=1, core_count=cores)
    R.set_prim(w0)
    R.set_boundary([(4, 63, 1, None)])
    for _ in range(warmup):
        R.step_cfl()
    t0 = time.perf_counter()
    done = 0
    while True:
        R.step_cfl()
        done += 1
        el = time.perf_counter() - t0
        if budget_s is None and done >= steps:
            break
        if budget_s is not None and (el >= budget_s or done >= steps):
            break
    el = time.perf_counter() - t0
    R.close()
    side = math.ceil(math.sqrt(cores))  # DistGrid2D's children: ceil(sqrt(core_count))^2 (DistGrid.cpp:63-64)
    return {"value": N * N * done / el, "unit": "cell-updates/s", "cores": cores, "kind": "reference",
            "cpu_model": cpu_model(), "core_count": cores, "threads_spawned": side * side,
            "sample": f"{done} full {N}x{N} steps of the reference DistGrid2D (core_count={cores}, "
                      f"{side * side} child threads), {el:.1f} s wall"}, None


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    base = {"metric": METRIC, "unit": "cell-updates/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded KH shear layer, numpy PCG64 seed 1234)",
            "parallelism": "host threads (DistGrid2D children)", "config": config_line()}
    cb, why = reference_baseline(args.steps, args.warmup)
    if cb is None:
        base["unavailable"] = why
        print(json.dumps(base))
        return
    base["value"] = cb["value"]
    base["ms_per_step"] = 1e3 * N * N / cb["value"]
    base["cpu_baseline"] = cb
    base["e2e"] = {"value": cb["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(base))


def learned_guess_report(n=256, p_in=10.0, steps=10):
    """The learned star-pressure guess on the 3D blast configuration (n^3,
    p_in = 10): a network trained on the GPU from the configuration's training
    runs (learned.c4_training_set: seeded 128^3 blasts, inner pressure
    log-uniform in [10, 1e4], ~1e7 converged solves), then the blast run with
    the reference's mean guess, the analytic guess and the learned guess, cap
    lifted so every solve reaches the tolerance, plus the reference's own
    setting (mean guess, cap 6). The "perfect" arms start Newton from the
    converged star pressure of an uncounted first solve, exactly or with a
    relative error of 1e-9, 1e-6 or 1e-3, or from the mean guess on faces
    where that needs no more iterations: the fewest iterations any guess of
    that accuracy with a fallback to the mean can reach, i.e. the ceiling of
    the reduction such a guess can give."""
    import torch

    import dragon_b200 as dg
    from dragon_b200 import learned, problems

    t0 = time.perf_counter()
    net = learned.Network(seed=2024)
    info = learned.c4_training_set(net)
    fit = learned.fit(net, steps=6000, batch=16384, lr=3e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    out = {"train": {k: info[k] for k in ("runs", "n", "steps", "stride", "solves", "samples", "saturated_runs")},
           "workload": f"3D blast {n}^3, p_in {p_in:g}, MC, exact solver, {steps} steps"}
    out["train"].update({"rmse_ln_pstar": fit["rmse_log"], "gate": fit["gate"], "seconds": train_s})
    ref = None
    arms = [("mean_cap64", dg.GUESS_MEAN, 64, 0), ("reference_mean_cap6", dg.GUESS_MEAN, 6, 0),
            ("analytic_cap64", dg.GUESS_ANALYTIC, 64, 0), ("learned_cap64", dg.GUESS_LEARNED, 64, 0),
            ("perfect_cap64", dg.GUESS_PERFECT, 64, 0), ("perfect_err1e-9_cap64", dg.GUESS_PERFECT, 64, 9),
            ("perfect_err1e-6_cap64", dg.GUESS_PERFECT, 64, 6), ("perfect_err1e-3_cap64", dg.GUESS_PERFECT, 64, 3)]
    for name, guess, cap, err in arms:
        w, d = problems.blast_3d(n, ghosts=2, p_in=p_in)
        G = dg.Grid3D(n, n, n, d, d, d, ghosts=2, config=dg.Config(
            riemann=dg.RIEMANN_EXACT, limiter=dg.LIMITER_MC, exact_max_iters=cap, exact_guess=guess,
            perfect_guess_err_exp=err))
        G.w[...] = w
        if guess == dg.GUESS_LEARNED:
            G.set_network(net)
        G.advance_steps(1)
        G.newton_stats(reset=True)
        torch.cuda.synchronize()
        t = time.perf_counter()
        G.advance_steps(steps)
        ms = (time.perf_counter() - t) / steps * 1e3
        st = G.newton_stats()
        e = {"newton_iters_per_solve": st["newton_iters"] / max(1, st["exact_calls"]),
             "solves": st["exact_calls"], "two_rarefaction_faces": st["trrs"], "cap_hits": st["cap_hits"],
             "fallback_rate": (st["guess_rejects"] + st["judge_reruns"]) / max(1, st["exact_calls"]),
             "ms_per_step_wall": ms}
        if ref is None:
            ref = G.w.copy()
        else:
            e["rel_l1_vs_mean_cap64"] = [float(x) for x in problems.rel_l1(G.w[2:-2, 2:-2, 2:-2], ref[2:-2, 2:-2, 2:-2])]
        out[name] = e
        G.close()
    m, l_ = out["mean_cap64"]["newton_iters_per_solve"], out["learned_cap64"]["newton_iters_per_solve"]
    out["iteration_reduction_vs_mean"] = m / l_
    out["iteration_reduction_vs_analytic"] = out["analytic_cap64"]["newton_iters_per_solve"] / l_
    out["ceiling_reduction_vs_mean"] = {k[len("perfect_"):-len("_cap64")] or "exact": m / out[k]["newton_iters_per_solve"]
                                        for k in out if k.startswith("perfect")}
    net.close()
    return out


def mhd_report(n=1024, steps=20, warmup=3):
    """2D MHD Orszag-Tang n^2 (HLLD, MC, CTU + CT, BETA_GATED, periodic): the
    FP64 path and the mixed path on the same state, device time per step with
    L2 flushed, the mixed path's relative L1 per field against the FP64 state
    and max |div B| (in units of 1/dx) of both."""
    import torch

    import dragon_b200 as dg
    from dragon_b200 import problems

    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {"workload": f"2D MHD Orszag-Tang {n}^2, HLLD, MC, CTU+CT, BETA_GATED, periodic", "steps": steps + warmup}
    states = {}
    for name, prec in (("fp64", dg.PREC_FP64), ("mixed", dg.PREC_MIXED)):
        G = dg.Grid2D(n, n, dx, dy, ghosts=3, config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX, precision=prec))
        G.w[...] = w0
        G.B[...] = B0
        G.boundary = dg.Periodic()
        G.initialize_B_fields()
        G.advance_steps(warmup)
        stream = torch.cuda.ExternalStream(G._lib.dragon_gpu_stream(G._h))
        ev = []
        torch.cuda.synchronize()
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            G.advance_steps_async(1)
            b.record(stream)
            G.advance_wait()
            ev.append((a, b))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        Bf = G.B.copy()
        g = 3
        d = (Bf[g + 1:g + n + 1, g:g + n, 0] - Bf[g:g + n, g:g + n, 0]) + (Bf[g:g + n, g + 1:g + n + 1, 1] - Bf[g:g + n, g:g + n, 1])
        states[name] = (G.w.copy(), Bf)
        out[name] = {"ms_per_step": ms, "value": n * n / (ms / 1e3), "unit": "cell-updates/s",
                     "max_abs_divB_dx": float(np.abs(d).max())}
        G.close()
    g = 3
    l1 = problems.rel_l1(states["mixed"][0][g:-g, g:-g], states["fp64"][0][g:-g, g:-g])
    lb = problems.rel_l1(states["mixed"][1][g:-g, g:-g, :2], states["fp64"][1][g:-g, g:-g, :2])
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["mixed"]["rel_l1_vs_fp64_per_field"] = [float(x) for x in l1]
    out["mixed"]["rel_l1_fields"] = ["rho", "p", "vx", "vy", "vz", "Bx", "By", "Bz"]
    out["mixed"]["rel_l1_face_B_vs_fp64"] = [float(x) for x in lb]
    return out


def mixed3d_report(n=256, steps=8, warmup=2):
    """The mixed FP32/FP64 3D hydro step against the FP64 one: the 3D blast
    n^3 (p_in 10, MC, HLLC, outflow), device time per CFL step (CUDA events on
    the grid's stream, L2 flushed), and the relative L1 per field of the two
    states after warmup + steps steps from the same initial state."""
    import torch

    import dragon_b200 as dg
    from dragon_b200 import problems

    w5, d = problems.blast_3d(n, ghosts=2, p_in=10.0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {"workload": f"3D blast {n}^3, p_in 10, MC, HLLC, outflow", "steps": steps + warmup}
    states = {}
    for name, prec in (("fp64", dg.PREC_FP64), ("mixed", dg.PREC_MIXED)):
        G = dg.Grid3D(n, n, n, d, d, d, ghosts=2,
                      config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MC, precision=prec))
        G.w[...] = w5
        G.advance_steps(warmup)
        stream = torch.cuda.ExternalStream(G._lib.dragon_gpu_stream(G._h))
        ev = []
        torch.cuda.synchronize()
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            G.advance_steps_async(1)
            b.record(stream)
            G.advance_wait()
            ev.append((a, b))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        out[name] = {"ms_per_step": ms, "value": n ** 3 / (ms / 1e3), "unit": "cell-updates/s"}
        states[name] = G.w[2:-2, 2:-2, 2:-2].reshape(-1, 5).copy()
        G.close()
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["mixed"]["rel_l1_vs_fp64_per_field"] = [float(x) for x in problems.rel_l1(states["mixed"], states["fp64"])]
    out["mhd"] = mixed3d_mhd_report(flush, steps=steps, warmup=warmup)
    return out


def mixed3d_mhd_report(flush, n=128, steps=8, warmup=2):
    """The mixed 3D MHD step against the FP64 one: the n^3 blast (p_in 10) in
    the uniform field (0.5, 0.3, 0.2), HLLD, MC, outflow; device time per CFL
    step and the relative L1 per field (cells and face B) after warmup + steps
    steps from the same initial state."""
    import torch

    import dragon_b200 as dg
    from dragon_b200 import workloads

    out = {"workload": f"3D MHD blast {n}^3, p_in 10, B (0.5, 0.3, 0.2), HLLD, MC, outflow"}
    states = {}
    for name, mixed in (("fp64", False), ("mixed", True)):
        G = workloads.blast3d(n, dg.RIEMANN_HLLD, True, mixed)
        G.advance_steps(warmup)
        stream = torch.cuda.ExternalStream(G._lib.dragon_gpu_stream(G._h))
        ev = []
        torch.cuda.synchronize()
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            G.advance_steps_async(1)
            b.record(stream)
            G.advance_wait()
            ev.append((a, b))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        out[name] = {"ms_per_step": ms, "value": n ** 3 / (ms / 1e3), "unit": "cell-updates/s"}
        g = G.ghosts
        states[name] = (G.w[g:-g, g:-g, g:-g].reshape(-1, 8).copy(), G.B[g:-g, g:-g, g:-g].reshape(-1, 3).copy())
        G.close()
    from dragon_b200 import problems
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["mixed"]["rel_l1_vs_fp64_per_field"] = [float(x) for x in problems.rel_l1(states["mixed"][0],
                                                                                 states["fp64"][0])]
    out["mixed"]["rel_l1_face_B_vs_fp64"] = [float(x) for x in problems.rel_l1(states["mixed"][1], states["fp64"][1])]
    return out


def stated_length_report(n=1024, kh_steps=2000, ot_time=0.5):
    """The mixed path against the FP64 path (bit-identical to the reference) at
    the stated lengths of the two 2D configurations: the shear layer for
    kh_steps steps and Orszag-Tang to t = ot_time, both n^2, each grid pair
    from the same initial state; relative L1 per field of the interiors, the
    step counts and the device-loop wall time of each path."""
    import torch

    import dragon_b200 as dg
    from dragon_b200 import problems

    out = {}
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=1234)
    st = {}
    for name, prec in (("fp64", dg.PREC_FP64), ("mixed", dg.PREC_MIXED)):
        G = dg.Grid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER,
                                                               precision=prec))
        G.w[...] = w0
        G.boundary = dg.Periodic()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = G.advance_steps(kh_steps)
        st[name] = (G.w.copy(), time.perf_counter() - t0, r.time_advanced)
        G.close()
    l1 = problems.rel_l1(st["mixed"][0][2:-2, 2:-2], st["fp64"][0][2:-2, 2:-2])
    out["shear_layer"] = {"grid": n, "steps": kh_steps, "t_fp64": st["fp64"][2], "t_mixed": st["mixed"][2],
                          "rel_l1_vs_fp64": dict(zip(["rho", "p", "vx", "vy", "vz"], (float(x) for x in l1))),
                          "wall_s_fp64": st["fp64"][1], "wall_s_mixed": st["mixed"][1]}
    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
    st = {}
    for name, prec in (("fp64", dg.PREC_FP64), ("mixed", dg.PREC_MIXED)):
        G = dg.Grid2D(n, n, dx, dy, ghosts=3, config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX, precision=prec))
        G.w[...] = w0
        G.B[...] = B0
        G.boundary = dg.Periodic()
        G.initialize_B_fields()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = G.advance(ot_time)
        Bf = G.B.copy()
        g = 3
        d = (Bf[g + 1:g + n + 1, g:g + n, 0] - Bf[g:g + n, g:g + n, 0]) + \
            (Bf[g:g + n, g + 1:g + n + 1, 1] - Bf[g:g + n, g:g + n, 1])
        st[name] = (G.w.copy(), Bf, time.perf_counter() - t0, r.steps, float(np.abs(d).max()))
        G.close()
    g = 3
    l1 = problems.rel_l1(st["mixed"][0][g:-g, g:-g], st["fp64"][0][g:-g, g:-g])
    lb = problems.rel_l1(st["mixed"][1][g:-g, g:-g, :2], st["fp64"][1][g:-g, g:-g, :2])
    out["orszag_tang"] = {"grid": n, "t": ot_time, "steps_fp64": st["fp64"][3], "steps_mixed": st["mixed"][3],
                          "rel_l1_vs_fp64": dict(zip(["rho", "p", "vx", "vy", "vz", "Bx", "By", "Bz"],
                                                     (float(x) for x in l1))),
                          "rel_l1_face_B_vs_fp64": [float(x) for x in lb],
                          "max_abs_divB_dx": {"fp64": st["fp64"][4], "mixed": st["mixed"][4]},
                          "wall_s_fp64": st["fp64"][2], "wall_s_mixed": st["mixed"][2]}
    return out


def custom_bc_report(n=1024, steps=20, warmup=3):
    """A user GhostFill element (an inflow jet on X-, the reference's Jet
    pattern) on the n^2 shear layer against the same grid with built-in
    elements only: wall time per CFL step of advance_steps. The jet runs as a
    host apply() (only the slabs along its face cross the host link) and as a
    device fill compiled with NVRTC (DeviceGhostFill: inside the device
    advance loop); both give the same states bit for bit."""
    import torch

    import dragon_b200 as dg
    from dragon_b200 import problems

    class Jet(dg.GhostFill):
        def __init__(self, dy, g):
            super().__init__("X-", True)
            self.dy, self.g = dy, g

        def apply(self, grid):
            w, g = grid.w, self.g
            ys = (np.arange(w.shape[1]) - g + 0.5) * self.dy
            jet = np.abs(ys - 0.5) < 0.1
            for gl in range(1, g + 1):
                w[g - gl] = w[g]
                w[g - gl, jet] = (2.0, 3.0, 1.5, 0.0, 0.0)

    jet_src = """
__device__ void jet(const dragon_fill_ctx& c, int i, int j, int k) {
    for (int f = 0; f < c.nf; f++) c.set(f, i, j, k, c.get(f, 0, j, k));
    if (fabs((j + 0.5) * c.d[1] - 0.5) < 0.1) {
        c.set(DRAGON_RHO, i, j, k, 2.0);
        c.set(DRAGON_P, i, j, k, 3.0);
        c.set(DRAGON_VX, i, j, k, 1.5);
        c.set(DRAGON_VY, i, j, k, 0.0);
        c.set(DRAGON_VZ, i, j, k, 0.0);
    }
}
"""
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=1234)
    out = {"workload": f"shear layer {n}^2, X- inflow jet (user element) + Outflow X+ + Periodic Y"}
    states = {}
    for name, bl in (("builtin", dg.Outflow("X") + dg.Periodic("Y")),
                     ("user_element", dg.Periodic("Y") + Jet(dy, 2)),
                     ("device_element", dg.Periodic("Y") + dg.DeviceGhostFill(jet_src, "jet", faces="X-"))):
        G = dg.Grid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
        G.w[...] = w0
        G.boundary = bl
        G.advance_steps(warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        G.advance_steps(steps)
        torch.cuda.synchronize()
        out[name + "_ms_per_step"] = (time.perf_counter() - t0) / steps * 1e3
        states[name] = G.w.copy()
        G.close()
    out["ratio"] = out["user_element_ms_per_step"] / out["builtin_ms_per_step"]
    out["device_ratio"] = out["device_element_ms_per_step"] / out["builtin_ms_per_step"]
    out["device_equals_host_element"] = bool(np.array_equal(states["device_element"], states["user_element"]))
    return out


def hoard_report(n=1024, reps=8, intervals=(50, 250), frames=6):
    """Output from device buffers (DRAGONHOARD's writeToFile) on the n^2 FP64
    shear layer with the reference's default options (primitive values + E as
    float, deflate level 4): the pack kernel's device time and bandwidth (L2
    flushed; algorithmic bytes = 5 FP64 fields read + the datasets written),
    the wall time of a complete file (pack, download, deflate on every host
    core, write) compressed and uncompressed, the same file built on the host
    from the downloaded padded state (the route without a device pack), and
    the wall time per step of runs that snapshot every k steps (k in
    `intervals`) asynchronously against the same run without snapshots: the
    stepping hides a file when k steps take longer than writing one."""
    import tempfile

    import torch

    import dragon_b200 as dg
    from dragon_b200 import hoard, problems

    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=1234)
    G = dg.Grid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.w[...] = w0
    G.boundary = dg.Periodic()
    G.advance_steps(3)
    tmp = tempfile.mkdtemp(prefix="hoard_")
    old_dir = hoard.output_dir
    hoard.output_dir = tmp
    out = {"workload": f"shear layer {n}^2 FP64, write option 3 (primitive + E as float), deflate 4",
           "host_threads": os.cpu_count()}
    try:
        G._to_device()
        stream = torch.cuda.ExternalStream(G._lib.dragon_gpu_stream(G._h))
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        raw = hoard.Options(compression_level=0)
        ev = []
        for r in range(reps + 2):
            hoard.wait(G)
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                # a fixed ~1 ms device delay, so the host has enqueued the pack
                # before the start event fires and the events time the kernel alone
                torch.cuda._sleep(2_000_000)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            hoard.write_to_file(G, 0.0, r, "pack", wait=False, opts=raw)
            b.record(stream)
            if r >= 2:
                ev.append((a, b))
        hoard.wait(G)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
        cells = n * n
        alg = cells * (5 * 8 + 5 * 8 + 4)
        peak, peak_kind = measured_peaks()
        out["pack"] = {"kernel": "k_hoard_pack", "ms": ms, "bytes_per_cell": 84, "achieved_gbs": alg / ms / 1e6,
                       "peak_gbs": peak, "peak_source": peak_kind, "frac": alg / ms / 1e6 / peak}
        for name, opts in (("deflate4", hoard.Options()), ("uncompressed", raw)):
            t0 = time.perf_counter()
            for r in range(3):
                hoard.write_to_file(G, 0.0, r, f"{name}_{r}", opts=opts)
            dt = (time.perf_counter() - t0) / 3
            size = os.path.getsize(os.path.join(tmp, f"{name}_0.h5"))
            out["file_" + name] = {"s_per_file": dt, "bytes": size, "mb_per_s_of_datasets": cells * 44 / dt / 1e6}
        # the host route: download the padded state, flatten and convert on the host, write
        t0 = time.perf_counter()
        for r in range(3):
            G._dev_dirty = True
            w = G.w[2:-2, 2:-2]
            ds = {"/fluid/rho": w[..., 0].T, "/fluid/v/x": w[..., 2].T, "/fluid/v/y": w[..., 3].T,
                  "/fluid/v/z": w[..., 4].T, "/fluid/p": w[..., 1].T,
                  "/fluid/E": (w[..., 1] / (5.0 / 3.0 - 1.0) + (w[..., 0] / 2.0) *
                               (w[..., 2] ** 2 + w[..., 3] ** 2 + w[..., 4] ** 2)).T.astype(np.float32)}
            hoard.write_h5(os.path.join(tmp, f"host_{r}.h5"), {"dim": 2}, ds, level=4)
        out["file_host_route"] = {"s_per_file": (time.perf_counter() - t0) / 3}
        # stepping with asynchronous snapshots
        out["stepping"] = []
        for every in intervals:
            G.advance_steps(every)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(frames):
                G.advance_steps(every)
            torch.cuda.synchronize()
            base = (time.perf_counter() - t0) / (frames * every) * 1e3
            t0 = time.perf_counter()
            for f in range(frames):
                G.advance_steps(every)
                hoard.write_to_file(G, 0.0, f, f"frame_{hoard.cycle_string(f)}", wait=False)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            hoard.wait(G)  # the last file: no steps left to hide it
            tail = time.perf_counter() - t1
            snap = (t1 - t0) / (frames * every) * 1e3
            out["stepping"].append({"every_steps": every, "frames": frames, "ms_per_step_no_output": base,
                                    "ms_per_step_with_async_output": snap, "overhead": snap / base - 1.0,
                                    "last_file_wait_s": tail})
    finally:
        hoard.output_dir = old_dir
        G.close()
        import shutil
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def _batch_run(precision, steps, one_by_one_steps):
    """One precision of the batched uneven-instance workload: the batch
    (autotuned, then timed over `steps` steps) and the same grids advanced one
    after another. Returns the report and the batch's grids (still open)."""
    import torch

    import dragon_b200 as dg
    from dragon_b200 import batch, problems

    one, two = problems.batch_instances()

    def make():
        grids = []
        for spec in one:
            G = dg.Grid1D(spec["n"], spec["dx"], ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLX,
                                                                              limiter=dg.LIMITER_MC,
                                                                              precision=precision))
            G.w[...] = spec["w"]
            grids.append(G)
        for spec in two:
            n = spec["n"]
            G = dg.Grid2D(n, n, spec["dx"], spec["dx"], ghosts=3,
                          config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX, precision=precision))
            G.w[...] = spec["w"]
            G.B[...] = spec["B"]
            G.boundary = dg.Periodic()
            G.initialize_B_fields()
            grids.append(G)
        return grids

    cells = sum(s["n"] for s in one) + sum(s["n"] ** 2 for s in two)
    grids = make()
    b = batch.Batch(grids)
    t0 = time.perf_counter()
    tune, _ = b.autotune(6)
    tune_s = time.perf_counter() - t0
    b.advance_steps(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = b.advance_steps(steps)
    wall = time.perf_counter() - t0
    ref = make()
    for G in ref:
        G.advance_steps(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for G in ref:
        G.advance_steps(one_by_one_steps)
    torch.cuda.synchronize()
    wall1 = time.perf_counter() - t0
    for G in ref:
        G.close()
    rate = cells * steps / wall
    rate1 = cells * one_by_one_steps / wall1
    report = {"instances": len(one) + len(two), "cells_per_step": cells, "steps": steps,
              "value": rate, "unit": "cell-updates/s", "device_value": cells * steps / (st["replay_ms"] / 1e3),
              "one_by_one_value": rate1, "one_by_one_steps": one_by_one_steps, "speedup_vs_one_by_one": rate / rate1,
              "work_items_per_step": st["work_items"], "graph_replays": st["graph_replays"],
              "retries": st["retries"], "spin_timeouts": st["spin_timeouts"],
              "tuning": {"tile_1d": tune.tile_1d, "ctas_per_sm": tune.ctas_per_sm, "order": tune.order,
                         "graph_steps": tune.graph_steps, "mhd_tiles": tune.mhd_tiles, "wave": tune.wave},
              "autotune_seconds": tune_s}
    return report, grids


def batch_report(steps=500, one_by_one_steps=50):
    """Batched uneven instances: 2048 1D hydro Riemann problems (N log-uniform
    in [64, 4096], seeded states) and 256 2D MHD blasts (64^2 / 128^2 / 256^2,
    HLLD + CT, periodic), each with its own CFL dt, advanced together by the
    persistent work-queue kernel (autotuned launch shape, CUDA-graph replays);
    against the same grids advanced one after another. The workload runs in
    mixed FP32/FP64 (the reported value) and in FP64; after the timed steps the
    mixed states are compared with the FP64 ones (relative L1 per field, summed
    over the members of each kind)."""
    import dragon_b200 as dg

    mixed, gm = _batch_run(dg.PREC_MIXED, steps, one_by_one_steps)
    fp64, gf = _batch_run(dg.PREC_FP64, steps, one_by_one_steps)
    names = {1: ["rho", "p", "vx", "vy", "vz"], 2: ["rho", "p", "vx", "vy", "vz", "Bx", "By", "Bz"]}
    num, den = {}, {}
    for G, R in zip(gm, gf):
        g = G.ghosts
        sl = tuple(slice(g, g + n) for n in G.n)
        a, r = G.w[sl].reshape(-1, G.w.shape[-1]), R.w[sl].reshape(-1, R.w.shape[-1])
        num[G.dim] = num.get(G.dim, 0) + np.abs(a - r).sum(axis=0)
        den[G.dim] = den.get(G.dim, 0) + np.abs(r).sum(axis=0)
    l1 = {("1d_hydro" if d == 1 else "2d_mhd"): {k: float(v) for k, v in zip(names[d], num[d] / np.where(den[d] > 0, den[d], 1))}
          for d in num}
    for G in gm + gf:
        G.close()
    out = {"workload": "2048 1D hydro Riemann problems (N log-uniform [64,4096]) + 256 2D MHD blasts "
                       "(64^2/128^2/256^2), HLLC / HLLD, MC, own CFL dt each, mixed FP32/FP64",
           **mixed, "l1_vs_fp64_after_steps": l1,
           "fp64": {k: fp64[k] for k in ("value", "device_value", "one_by_one_value", "speedup_vs_one_by_one",
                                         "retries", "tuning")}}
    out["mixed_vs_fp64"] = mixed["value"] / fp64["value"]
    return out


def dist_report(ws, dev, n=4096, steps=10, warmup=2):
    """Strong scaling of one sharded grid (multi-GPU runs only): an n^2 shear
    layer cut into ws x slabs (DistGrid2D over NCCL: per step the slabs' ghost
    fill, x-halo exchange, CFL all-reduce MIN, step and all-or-nothing
    commit), `steps` CFL steps timed with CUDA events on each slab's stream,
    max over ranks."""
    import torch
    import torch.distributed as dist

    import dragon_b200 as dg
    from dragon_b200 import problems
    from dragon_b200.dist import DistGrid2D

    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=1234)
    G = DistGrid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.boundary = dg.Periodic()
    G.scatter(w0)
    del w0
    G.advance_steps(warmup)
    slab = G.local.grid
    stream = torch.cuda.ExternalStream(slab._lib.dragon_gpu_stream(slab._h), device=dev)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    G.advance_steps(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = t.item()
    slab.close()
    return {"workload": f"shear layer {n}^2 in {ws} x slabs (DistGrid2D, NCCL), HLLC, van Leer, periodic",
            "steps": steps, "ms_per_step": ms / steps, "value": n * n * steps / (ms / 1e3), "unit": "cell-updates/s",
            "scaling": "strong"}


def summary_of(d):
    """The headline numbers of each detailed section, rounded (the bench line's
    last key, so a tail of the line keeps it)."""
    out = {}
    if "mixed" in d:
        m = d["mixed"]
        out["mixed"] = {"value": m["value"], "speedup_vs_fp64": m["speedup_vs_fp64"],
                        "kernel_ms": m["kernel_ms_avg"], "hbm_frac": m["roofline_hbm_frac"],
                        "max_rel_l1_vs_fp64": max(m["rel_l1_vs_fp64_per_field"]),
                        "steps_compared": m["steps_compared"]}
    if "stated_length" in d:
        k, o = d["stated_length"]["shear_layer"], d["stated_length"]["orszag_tang"]
        out["mixed_at_stated_length"] = {
            "shear_layer_1024_2000_steps": k["rel_l1_vs_fp64"],
            "orszag_tang_1024_t0.5": dict(o["rel_l1_vs_fp64"], steps=o["steps_fp64"],
                                          divB_dx=max(o["max_abs_divB_dx"].values()))}
    if "mhd" in d:
        m = d["mhd"]
        out["mhd_orszag_tang_1024"] = {"fp64_value": m["fp64"]["value"], "mixed_value": m["mixed"]["value"],
                                       "mixed_speedup": m["mixed"]["speedup_vs_fp64"]}
    if "mixed3d" in d:
        m = d["mixed3d"]
        out["mixed_3d_blast_256"] = {"fp64_value": m["fp64"]["value"], "mixed_value": m["mixed"]["value"],
                                     "mixed_speedup": m["mixed"]["speedup_vs_fp64"],
                                     "max_rel_l1_vs_fp64": max(m["mixed"]["rel_l1_vs_fp64_per_field"])}
        if "mhd" in m:
            h = m["mhd"]
            out["mixed_3d_mhd_blast_128"] = {"fp64_value": h["fp64"]["value"], "mixed_value": h["mixed"]["value"],
                                             "mixed_speedup": h["mixed"]["speedup_vs_fp64"],
                                             "max_rel_l1_vs_fp64": max(h["mixed"]["rel_l1_vs_fp64_per_field"] +
                                                                       h["mixed"]["rel_l1_face_B_vs_fp64"])}
    if "learned_guess" in d:
        g = d["learned_guess"]
        out["learned_guess"] = {k: g[k] for k in g if k.startswith(("iteration_reduction", "ceiling_reduction"))}
        out["learned_guess"]["train_samples"] = g["train"]["samples"]
        out["learned_guess"]["iters_per_solve"] = {k: g[k]["newton_iters_per_solve"] for k in g
                                                   if isinstance(g[k], dict) and "newton_iters_per_solve" in g[k]}
    if "custom_bc" in d:
        out["user_ghostfill_step_vs_builtin"] = {"host_apply": d["custom_bc"]["ratio"],
                                                 "device_fill": d["custom_bc"]["device_ratio"]}
    if "hoard" in d:
        h = d["hoard"]
        out["hoard_output_1024"] = {"pack_ms": h["pack"]["ms"], "pack_hbm_frac": h["pack"]["frac"],
                                    "file_s": h["file_deflate4"]["s_per_file"],
                                    "host_route_file_s": h["file_host_route"]["s_per_file"],
                                    "async_output_overhead": {f"every_{x['every_steps']}": x["overhead"]
                                                              for x in h["stepping"]}}
    if "dist" in d:
        out["distgrid_4096_strong"] = {"value": d["dist"]["value"], "ms_per_step": d["dist"]["ms_per_step"]}
    if "batch" in d:
        b = d["batch"]
        out["batch_c5"] = {"mixed_value": b["value"], "fp64_value": b["fp64"]["value"],
                           "vs_one_by_one": b["speedup_vs_one_by_one"], "mixed_vs_fp64": b["mixed_vs_fp64"]}
    return sig(out, 4)


def run_gpu(args):
    import torch
    import torch.distributed as dist

    import dragon_b200 as dg
    from dragon_b200 import _lib, problems

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    cfg = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER, cfl=dg.CFL_ADD,
                    precision=dg.PREC_MIXED if args.mixed else dg.PREC_FP64)
    w0, dx, dy = problems.kelvin_helmholtz_2d(N, ghosts=2, seed=1234 + rank)
    G = dg.Grid2D(N, N, dx, dy, ghosts=2, config=cfg)
    G.w[...] = w0
    G.boundary = dg.Periodic()
    L = G._lib
    h = G._h
    stream = torch.cuda.ExternalStream(L.dragon_gpu_stream(h), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    # warm-up (also uploads the state and compiles nothing: kernels are prebuilt)
    G.advance_steps(max(args.warmup, 1))
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            dist.barrier()

    # ---- value: K steps, state resident in HBM, L2 flushed before each step
    L.dragon_gpu_profile_enable(h, 1)
    L.dragon_gpu_profile_read(h, None, None, 1)
    launches0 = G.launch_count()
    step_ms = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            # enqueue the step, mark its end on the stream, then read its outcome
            st = _lib.AdvanceStats()
            _lib.check(L.dragon_gpu_advance_steps_async(h, 1))
            e1.record(stream)
            _lib.check(L.dragon_gpu_advance_wait(h, __import__("ctypes").byref(st)))
            step_ms.append((e0, e1))
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    barrier()
    ms = sum(a.elapsed_time(b) for a, b in step_ms)
    launches = G.launch_count() - launches0
    kms = __import__("ctypes").c_double()
    kn = __import__("ctypes").c_longlong()
    L.dragon_gpu_profile_read(h, __import__("ctypes").byref(kms), __import__("ctypes").byref(kn), 1)
    L.dragon_gpu_profile_enable(h, 0)
    if ws > 1:
        t = torch.tensor([ms, kms.value], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, kmax = t[0].item(), t[1].item()
    else:
        kmax = kms.value
    ms_per_step = ms / args.steps
    value = ws * N * N * args.steps / (ms / 1e3)
    fp64_state = G.w.copy()  # after warm-up + K steps, for the mixed path's L1

    # ---- mixed FP32/FP64 path: same input, same steps, same timing procedure
    mixed = None
    if not args.no_mixed:
        cfg_m = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER, cfl=dg.CFL_ADD, precision=dg.PREC_MIXED)
        Gm = dg.Grid2D(N, N, dx, dy, ghosts=2, config=cfg_m)
        Gm.w[...] = w0
        Gm.boundary = dg.Periodic()
        Lm, hm = Gm._lib, Gm._h
        stream_m = torch.cuda.ExternalStream(Lm.dragon_gpu_stream(hm), device=dev)
        Gm.advance_steps(max(args.warmup, 1))
        Lm.dragon_gpu_profile_enable(hm, 1)
        Lm.dragon_gpu_profile_read(hm, None, None, 1)
        ev = []
        barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            with torch.cuda.stream(stream_m):
                flush.fill_(1.0)
                a_ = torch.cuda.Event(enable_timing=True)
                b_ = torch.cuda.Event(enable_timing=True)
                a_.record(stream_m)
            _lib.check(Lm.dragon_gpu_advance_steps_async(hm, 1))
            b_.record(stream_m)
            _lib.check(Lm.dragon_gpu_advance_wait(hm, None))
            ev.append((a_, b_))
        torch.cuda.synchronize()
        barrier()
        ms_m = sum(a.elapsed_time(b) for a, b in ev)
        kms_m = __import__("ctypes").c_double()
        kn_m = __import__("ctypes").c_longlong()
        Lm.dragon_gpu_profile_read(hm, __import__("ctypes").byref(kms_m), __import__("ctypes").byref(kn_m), 1)
        if ws > 1:
            t = torch.tensor([ms_m], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_m = t.item()
        g = 2
        l1 = problems.rel_l1(Gm.w[g:-g, g:-g], fp64_state[g:-g, g:-g])
        km = kms_m.value / max(1, kn_m.value)
        mixed = {"value": ws * N * N * args.steps / (ms_m / 1e3), "unit": "cell-updates/s",
                 "ms_per_step": ms_m / args.steps, "speedup_vs_fp64": ms / ms_m,
                 "rel_l1_vs_fp64_per_field": [float(x) for x in l1],
                 "rel_l1_fields": ["rho", "p", "vx", "vy", "vz"],
                 "steps_compared": args.steps + max(args.warmup, 1),
                 "kernel": "k_step2d_hydro_mixed", "kernel_ms_avg": km,
                 "roofline_hbm_frac": (N * N * CELL_BYTES / (km / 1e3) / 1e9) / measured_peaks()[0] if km > 0 else None}
        Gm.close()

    # ---- e2e: through the C ABI from pinned host memory, every step
    e2e_steps = max(1, min(args.steps, 10))
    e2e_serial_ms = e2e_run(G, [G], dev, e2e_steps, barrier)
    e2e_grids = [G]
    for _ in range(max(1, args.e2e_inflight) - 1):
        Gx = dg.Grid2D(N, N, dx, dy, ghosts=2, config=cfg)
        Gx.w[...] = w0
        Gx.boundary = dg.Periodic()
        Gx.advance_steps(1)
        e2e_grids.append(Gx)
    e2e_ms = e2e_run(G, e2e_grids, dev, e2e_steps, barrier)
    for Gx in e2e_grids[1:]:
        Gx.close()
    if ws > 1:
        t = torch.tensor([e2e_ms, e2e_serial_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms, e2e_serial_ms = t[0].item(), t[1].item()
    e2e_value = ws * N * N * e2e_steps * len(e2e_grids) / (e2e_ms / 1e3)
    e2e_serial_value = ws * N * N * e2e_steps / (e2e_serial_ms / 1e3)
    bytes_step = G.w.nbytes
    link = copy_bound(dev, bytes_step, N * N)
    dist_sec = dist_report(ws, dev) if ws > 1 and not args.no_dist else None

    if rank == 0:
        peak, peak_kind = measured_peaks()
        k_avg_ms = kms.value / max(1, kn.value)
        achieved = N * N * CELL_BYTES / (k_avg_ms / 1e3) / 1e9 if k_avg_ms > 0 else None
        traffic = traffic_from_profile()
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not args.mixed else "f32/f64",
            "data": "synthetic (seeded KH shear layer, numpy PCG64 seed 1234 + rank)",
            "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
            "config": dict(config_line(), precision="mixed" if args.mixed else "fp64"),
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": bytes_step,
                    "d2h_bytes_per_step": bytes_step, "steps": e2e_steps * len(e2e_grids),
                    "grids_in_flight": len(e2e_grids), "one_grid_value": e2e_serial_value,
                    "copy_bound": link, "frac_of_copy_bound": e2e_value / ws / link["value"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "kernel": "k_step2d_hydro", "kernel_ms_avg": k_avg_ms,
                         "bytes_per_cell": CELL_BYTES, "peak_source": peak_kind},
            "roofline_fp64": roofline_fp64(k_avg_ms, dev),
            "gpu_launches": launches,
            "clocks": clocks,
            "wall_s_timed": t_wall,
        }
        detail = {}
        if mixed is not None:
            detail["mixed"] = mixed
        if not args.no_learned:
            detail["learned_guess"] = learned_guess_report()
        if not args.no_batch:
            detail["batch"] = batch_report()
        if not args.no_mhd:
            detail["mhd"] = mhd_report()
        if not args.no_mixed3d:
            detail["mixed3d"] = mixed3d_report()
        if not args.no_stated_length:
            detail["stated_length"] = stated_length_report()
        if not args.no_custom_bc:
            detail["custom_bc"] = custom_bc_report()
        if not args.no_hoard:
            detail["hoard"] = hoard_report()
        if not args.no_cpu_baseline:
            cb, why = reference_baseline(1000, 0, budget_s=args.cpu_budget)
            line["cpu_baseline"] = cb if cb else {"unavailable": why}
        line["e2e"].pop("copy_bound", None)
        line["e2e"]["copy_bound_value"] = link["value"]
        detail["e2e_copy_bound"] = link
        if dist_sec is not None:
            detail["dist"] = dist_sec
        line["summary"] = summary_of(detail)
        print("detail: " + json.dumps(detail), file=sys.stderr, flush=True)
        print(json.dumps(sig(line, 6)), flush=True)
    G.close()
    if ws > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dragon_b200", choices=["dragon_b200", "reference"])
    ap.add_argument("--mixed", action="store_true", help="mixed FP32/FP64 path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned star-pressure guess report")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched uneven-instance report")
    ap.add_argument("--no-mhd", action="store_true", help="skip the 2D MHD (Orszag-Tang) report")
    ap.add_argument("--no-mixed3d", action="store_true", help="skip the mixed 3D hydro (256^3 blast) report")
    ap.add_argument("--no-hoard", action="store_true", help="skip the output-from-device-buffers report")
    ap.add_argument("--no-custom-bc", action="store_true", help="skip the user-GhostFill step cost")
    ap.add_argument("--no-dist", action="store_true", help="multi-GPU runs: skip the sharded 4096^2 grid")
    ap.add_argument("--no-stated-length", action="store_true",
                    help="skip the mixed-vs-FP64 comparison at the configurations' stated lengths")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--e2e-inflight", type=int, default=E2E_INFLIGHT,
                    help="grids whose end-to-end steps overlap on separate streams")
    ap.add_argument("--grid", type=int, default=1024, help="cells per axis (default: the 1024^2 workload)")
    args = ap.parse_args()
    global N, WORKLOAD
    if args.grid != N:
        N = args.grid
        WORKLOAD = WORKLOAD.replace("1024sq", f"{N}sq")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
