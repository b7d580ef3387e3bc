#!/usr/bin/env python
"""SRM throughput benchmark (point*harmonics per second) on B200.

Workload (default): structured 512 x 512 x 512 grid at 25 m, von Karman ACF
(Hurst 0.5, correlation lengths 3000/3000/1000 m, sigma 0.05), 20 000
harmonics, seed 1234 -- the precision configuration the tensor-core form is
specified on. Synthetic by construction (the SRM draws its own harmonics).

One step = one pass of the SRM sum over the whole grid: FP64 per-axis phase
tables from the harmonic table, then the factorised tcgen05 split-BF16 sum
(scaled field written to HBM). `value` times K such steps with the harmonic
table already on the device; `e2e` times K calls of the public C ABI
(scarf_execute) with a pinned host output buffer: host sampler, H2D of the
harmonic table, device sum, statistics, D2H of the field (`e2e.pageable`: the
same into a malloc'd field). `accuracy` compares every point of the field
with the FP64 sum over the same harmonics; `direct_sum` times the FP32 direct
sum over the whole table on the same grid.

The other configurations are measured on their own (`configs`, single GPU):
128^3 x 5 000 (plain direct sum, and the tensor-core form beside it),
2e6 unstructured points x 10 000 (direct sum), 2048 x 2048 x 512 x 50 000
(tensor-core form), each with kernel time, roofline, end to end through
scarf_execute, full-field error against FP64 and, for the first two, the CPU
restatement over the whole workload; `batched` is the 256-field
configuration.

--impl reference times the CPU restatement of the reference's SRM (the
reference itself cannot be built here: no Fortran compiler, MPI or TRNG4)
on all host threads over a bounded slab of the same workload.

Multi-GPU (torchrun, N ranks): each rank computes its own 512^3 z-slab of a
512 x 512 x 512N global grid with the same seed (weak scaling, no data-path
collective); the only exchange is the Chan merge of (n, mean, var) in e2e.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SRM point·harmonics/s, TC split-precision vs FP32 direct sum, ≤1e-5 rel-RMS"
UNIT = "pt*harm/s"
WORKLOAD = dict(nx=512, ny=512, nz=512, ds=25.0, acf=0, hurst=0.5, cl=[3000.0, 3000.0, 1000.0], sigma=0.05,
                nharm=20000, seed=1234)
FLOP_PER_PTHARM = 12  # 2 real MACs per harmonic and point (complex as real K=2) x 3 split products
DIRECT_HARM = 2000    # harmonics of the direct sum's warm-up launch (the timed launch sums the whole table)


def workload_name(w) -> str:
    return (f"srm_structured_{w['nx']}x{w['ny']}x{w['nz']}_ds{w['ds']:g}m_vk_h{w['hurst']:g}"
            f"_cl{'/'.join(f'{c:g}' for c in w['cl'])}_nharm{w['nharm']}")


def load_peaks():
    """(burst, sustained) dense bf16 TFLOP/s and their source."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        burst = d.get("bf16_tflops")
        return burst, d.get("bf16_tflops_sustained", burst), "measured"
    return 1590.0, 1400.0, "fallback"


def pick_peak(clocks: dict):
    """The burst peak: every kernel here is timed in isolation (back-to-back
    launches of the kernel alone), which is what the burst cuBLAS figure
    measures. The sustained, power-capped figure is reported beside it."""
    burst, sustained, src = load_peaks()
    sm, mx = clocks.get("sm_mhz"), clocks.get("sm_max_mhz")
    note = "" if sm is None or not mx else f" (the timed launches ran at a median {sm:.0f} of {mx:.0f} MHz)"
    return burst, sustained, f"{src} bf16 dense, burst{note}"


def profile_traffic():
    """DRAM bytes per launch of the tensor-core kernel from the committed ncu
    summary (None until a capture exists)."""
    p = ROOT / "profiles" / "srm_tc_kernel_traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_full_launch:"):
            return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    """nvidia-smi clocks, power and throttle reasons sampled every 50 ms; only
    samples that arrive between mark_start() and mark_end() (the timed region)
    are summarised."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.stamped = []
        self.t0 = self.t1 = None

    def _read(self):
        for line in self.proc.stdout:
            if line.strip():
                self.stamped.append((time.perf_counter(), line))

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            time.sleep(0.2)  # the first sample precedes the region
        except Exception:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.06)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.reader.join(timeout=5)
        t0 = self.t0 if self.t0 is not None else -float("inf")
        t1 = self.t1 if self.t1 is not None else float("inf")
        # A line stamped up to 60 ms after the region still describes it.
        self.lines = [l for t, l in self.stamped if t0 <= t <= t1 + 0.06]

    def summary(self):
        sm, pw, mx, reasons = [], [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                pw.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "power_w": float(np.median(pw)) if pw else None}


# ---------------------------------------------------------------------------
def run_reference(args, w):
    """CPU restatement of the reference SRM on all host threads (bounded slab)."""
    import oracle
    nth = os.cpu_count() or 1
    kw = dict(acf=w["acf"], nharm=w["nharm"], seed=w["seed"], hurst=w["hurst"], sigma=w["sigma"], ds=w["ds"],
              cl=w["cl"])
    fe = [w["nx"], w["ny"], w["nz"]]
    op = oracle.structured_params(fs=[1, 1, 1], fe=fe, **kw)
    so = oracle.setup(op)
    tab, _ = oracle.sample(op, so)
    nh = len(tab)
    # Calibrate on one x-row, then size a slab of rows for ~3 s per step.
    t0 = time.perf_counter()
    oracle.sum_structured_mt(so, [1, 1, 1], [w["nx"], 1, 1], w["ds"], tab, nth)
    rate = w["nx"] * nh / max(time.perf_counter() - t0, 1e-6)
    rows = int(max(1, min(w["ny"] * w["nz"], 3.0 * rate / (w["nx"] * nh))))
    n = [w["nx"], min(rows, w["ny"]), max(1, rows // w["ny"]) if rows > w["ny"] else 1]
    work = n[0] * n[1] * n[2] * nh
    for _ in range(args.warmup):
        oracle.sum_structured_mt(so, [1, 1, 1], n, w["ds"], tab, nth)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.sum_structured_mt(so, [1, 1, 1], n, w["ds"], tab, nth)
    dt = time.perf_counter() - t0
    value = work * args.steps / dt
    sample = f"{n[0]}x{n[1]}x{n[2]} points of the workload x {nh} harmonics per step (FP32 restatement, {nth} threads)"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (SRM draws its harmonics)",
            "impl": "reference",
            "config": {"workload": workload_name(w), "grid": fe, "nharm": w["nharm"], "form": "cpu_fp32_restatement",
                       "l2": "n/a (host)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference not buildable here (no gfortran/MPI/TRNG4); its SRM restated in C, op-order FP32"}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(w):
    """Rank-0 CPU baseline: FP32 restatement on all host threads, one bounded
    slab of the workload (~10-20 s of CPU work)."""
    import oracle
    nth = os.cpu_count() or 1
    kw = dict(acf=w["acf"], nharm=w["nharm"], seed=w["seed"], hurst=w["hurst"], sigma=w["sigma"], ds=w["ds"],
              cl=w["cl"])
    op = oracle.structured_params(fs=[1, 1, 1], fe=[w["nx"], w["ny"], w["nz"]], **kw)
    so = oracle.setup(op)
    tab, _ = oracle.sample(op, so)
    nh = len(tab)
    t0 = time.perf_counter()
    oracle.sum_structured_mt(so, [1, 1, 1], [w["nx"], 1, 1], w["ds"], tab, nth)
    rate = w["nx"] * nh / max(time.perf_counter() - t0, 1e-6)
    rows = int(max(1, min(w["ny"], 12.0 * rate / (w["nx"] * nh))))
    t0 = time.perf_counter()
    oracle.sum_structured_mt(so, [1, 1, 1], [w["nx"], rows, 1], w["ds"], tab, nth)
    dt = time.perf_counter() - t0
    return {"value": w["nx"] * rows * nh / dt, "unit": UNIT, "cores": nth, "kind": "port",
            "sample": f"{w['nx']}x{rows}x1 points x {nh} harmonics (FP32 restatement of the reference SRM, "
                      f"{nth} threads, {dt:.1f} s)"}


# ---------------------------------------------------------------------------
def run_batched(args, nfields=256):
    """The many-realisation workload: `nfields` fields of uneven sizes and
    spectra in one persistent launch (device work queue), captured once in a
    CUDA graph and replayed. Tables are drawn by the device-assisted sampler."""
    import torch

    import oracle
    import scarf3d_b200 as sb
    from scarf3d_b200.workloads import batched_fields, work_pt_harm

    spec = batched_fields(count=nfields)
    stream = torch.cuda.current_stream()
    params = [f["params"] for f in spec]
    setups = [f["setup"] for f in spec]
    # All tables in one page-locked host buffer (the sampler writes them in
    # place) and one device buffer, so that a step uploads them in one copy.
    # Each field's region is padded to 20 floats (80 B) so every table starts 16-byte aligned.
    offs = np.concatenate([[0], np.cumsum([-(-5 * max(p.nharm, 1) // 20) * 20 for p in params])]).astype(np.int64)
    h_tabs = torch.empty(int(offs[-1]), dtype=torch.float32, pin_memory=True)
    d_tabs = torch.empty(int(offs[-1]), dtype=torch.float32, device="cuda")
    views = [h_tabs[int(offs[i]):int(offs[i + 1])].numpy() for i in range(nfields)]
    t0 = time.perf_counter()
    tabs = sb.sample_device_batch(params, setups, stream.cuda_stream, out=views)[0]
    t_sample = time.perf_counter() - t0
    d_tabs.copy_(h_tabs, non_blocking=True)
    work = float(sum(int(np.prod(f["n"])) * len(t) for f, t in zip(spec, tabs)))
    outs = [torch.empty(int(np.prod(f["n"])), dtype=torch.float32, device="cuda") for f in spec]
    entries = [dict(setup=f["setup"], fs=[1, 1, 1], n=f["n"], ds=f["ds"], d_table=d_tabs.data_ptr() + 4 * int(o),
                    nh=len(t), d_field=out.data_ptr()) for f, t, o, out in zip(spec, tabs, offs[:-1], outs)]
    tuned = None
    if not args.no_autotune:
        tuned = sb.tc_batch_autotune(entries, stream.cuda_stream)
        sb.set_tc_variant(tuned["variant"])
        for e in entries:
            e["tile_j"] = tuned["tile_j"]
    batch = sb.TcBatch(entries, lambda nb: torch.empty(nb, dtype=torch.uint8, device="cuda"))
    batch.launch(stream.cuda_stream)
    batch.wait(stream.cuda_stream)
    cap = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=cap):
        batch.launch(torch.cuda.current_stream().cuda_stream)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        graph.replay()
    ev1.record()
    torch.cuda.synchronize()
    batch.wait(stream.cuda_stream)
    t_step = ev0.elapsed_time(ev1) / 1e3 / args.steps
    # Every point of every field against the FP64 sum over its own harmonics.
    from oracle import gpu_fp64
    errs, maxabs = [], []
    for f, o, t in zip(spec, outs, tabs):
        p_ = f["params"]
        op = oracle.params(acf=p_.acf, nharm=p_.nharm, seed=p_.seed, hurst=p_.hurst, sigma=p_.sigma, ds=p_.ds,
                           cl=list(p_.cl), nc=list(p_.nc), fc=list(p_.fc))
        r = gpu_fp64.compare_structured(o, oracle.setup(op), [1, 1, 1], f["n"], f["ds"], t)
        errs.append(r["rel_rms"])
        maxabs.append(r["max_abs"] / r["std_ref"])
    # End to end through the public API: device-assisted sampling, H2D of the
    # tables, the batched launch and D2H of every field into pinned memory.
    # The fields go to page-locked host buffers field by field as the launch
    # completes them (scarf_srm_tc_batch_set_host_outputs), inside wait().
    hosts = [torch.empty(o.numel(), dtype=torch.float32, pin_memory=True) for o in outs]
    batch.set_host_outputs([h.data_ptr() for h in hosts])
    torch.cuda.synchronize()
    # One step at a time: sample, upload, launch, copy out (median of 3).
    lat = []
    for _ in range(3):
        t0 = time.perf_counter()
        tabs2 = sb.sample_device_batch(params, setups, stream.cuda_stream, out=views)[0]
        d_tabs.copy_(h_tabs, non_blocking=True)
        graph.replay()
        batch.wait(stream.cuda_stream)
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t0)
    t_e2e = float(np.median(lat))
    e2e_ok = all(torch.equal(h, o.cpu()) for h, o in zip(hosts, outs))
    del graph
    sb.set_tc_variant(sb.TC_SINGLE)
    return {"fields": nfields, "work_pt_harm": work, "value": work / t_step, "unit": UNIT,
            "plan": None if tuned is None else {"variant": ["pair", "single", "single_tmem_a"][tuned["variant"]],
                                                "tile_j": tuned["tile_j"], "autotuned": True},
            "ms_per_step": t_step * 1e3, "graph_replayed": True, "sampling_s_device_assisted": t_sample,
            "accuracy_vs_fp64_full_field": {"fields": len(errs), "rel_rms_max": float(np.max(errs)),
                                            "rel_rms_median": float(np.median(errs)),
                                            "max_abs_over_std_max": float(np.max(maxabs)),
                                            "fields_over_1e-5": int(np.sum(np.asarray(errs) > 1e-5))},
            "e2e": {"value": work / t_e2e, "unit": UNIT, "s_per_step": t_e2e, "steps": len(lat),
                    "host_copy_matches_device": e2e_ok,
                    "tables_kept_equal": all(len(a) == len(b) for a, b in zip(tabs, tabs2)),
                    "h2d_bytes_per_step": int(h_tabs.numel() * 4),
                    "d2h_bytes_per_step": int(sum(o.numel() * 4 for o in outs))},
            "workload": f"{nfields} fields, axes log-uniform 32..256 (x16), VK/Gaussian alternating, cl U[500,5000] m, "
                        "nharm U[2000,20000], ds 50 m, meta-seed 20240"}


# ---------------------------------------------------------------------------
# The other configurations of the path, each measured on its own: kernel time
# (CUDA events around the summation kernel alone, on its launch stream), the
# roofline of that kernel, end to end through the public C ABI with host
# buffers (sampling, H2D, sum, statistics, D2H inside the timed region), the
# error of every point against the FP64 sum over the identical harmonics, and
# where it is affordable the CPU restatement over the whole workload.
CONFIG1 = dict(name="plain_structured_128cubed_ds50m_vk_h0.25_cl2000_nharm5000", n=[128, 128, 128], ds=50.0, acf=0,
               hurst=0.25, cl=[2000.0, 2000.0, 2000.0], sigma=0.05, nharm=5000, seed=1234)
CONFIG2 = dict(name="plain_unstructured_2e6pts_20x20x10km_gs_cl1500/1500/500_nharm10000", npts=2_000_000,
               box=[20000.0, 20000.0, 10000.0], pts_seed=7, dh=100.0, acf=1, hurst=0.0, cl=[1500.0, 1500.0, 500.0],
               sigma=0.1, nharm=10000, seed=7)
CONFIG5 = dict(name="large_structured_2048x2048x512_ds10m_vk_h0.3_cl5000/5000/2000_nharm50000", n=[2048, 2048, 512],
               ds=10.0, acf=0, hurst=0.3, cl=[5000.0, 5000.0, 2000.0], sigma=0.08, nharm=50000, seed=1234)
DIRECT_WARP_INSTR_PER_PTHARM = 0.513  # ncu: sm__inst_executed per point*harmonic of srm_direct_kernel (fast sincos)
DIRECT_MUFU_PER_PTHARM = 2            # __sinf and __cosf of the reduced phase
FP32_FLOP_PER_PTHARM = 9             # phase 3 mul + 2 add, accumulate 2 mul + 2 add (plus the sin/cos)


def _i3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def _direct_roofline(value, sm_max_mhz):
    """Roofline of the FP32 direct sum: its two SFU (XU pipe) operations per
    point*harmonic against 148 SMs x 16 per clock, with the issue rate (warp
    instructions per point*harmonic from ncu against 148 SMs x 4 schedulers)
    beside it; both at the SM clock."""
    clk = (sm_max_mhz or 1965.0) * 1e6
    achieved = value * DIRECT_MUFU_PER_PTHARM / 1e12
    peak = 148 * 16 * clk / 1e12
    issue = value * DIRECT_WARP_INSTR_PER_PTHARM / 1e12
    issue_peak = 148 * 4 * clk / 1e12
    fp32 = value * FP32_FLOP_PER_PTHARM / 1e12
    fp32_peak = 148 * 128 * 2 * clk / 1e12
    return {"bound": "sfu", "achieved": achieved, "peak": peak, "unit": "T MUFU-op/s", "frac": achieved / peak,
            "issue": {"achieved": issue, "peak": issue_peak, "unit": "T warp-instr/s", "frac": issue / issue_peak,
                      "instr_per_ptharm": DIRECT_WARP_INSTR_PER_PTHARM},
            "fp32_tflops": fp32, "fp32_peak_tflops": fp32_peak, "fp32_frac": fp32 / fp32_peak,
            "kernel": "srm_direct_kernel", "traffic": None}


def _tc_roofline(value, peaks):
    burst, sustained, src = peaks
    achieved = value * FLOP_PER_PTHARM / 1e12
    return {"bound": "tensor", "achieved": achieved, "peak": burst, "unit": "TFLOP/s", "frac": achieved / burst,
            "frac_of_sustained": achieved / sustained, "peak_kind": f"{src} bf16 dense, burst",
            "kernel": "srm_tc_kernel", "traffic": None}


def _kernel_times(launch, steps, warm=1):
    import scarf3d_b200 as sb
    ms = []
    for it in range(warm + steps):
        launch()
        if it >= warm:
            ms.append(float(sb.lib.scarf_last_kernel_ms()))
    return ms


def _structured_leg(cfg, forms, steps, e2e_steps, peaks, clocks, cpu_full=False, e2e_form=None):
    """One structured configuration: kernel timing per form, full-field error
    against FP64, end to end through scarf_execute with a host field."""
    import torch

    import oracle
    import scarf3d_b200 as sb
    from oracle import gpu_fp64

    n, ds = cfg["n"], cfg["ds"]
    npts = int(np.prod(n))
    fs, fe = [1, 1, 1], list(n)
    ds32 = np.float32(ds)
    nc = [0.0, 0.0, 0.0]
    fc = [float(np.float32(n[c] - 1) * ds32) for c in range(3)]
    kw = dict(acf=cfg["acf"], nharm=cfg["nharm"], seed=cfg["seed"], hurst=cfg["hurst"], sigma=cfg["sigma"], ds=ds,
              cl=cfg["cl"])
    p = sb.make_params(nc=nc, fc=fc, **kw)
    s = sb.compute_setup(p)
    t0 = time.perf_counter()
    tab, _ = sb.sample(p, s)
    t_sample = time.perf_counter() - t0
    nh = len(tab)
    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    field = torch.empty(npts, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    so = oracle.setup(oracle.params(nc=nc, fc=fc, **kw))
    out = {"workload": cfg["name"], "grid": list(n), "nharm": cfg["nharm"], "harmonics_kept": nh,
           "work_pt_harm": float(npts) * nh, "host_sampling_ms": t_sample * 1e3}
    for form in forms:
        if form == "tc":
            wb = sb.tc_workspace_bytes(3, n, nh)
            work = torch.empty(wb, dtype=torch.uint8, device="cuda")

            def launch():
                sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), _i3(fs), _i3(n), ds,
                                                        ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                        ctypes.c_void_p(field.data_ptr()),
                                                        ctypes.c_void_p(work.data_ptr()), wb, sptr))
        else:
            work = None

            def launch():
                sb.check(sb.lib.scarf_srm_direct_structured(ctypes.byref(s), _i3(fs), _i3(n), ds,
                                                            ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                            ctypes.c_void_p(field.data_ptr()), sptr))
        ms = _kernel_times(launch, steps)
        torch.cuda.synchronize()
        value = float(npts) * nh / (np.mean(ms) / 1e3)
        acc = gpu_fp64.compare_structured(field, so, fs, n, ds, tab)
        roof = _tc_roofline(value, peaks) if form == "tc" else _direct_roofline(value, clocks.get("sm_max_mhz"))
        out[form] = {"value": value, "unit": UNIT, "kernel_ms": float(np.mean(ms)), "launches_timed": len(ms),
                     "roofline": roof,
                     "accuracy_vs_fp64_full_field": {k: acc[k] for k in ("rel_rms", "max_abs", "std_ref", "points")}}
        if form == "tc":
            out[form]["plan"] = sb.tc_plan_info(3, n, nh)
        del work
    del field
    torch.cuda.empty_cache()
    # End to end: scarf_execute into a page-locked host field, with the
    # named form and (when timed above) the tensor-core form as well.
    host = torch.empty(npts, dtype=torch.float32, pin_memory=True)

    def e2e(form):
        sb.set_nharm(cfg["nharm"])
        sb.set_form(sb.FORM_TC if form == "tc" else sb.FORM_DIRECT)
        sb.set_stream(stream.cuda_stream)
        sb.scarf_initialize(fs=fs, fe=fe, ds=ds, acf=cfg["acf"], cl=cfg["cl"], sigma=cfg["sigma"], method=1,
                            hurst=cfg["hurst"], nc=np.asarray(nc, np.float32), fc=np.asarray(fc, np.float32))
        stats = np.zeros(8, np.float32)
        fptr = ctypes.c_void_p(host.data_ptr())
        sp = stats.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        try:
            sb.check(sb.lib.scarf_execute_ex(cfg["seed"], fptr, sp, 0))
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                sb.check(sb.lib.scarf_execute_ex(cfg["seed"], fptr, sp, 0))
            t_e2e = (time.perf_counter() - t0) / e2e_steps
        finally:
            sb.scarf_finalize()
            sb.set_form(sb.FORM_AUTO)
            sb.set_nharm(10000)
        return {"value": float(npts) * nh / t_e2e, "unit": UNIT, "form": form, "ms_per_step": t_e2e * 1e3,
                "steps": e2e_steps, "host_memory": "page-locked", "h2d_bytes_per_step": int(nh * 20),
                "d2h_bytes_per_step": int(npts * 4 + 8), "stats_std_mean": [float(stats[2]), float(stats[3])]}

    ef = e2e_form or forms[0]
    out["e2e"] = e2e(ef)
    if ef != "tc" and "tc" in forms:
        out["e2e_tc"] = e2e("tc")
    del host
    if cpu_full:
        nth = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.sum_structured_mt(so, fs, n, ds, tab, nth)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": float(npts) * nh / dt, "unit": UNIT, "cores": nth, "kind": "port",
                               "sample": f"the whole workload, {dt:.1f} s (FP32 restatement, {nth} threads)"}
    return out


def _points_leg(cfg, steps, e2e_steps, clocks, cpu_full=True):
    """The unstructured configuration: FP32 direct sum over a point set."""
    import torch

    import oracle
    import scarf3d_b200 as sb
    from oracle import gpu_fp64

    rng = np.random.default_rng(cfg["pts_seed"])
    pts = (rng.random((3, cfg["npts"])) * np.asarray(cfg["box"])[:, None]).astype(np.float32)
    x, y, z = (np.ascontiguousarray(a) for a in pts)
    npts = len(x)
    nc = [float(a.min()) for a in (x, y, z)]
    fc = [float(a.max()) for a in (x, y, z)]
    kw = dict(acf=cfg["acf"], nharm=cfg["nharm"], seed=cfg["seed"], hurst=cfg["hurst"], sigma=cfg["sigma"],
              ds=cfg["dh"], cl=cfg["cl"])
    p = sb.make_params(nc=nc, fc=fc, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    nh = len(tab)
    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    dx, dy, dz = (torch.from_numpy(a).cuda() for a in (x, y, z))
    field = torch.empty(npts, dtype=torch.float32, device="cuda")
    sptr = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def launch():
        sb.check(sb.lib.scarf_srm_direct_points(ctypes.byref(s), ctypes.c_void_p(dx.data_ptr()),
                                                ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(dz.data_ptr()),
                                                npts, ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                ctypes.c_void_p(field.data_ptr()), sptr))
    ms = _kernel_times(launch, steps)
    torch.cuda.synchronize()
    value = float(npts) * nh / (np.mean(ms) / 1e3)
    so = oracle.setup(oracle.params(nc=nc, fc=fc, **kw))
    acc = gpu_fp64.compare_points(field, so, dx, dy, dz, tab)
    out = {"workload": cfg["name"], "points": npts, "nharm": cfg["nharm"], "harmonics_kept": nh, "dh": cfg["dh"],
           "work_pt_harm": float(npts) * nh,
           "direct": {"value": value, "unit": UNIT, "kernel_ms": float(np.mean(ms)), "launches_timed": len(ms),
                      "roofline": _direct_roofline(value, clocks.get("sm_max_mhz")),
                      "accuracy_vs_fp64_full_field": {k: acc[k] for k in ("rel_rms", "max_abs", "std_ref",
                                                                          "points")}}}
    # End to end: scarf_nocart_initialize + scarf_execute into a page-locked host field.
    host = torch.empty(npts, dtype=torch.float32, pin_memory=True)
    sb.set_nharm(cfg["nharm"])
    sb.set_stream(torch.cuda.current_stream().cuda_stream)
    sb.scarf_initialize(x=x, y=y, z=z, dh=cfg["dh"], acf=cfg["acf"], cl=cfg["cl"], sigma=cfg["sigma"], method=1)
    stats = np.zeros(8, np.float32)
    fptr = ctypes.c_void_p(host.data_ptr())
    sp = stats.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    try:
        sb.check(sb.lib.scarf_execute_ex(cfg["seed"], fptr, sp, 0))
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            sb.check(sb.lib.scarf_execute_ex(cfg["seed"], fptr, sp, 0))
        t_e2e = (time.perf_counter() - t0) / e2e_steps
    finally:
        sb.scarf_finalize()
        sb.set_nharm(10000)
    out["e2e"] = {"value": float(npts) * nh / t_e2e, "unit": UNIT, "form": "direct", "ms_per_step": t_e2e * 1e3,
                  "steps": e2e_steps, "host_memory": "page-locked", "h2d_bytes_per_step": int(nh * 20 + 12 * npts),
                  "d2h_bytes_per_step": int(npts * 4 + 8), "stats_std_mean": [float(stats[2]), float(stats[3])]}
    if cpu_full:
        nth = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.sum_points_mt(so, x, y, z, tab, nth)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": float(npts) * nh / dt, "unit": UNIT, "cores": nth, "kind": "port",
                               "sample": f"the whole workload, {dt:.1f} s (FP32 restatement, {nth} threads)"}
    return out


def run_fim(args, clocks):
    """The reference's other method (FIM, method 0) on the precision
    configuration's grid: 512^3 at 25 m, von Karman H=0.5, cl 3000/3000/1000 m,
    no padding (internal grid 514^3). Timed through scarf_execute into a
    device field (stats[4..7]: spectrum, symmetry, transform with statistics,
    mapping) and into a page-locked host field; every point checked against
    the CPU restatement at sampled points of the internal grid is left to the
    tests (the full oracle needs the whole spectrum on the host)."""
    import torch

    import scarf3d_b200 as sb

    n = [512, 512, 512]
    npts = int(np.prod(n))
    sb.set_stream(torch.cuda.current_stream().cuda_stream)
    sb.scarf_initialize(fs=[1, 1, 1], fe=n, ds=25.0, acf=0, cl=[3000.0, 3000.0, 1000.0], sigma=0.05, method=0,
                        hurst=0.5)
    try:
        dev = torch.empty(npts, dtype=torch.float32, device="cuda")
        for _ in range(2):
            sb.scarf_execute(1234, dev)
        parts, t_dev = [], []
        for _ in range(max(3, min(args.steps, 10))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, st = sb.scarf_execute(1234, dev)
            t_dev.append(time.perf_counter() - t0)
            parts.append([float(v) for v in st[4:8]])
        host = torch.empty(npts, dtype=torch.float32, pin_memory=True)
        sb.scarf_execute(1234, host.numpy())
        t_host = []
        for _ in range(3):
            t0 = time.perf_counter()
            sb.scarf_execute(1234, host.numpy())
            t_host.append(time.perf_counter() - t0)
        same = bool(torch.equal(host, dev.cpu()))
    finally:
        sb.scarf_finalize()
    ph = np.mean(np.asarray(parts), axis=0)
    # internal grid 514^3: spectrum writes n3 n2 (n1/2+1) complex (8 B), the
    # transform reads/writes them and writes the real grid (4 B per point)
    internal = 514 ** 3
    spec_bytes = 514 * 514 * 258 * 8
    return {"workload": "fim_structured_512x512x512_ds25m_vk_h0.5_cl3000/3000/1000_nopad", "points": npts,
            "internal_grid": [514, 514, 514], "unit": "points/s",
            "device": {"value": npts / float(np.median(t_dev)), "s_per_call": float(np.median(t_dev)),
                       "spectrum_s": ph[0], "symmetry_s": ph[1], "transform_stats_s": ph[2], "mapping_s": ph[3],
                       "spectrum_gbs": spec_bytes / ph[0] / 1e9 if ph[0] > 0 else None,
                       "internal_points": internal},
            "e2e": {"value": npts / float(np.median(t_host)), "s_per_call": float(np.median(t_host)),
                    "host_memory": "page-locked", "d2h_bytes_per_step": npts * 4,
                    "field_equals_device_output": same}}


def run_configs(args, peaks, clocks):
    """Configurations 1, 2 and 5 (the batched configuration has its own leg)."""
    import torch
    res = {}
    legs = args.configs.split(",") if args.configs else []
    if "1" in legs:
        res["config1"] = _structured_leg(CONFIG1, ["direct", "tc"], steps=min(args.steps, 10), e2e_steps=5,
                                         peaks=peaks, clocks=clocks, cpu_full=True, e2e_form="direct")
        torch.cuda.empty_cache()
    if "2" in legs:
        res["config2"] = _points_leg(CONFIG2, steps=min(args.steps, 10), e2e_steps=3, clocks=clocks)
        torch.cuda.empty_cache()
    if "5" in legs:
        res["config5"] = _structured_leg(CONFIG5, ["tc"], steps=min(args.steps, 3), e2e_steps=2, peaks=peaks,
                                         clocks=clocks)
        torch.cuda.empty_cache()
    return res


def run_b200(args, w):
    import torch
    import torch.distributed as dist

    import scarf3d_b200 as sb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    ds = w["ds"]
    fs = [1, 1, 1 + rank * nz]
    fe = [nx, ny, nz * (rank + 1)]
    n = [nx, ny, nz]
    npts = nx * ny * nz
    # Global extent of the N-slab grid: every rank draws the same harmonics.
    nc = [0.0, 0.0, 0.0]
    fc = [float(np.float32(nx - 1) * np.float32(ds)), float(np.float32(ny - 1) * np.float32(ds)),
          float(np.float32(nz * world - 1) * np.float32(ds))]
    kw = dict(acf=w["acf"], nharm=w["nharm"], seed=w["seed"], hurst=w["hurst"], sigma=w["sigma"], ds=ds, cl=w["cl"])
    p = sb.make_params(nc=nc, fc=fc, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    nh = len(tab)
    i3 = lambda v: (ctypes.c_int * 3)(*[int(x) for x in v])  # noqa: E731

    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    field = torch.empty(npts, dtype=torch.float32, device="cuda")
    # Plans of this grid picked by the autotuner (before any timed region):
    # the device-field plan of the timed step and the fixed-column plan that
    # scarf_execute uses in the end-to-end leg.
    tuned = None
    if not args.no_autotune:
        st0 = torch.cuda.current_stream().cuda_stream
        tuned = {"device_field": sb.tc_autotune(s, fs, n, ds, d_tab.data_ptr(), nh, stream_handle=st0),
                 "execute": sb.tc_autotune(s, fs, n, ds, d_tab.data_ptr(), nh, fixed_columns=True,
                                           stream_handle=st0)}
        sb.set_tc_autotune(1)
    plan = sb.tc_plan_info(3, n, nh)
    wbytes = sb.tc_workspace_bytes(3, n, nh)
    work = torch.empty(wbytes, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    sb.check(sb.lib.scarf_set_kernel_timing(1))

    def tc_step():
        sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), i3(fs), i3(n), ds, ctypes.c_void_p(d_tab.data_ptr()),
                                                nh, ctypes.c_void_p(field.data_ptr()),
                                                ctypes.c_void_p(work.data_ptr()), wbytes, sptr))
        return float(sb.lib.scarf_last_kernel_ms())

    for _ in range(args.warmup):
        tc_step()
    torch.cuda.synchronize()
    kernel_ms = []
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        clk.mark_start()
        ev0.record(stream)
        for _ in range(args.steps):
            kernel_ms.append(tc_step())
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.mark_end()
        barrier()
    t_local = ev0.elapsed_time(ev1) / 1e3
    t = max_over_ranks(t_local)
    work_total = float(npts) * nh * world * args.steps
    value = work_total / t
    k_avg_s = float(np.mean(kernel_ms)) / 1e3
    k_avg_s = max_over_ranks(k_avg_s)

    # Accuracy of the tensor-core field (rank 0): every point against the FP64
    # sum over the identical harmonics (on the GPU, oracle/gpu_fp64.py), and at
    # sampled points against the CPU FP64 oracle and FP32 restatement, all
    # normalised by the field's standard deviation.
    acc = None
    if rank == 0:
        import oracle
        from oracle import gpu_fp64
        op = oracle.params(nc=nc, fc=fc, **kw)
        so = oracle.setup(op)
        full = gpu_fp64.compare_structured(field, so, fs, n, ds, tab)
        rng = np.random.default_rng(0)
        idx = np.sort(rng.choice(npts, size=384, replace=False)).astype(np.int64)
        fstd = full["std_ref"]
        got = field[torch.from_numpy(idx).cuda()].cpu().numpy().astype(np.float64)
        r64 = oracle.sum_structured(so, fs, n, ds, tab, idx=idx, f64=True)
        r32 = oracle.sum_structured(so, fs, n, ds, tab, idx=idx)
        acc = {"full_field": {k: full[k] for k in ("rel_rms", "max_abs", "std_ref", "points")},
               "rel_rms_vs_fp64": full["rel_rms"], "max_abs_vs_fp64": full["max_abs"],
               "sampled_cpu_oracle": {"points": int(len(idx)),
                                      "rel_rms_vs_fp64": float(np.sqrt(np.mean((got - r64) ** 2)) / fstd),
                                      "max_abs_vs_fp64": float(np.max(np.abs(got - r64))),
                                      "rel_rms_fp32_restatement_vs_fp64":
                                          float(np.sqrt(np.mean((r32 - r64) ** 2)) / fstd)}}

    # Operand precision of the tensor-core form: every split (FP16 / BF16
    # hi-lo parts, 3 or 2 products) timed on the same grid and scored over the
    # whole field against FP64; both 3-product splits meet 1e-5, the default
    # (BF16, 3 products) is the faster of the two under the power cap.
    precision = None
    if rank == 0 and not args.no_precision:
        precision = []
        for otype, terms in ((0, 3), (1, 3), (0, 2), (1, 2)):
            sb.set_tc_precision(otype, terms)
            try:
                pb = sb.tc_workspace_bytes(3, n, nh)
                pwork = torch.empty(pb, dtype=torch.uint8, device="cuda")

                def plaunch():
                    sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), i3(fs), i3(n), ds,
                                                            ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                            ctypes.c_void_p(field.data_ptr()),
                                                            ctypes.c_void_p(pwork.data_ptr()), pb, sptr))
                pms = _kernel_times(plaunch, 3)
                torch.cuda.synchronize()
                pf = gpu_fp64.compare_structured(field, so, fs, n, ds, tab)
                precision.append({"operands": ["fp16", "bf16"][otype], "terms": terms,
                                  "kernel_ms": float(np.mean(pms)),
                                  "value": float(npts) * nh / (np.mean(pms) / 1e3),
                                  "rel_rms_vs_fp64": pf["rel_rms"], "max_abs_vs_fp64": pf["max_abs"],
                                  "meets_1e-5": bool(pf["rel_rms"] <= 1e-5)})
                del pwork
            finally:
                sb.set_tc_precision()

    # FP32 direct sum on the same grid and the same harmonics (one warm-up
    # launch over the first DIRECT_HARM harmonics, then the whole table).
    sb.check(sb.lib.scarf_srm_direct_structured(ctypes.byref(s), i3(fs), i3(n), ds, ctypes.c_void_p(d_tab.data_ptr()),
                                                min(DIRECT_HARM, nh), ctypes.c_void_p(field.data_ptr()), sptr))
    sb.check(sb.lib.scarf_srm_direct_structured(ctypes.byref(s), i3(fs), i3(n), ds, ctypes.c_void_p(d_tab.data_ptr()),
                                                nh, ctypes.c_void_p(field.data_ptr()), sptr))
    d_ms = [float(sb.lib.scarf_last_kernel_ms())]
    direct_rate = npts * nh / (np.mean(d_ms) / 1e3)
    direct_acc = None
    if rank == 0:
        dfull = gpu_fp64.compare_structured(field, so, fs, n, ds, tab)
        direct_acc = {k: dfull[k] for k in ("rel_rms", "max_abs", "std_ref", "points")}

    # End to end through the public C ABI (scarf_execute), pinned host field.
    del work
    host = torch.empty(npts, dtype=torch.float32, pin_memory=True)
    opt_fc = np.asarray(fc, np.float32)
    opt_nc = np.asarray(nc, np.float32)
    sb.set_nharm(w["nharm"])
    sb.set_form(sb.FORM_AUTO)
    sb.set_stream(stream.cuda_stream)
    sb.scarf_initialize(fs=fs, fe=fe, ds=ds, acf=w["acf"], cl=w["cl"], sigma=w["sigma"], method=1,
                        hurst=w["hurst"], nc=opt_nc, fc=opt_fc)
    stats = np.zeros(8, np.float32)
    fptr = ctypes.c_void_p(host.data_ptr())
    sptr_stats = stats.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    for _ in range(max(1, args.warmup)):
        sb.check(sb.lib.scarf_execute_ex(w["seed"], fptr, sptr_stats, 0))
    barrier()
    host_s, device_s = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sb.check(sb.lib.scarf_execute_ex(w["seed"], fptr, sptr_stats, 0))
        # stats[4]: host time (setup + harmonic sampling); stats[5]: device
        # time from the table upload to the last byte of the field on the host
        host_s.append(float(stats[4]))
        device_s.append(float(stats[5]))
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    if world > 1:
        # Chan merge of (n, mean, var) across ranks (scarflib_common.f90:823-875).
        from scarf3d_b200.distributed import merge_stats_across_ranks
        merge_stats_across_ranks(float(stats[2]) ** 2, float(stats[3]), npts)
    e2e_value = work_total / t_e2e
    # The same calls into a pageable (malloc'd) host field, as the reference's
    # own C callers allocate it.
    pageable = np.empty(npts, np.float32)
    pageable[:] = 0.0  # touch every page before timing, as a caller's array would be
    pptr = ctypes.c_void_p(pageable.ctypes.data)
    sb.check(sb.lib.scarf_execute_ex(w["seed"], pptr, sptr_stats, 0))
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sb.check(sb.lib.scarf_execute_ex(w["seed"], pptr, sptr_stats, 0))
    t_e2e_pageable = max_over_ranks(time.perf_counter() - t0)
    pageable_ok = bool(np.array_equal(pageable, host.numpy()))
    del pageable
    sb.scarf_finalize()

    clocks = clk.summary()
    peak, peak_sustained, peak_kind = pick_peak(clocks)
    flops_launch = float(npts) * nh * FLOP_PER_PTHARM
    achieved = flops_launch / k_avg_s / 1e12
    traffic = profile_traffic()
    batched = run_batched(args) if (world == 1 and not args.no_batched) else None
    configs = run_configs(args, load_peaks(), clocks) if world == 1 else None
    fim_leg = run_fim(args, clocks) if (world == 1 and not args.no_fim) else None
    if rank == 0:
        cpu = cpu_baseline_sample(w) if world == 1 else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3-split (fp32 accumulate); fp64 phase tables",
            "data": "synthetic (harmonics drawn by the SRM sampler, seed 1234)",
            "config": {"workload": workload_name(w), "grid_per_gpu": n, "global_grid": [nx, ny, nz * world],
                       "nharm": w["nharm"], "harmonics_kept": nh, "form": "tcgen05 BF16 hi/lo 3-product",
                       "l2": "inputs and output larger than L2 (tables 246 MB, field 537 MB per GPU)",
                       "plan": {"variant": ["pair", "single", "single_tmem_a"][plan["variant"]],
                                "tile": [128 // plan["tile_j"], plan["tile_j"]],
                                "longest_axis_as_columns": bool(plan["permute"]),
                                "autotuned": tuned is not None,
                                "tuned": tuned},
                       "parallelism": f"z-slabs x{world}"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind, "peak_sustained": peak_sustained,
                         "frac_of_sustained": achieved / peak_sustained,
                         "kernel": "srm_tc_kernel", "kernel_ms": k_avg_s * 1e3,
                         "flop_per_launch": flops_launch,
                         # the field's one store per point, as HBM write bandwidth over the launch
                         "output_store": {"bytes": npts * 4, "gbs": npts * 4 / k_avg_s / 1e9}},
            "direct_sum": {"value": direct_rate, "unit": UNIT, "harmonics_timed": nh,
                           "kernel_ms": float(np.mean(d_ms)), "tc_over_direct": value / direct_rate,
                           "roofline": _direct_roofline(direct_rate, clocks.get("sm_max_mhz")),
                           "accuracy_vs_fp64_full_field": direct_acc},
            "accuracy": acc,
            "precision_plans": precision,
            "batched": batched,
            "configs": configs,
            "fim": fim_leg,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(nh * 20),
                    "d2h_bytes_per_step": int(npts * 4 + 8), "ms_per_step": t_e2e / args.steps * 1e3,
                    "host_sampling_ms": float(np.mean(host_s)) * 1e3, "device_ms": float(np.mean(device_s)) * 1e3,
                    "host_memory": "page-locked",
                    "pageable": {"value": work_total / t_e2e_pageable, "unit": UNIT,
                                 "ms_per_step": t_e2e_pageable / args.steps * 1e3,
                                 "host_memory": "pageable (numpy, malloc'd)", "field_equals_pinned": pageable_ok}},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_precision_grid(args, w):
    """The operand-precision comparison on the grid and harmonic count given
    (every point against FP64): one line of JSON."""
    import torch

    import oracle
    import scarf3d_b200 as sb
    from oracle import gpu_fp64

    n = [w["nx"], w["ny"], w["nz"]]
    ds = w["ds"]
    fs = [1, 1, 1]
    ds32 = np.float32(ds)
    nc = [0.0, 0.0, 0.0]
    fc = [float(np.float32(n[c] - 1) * ds32) for c in range(3)]
    kw = dict(acf=w["acf"], nharm=w["nharm"], seed=w["seed"], hurst=w["hurst"], sigma=w["sigma"], ds=ds, cl=w["cl"])
    p = sb.make_params(nc=nc, fc=fc, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    nh = len(tab)
    so = oracle.setup(oracle.params(nc=nc, fc=fc, **kw))
    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    field = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    sptr = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    sb.check(sb.lib.scarf_set_kernel_timing(1))
    rows = []
    for otype, terms in ((0, 3), (1, 3), (0, 2)):
        sb.set_tc_precision(otype, terms)
        try:
            wb = sb.tc_workspace_bytes(3, n, nh)
            work = torch.empty(wb, dtype=torch.uint8, device="cuda")

            def launch():
                sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), _i3(fs), _i3(n), ds,
                                                        ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                        ctypes.c_void_p(field.data_ptr()),
                                                        ctypes.c_void_p(work.data_ptr()), wb, sptr))
            ms = _kernel_times(launch, max(1, args.steps))
            torch.cuda.synchronize()
            r = gpu_fp64.compare_structured(field, so, fs, n, ds, tab)
            rows.append({"operands": ["fp16", "bf16"][otype], "terms": terms, "kernel_ms": float(np.mean(ms)),
                         "rel_rms_vs_fp64": r["rel_rms"], "max_abs_over_std": r["max_abs"] / r["std_ref"]})
            del work
        finally:
            sb.set_tc_precision()
    return {"grid": n, "nharm": w["nharm"], "harmonics_kept": nh, "precision_plans": rows}


def run_profile_leg(args, w):
    """One leg alone, for ncu captures of its kernels (prints no bench line):
    tc = table builders + tensor-core sum (warm-up, then one launch) on the
    grid and harmonic count given; direct = the FP32 direct sum over 2 000
    harmonics of it; batched = the 256-field batch (device-assisted sampling,
    builders, persistent launch); fim = scarf_execute with method 0 on the
    grid; execute = scarf_execute (tensor-core form, statistics records) into
    a device field."""
    import torch

    import scarf3d_b200 as sb

    torch.cuda.set_device(0)
    if args.profile_leg == "batched":
        print(json.dumps(run_batched(args, nfields=args.fields)), flush=True)
        return
    if args.profile_leg == "precision":
        print(json.dumps(run_precision_grid(args, w)), flush=True)
        return
    n = [w["nx"], w["ny"], w["nz"]]
    ds = w["ds"]
    fs = [1, 1, 1]
    ds32 = np.float32(ds)
    nc = [0.0, 0.0, 0.0]
    fc = [float(np.float32(n[c] - 1) * ds32) for c in range(3)]
    kw = dict(acf=w["acf"], nharm=w["nharm"], seed=w["seed"], hurst=w["hurst"], sigma=w["sigma"], ds=ds, cl=w["cl"])
    if args.profile_leg in ("fim", "execute"):
        sb.set_nharm(w["nharm"])
        sb.set_form(sb.FORM_TC)
        sb.scarf_initialize(fs=fs, fe=n, ds=ds, acf=w["acf"], cl=w["cl"], sigma=w["sigma"],
                            method=0 if args.profile_leg == "fim" else 1, hurst=w["hurst"],
                            nc=np.asarray(nc, np.float32), fc=np.asarray(fc, np.float32))
        dev = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
        for _ in range(args.warmup + args.steps):
            sb.scarf_execute(w["seed"], dev)
        sb.scarf_finalize()
        return
    p = sb.make_params(nc=nc, fc=fc, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    nh = len(tab) if args.profile_leg == "tc" else min(DIRECT_HARM, len(tab))
    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    field = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    sptr = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    wb = sb.tc_workspace_bytes(3, n, nh)
    work = torch.empty(max(wb, 1), dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup + args.steps):
        if args.profile_leg == "tc":
            sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), _i3(fs), _i3(n), ds,
                                                    ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                    ctypes.c_void_p(field.data_ptr()),
                                                    ctypes.c_void_p(work.data_ptr()), wb, sptr))
        else:
            sb.check(sb.lib.scarf_srm_direct_structured(ctypes.byref(s), _i3(fs), _i3(n), ds,
                                                        ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                        ctypes.c_void_p(field.data_ptr()), sptr))
    torch.cuda.synchronize()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--grid", type=int, nargs=3, default=None, help="override the grid (profiling of small cases)")
    ap.add_argument("--ds", type=float, default=None)
    ap.add_argument("--hurst", type=float, default=None)
    ap.add_argument("--cl", type=float, nargs=3, default=None)
    ap.add_argument("--sigma", type=float, default=None)
    ap.add_argument("--nharm", type=int, default=None)
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-field batched measurement")
    ap.add_argument("--fields", type=int, default=256,
                    help="fields of the batched profile leg (the first N of the 256-field workload)")
    ap.add_argument("--no-autotune", action="store_true", help="default plans instead of autotuned ones")
    ap.add_argument("--no-precision", action="store_true", help="skip the operand-precision comparison")
    ap.add_argument("--no-fim", action="store_true", help="skip the FIM (method 0) measurement")
    ap.add_argument("--profile-leg", choices=["tc", "direct", "batched", "fim", "execute", "precision"], default=None,
                    help="run one leg alone for a profiler capture (no bench line)")
    ap.add_argument("--configs", default="1,2,5",
                    help="other configurations to measure (comma list of 1, 2, 5; empty to skip)")
    args = ap.parse_args()
    w = dict(WORKLOAD)
    if args.grid:
        w["nx"], w["ny"], w["nz"] = args.grid
    if args.nharm:
        w["nharm"] = args.nharm
    for key in ("ds", "hurst", "cl", "sigma"):
        if getattr(args, key) is not None:
            w[key] = getattr(args, key) if key != "cl" else list(getattr(args, key))
    if args.profile_leg:
        run_profile_leg(args, w)
        return
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference(args, w)
    else:
        run_b200(args, w)


if __name__ == "__main__":
    main()
