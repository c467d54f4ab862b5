#!/usr/bin/env python
"""Benchmark of astroflow's dedispersion hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

One step = one pass of the path (binning, RFI stages, dedispersion) over one
chunk already resident in HBM.  Default workload (the configuration the
headline metric is quoted on): 4096 channels of 8-bit samples, 2^20 samples of
49.152 us, DM 0-3000 in steps of 0.5 (6001 trials), subband width 64, IQRM
(std, radius 5, 3 sigma, one window) and the zero-DM filter on, with sinusoidal
RFI channels, broadband impulses and three dispersed pulses injected.

Prints one JSON line (rank 0).  `value` is DM-trial*samples per second over all
ranks (weak scaling: every rank dedisperses its own chunk; the path has no
exchange between GPUs).  `e2e` is the same metric through the C ABI with host
buffers (dd_run_host: host->device copy, run, device->host copy per step);
`e2e_dropin` the same through the drop-in _astroflow_core._dedisperse_spec (host
numpy chunk in, the 512x512x3 images of every t_sample slice out, made on the
GPU).
`--impl reference` times the reference's own CPU implementation of the path
(include/cpucal.hpp, built from source into oracle/_ref) on this host's cores;
`--impl reference-gpu` times the reference's own GPU path (src/core/dedispered.cu
built for sm_100a, its own per-stage timers) on the same chunk.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DM-trial·samples/s"
UNIT = "DM-trial·samples/s"

WORKLOADS = {
    # 4096 ch u8, 2^20 samples, DM 0:0.5:3000, subband width 64, IQRM + zero-DM
    "wideband-4096ch-u8-2^20-6001dm-subband64-rfi": dict(
        nchans=4096, nsamp=1 << 20, nbits=8, dm=(0.0, 3000.0, 0.5), algorithm="subband",
        subband_width=64, ds=1, rfi=dict(use_zero_dm=True, use_iqrm=True, use_mask=False,
                                         iqrm=dict(mode=1, radius_frac=0.00134, nsigma=3.0,
                                                   geofactor=1.5, win_sec=0.0, hop_sec=0.5,
                                                   include_tail=True)),
        chunk=dict(rfi_frac=0.05, rfi_amp=60.0, impulses=20, imp_amp=50.0,
                   pulses=[(120.0, 4.0, 1e-3, 12.0), (780.0, 12.0, 1e-3, 12.0),
                           (2400.0, 20.0, 1e-3, 12.0)])),
    # the same configuration on 2^17 samples (ncu captures: a few GB on the device)
    "wideband-4096ch-u8-2^17-6001dm-subband64-rfi": dict(
        nchans=4096, nsamp=1 << 17, nbits=8, dm=(0.0, 3000.0, 0.5), algorithm="subband",
        subband_width=64, ds=1, rfi=dict(use_zero_dm=True, use_iqrm=True, use_mask=False,
                                         iqrm=dict(mode=1, radius_frac=0.00134, nsigma=3.0,
                                                   geofactor=1.5, win_sec=0.0, hop_sec=0.5,
                                                   include_tail=True)),
        chunk=dict(rfi_frac=0.05, rfi_amp=60.0, impulses=20, imp_amp=50.0,
                   pulses=[(120.0, 0.5, 1e-3, 12.0), (780.0, 1.5, 1e-3, 12.0),
                           (2400.0, 2.5, 1e-3, 12.0)])),
    # the first range of the 8192-channel 16-bit configuration on 2^18 samples (ncu
    # captures of the 16-bit stage 1: a few GB on the device)
    "large-8192ch-u16-2^18-2001dm-subband64-rfi": dict(
        nchans=8192, nsamp=1 << 18, nbits=16, dm=(0.0, 500.0, 0.25), algorithm="subband",
        subband_width=64, ds=1, rfi=dict(use_zero_dm=True, use_iqrm=True, use_mask=False,
                                         iqrm=dict(mode=0, radius_frac=0.1, nsigma=3.0,
                                                   geofactor=1.5, win_sec=0.0, hop_sec=0.5,
                                                   include_tail=True)),
        chunk=dict(rfi_frac=0.08, rfi_amp=6000.0, impulses=20, imp_amp=5000.0,
                   pulses=[(120.0, 1.0, 1e-3, 1200.0), (400.0, 2.0, 1e-3, 1200.0)])),
    # 1024 ch u8, 2^17 samples, DM 0:1:1000, brute force (the CPU path's semantics)
    "plain-1024ch-u8-2^17-1001dm-brute": dict(
        nchans=1024, nsamp=1 << 17, nbits=8, dm=(0.0, 1000.0, 1.0), algorithm="brute",
        subband_width=32, ds=1, rfi=None,
        chunk=dict(pulses=[(565.0, 2.0, 1e-3, 12.0)])),
    # 64 seeded heterogeneous chunks (nchan 1024-4096, 8/16-bit, 2^15-2^19 samples,
    # two bands, DM ranges up to 3000, downsampling 1-8), dedispersed as batches
    "batched-64-heterogeneous-subband32": dict(kind="batch", nchunks=64, seed=2024,
                                               subband_width=32, budget_gb=140.0),
    # the same draw restricted to short chunks (2^15-2^16 samples), where launch
    # overhead is a larger share of each plain call
    "batched-256-short-subband32": dict(kind="batch", nchunks=256, seed=2025, subband_width=32,
                                        budget_gb=140.0, log2_nsamp=(15.0, 16.0)),
    # 8192 ch u16, 2^21 samples, three DM ranges on one resident chunk (DM 0:0.25:500 ds 1,
    # 500:0.5:2000 ds 2, 2000:1:5000 ds 4), subband width 64 (128 subbands), IQRM + zero-DM
    "large-8192ch-u16-2^21-multirange-subband64-rfi": dict(
        kind="multirange", nchans=8192, nsamp=1 << 21, nbits=16, subband_width=64,
        ranges=[(0.0, 500.0, 0.25, 1), (500.0, 2000.0, 0.5, 2), (2000.0, 5000.0, 1.0, 4)],
        rfi=dict(use_zero_dm=True, use_iqrm=True, use_mask=False,
                 iqrm=dict(mode=1, radius_frac=0.00067, nsigma=3.0, geofactor=1.5, win_sec=0.0,
                           hop_sec=0.5, include_tail=True)),
        chunk=dict(rfi_frac=0.08, rfi_amp=6000.0, impulses=20, imp_amp=5000.0,
                   pulses=[(300.0, 20.0, 1e-3, 1200.0), (1200.0, 50.0, 1e-3, 1200.0),
                           (3500.0, 70.0, 1e-3, 1200.0)])),
    # 19 beams streaming 0.5 s chunks of 4096 ch u8 in real time (DM 0:1:3000, zero-DM +
    # IQRM) plus Poisson file requests (2/s, 1024-4096 ch, 5-60 s) under a 150 GB budget;
    # --steps = seconds of served time
    "serving-19beams-4096ch-u8-3001dm-files": dict(
        kind="serve", beams=19, nchans=4096, chunk_s=0.5, tsamp=49.152e-6, dm=(0.0, 3000.0, 1.0),
        subband_width=64, file_rate=2.0, file_s=(5.0, 60.0), file_nchans=(1024, 2048, 4096),
        budget_gb=150.0, seed=77),
}
DEFAULT_WORKLOAD = "wideband-4096ch-u8-2^20-6001dm-subband64-rfi"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        smax = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(self.rows)}


# ---------------------------------------------------------------- reference CPU
def reference_cpu_rate(x_host: np.ndarray, hdr: dict, wl: dict, target_s: float):
    """Time the reference's cpucal::dedispered_fil_omp (built from source into
    oracle/_ref) on a bounded sample of the workload: every k-th DM trial of the
    workload's grid over the chunk's first n = min(nsamp, 2^18) samples.  n is
    longer than the largest delay of every workload plus a 0.5 s slice, so the
    share of delayed samples past the sample's end (which the reference skips,
    include/cpucal.hpp:181) stays small; the reference parallelises over DM
    trials, so the sample keeps at least one trial per thread, and k is chosen
    so that one call takes about target_s seconds.  Returns (DM-trial*samples/s,
    threads, sample description, seconds of the timed call)."""
    from oracle import oracle as O

    lib = O.ref_cpu()
    threads = int(lib.ref_cpu_threads())
    nchans = hdr["nchans"]
    n = min(x_host.shape[0], 1 << 18)
    lo, hi, step = wl["dm"]
    freq = O.freq_table_fil(hdr["fch1"], hdr["foff"], nchans)
    fs, fe = float(np.float32(freq[0])), float(np.float32(freq[-1]))
    ndm_full = O.dm_steps(lo, hi, step)
    xs = np.ascontiguousarray(x_host[:n])

    def run(k):
        st = float(np.float32(step * k))
        t = time.perf_counter()
        O.ref_bruteforce_cpu(xs, nchans, hdr["fch1"], hdr["foff"], hdr["tsamp"], lo, hi, fs, fe,
                             st, 1, n * hdr["tsamp"] * 0.999)
        return time.perf_counter() - t, O.dm_steps(lo, hi, st)

    k = max(1, ndm_full // threads)
    dt, nd = run(k)
    grow = int(target_s / max(dt, 1e-3))
    if grow > 1:
        k = max(1, k // grow)
        dt, nd = run(k)
    rate = nd * n / dt
    sample = (f"reference cpucal::dedispered_fil_omp (brute force, the reference's CPU path) on "
              f"{nd} of the {ndm_full} DM trials (every {k}-th, DM {lo:g} to {hi:g}) over the "
              f"first {n} samples x {nchans} channels, {threads} OpenMP threads; the rate is "
              f"extrapolated to the full DM grid and chunk")
    return rate, threads, sample, dt


def bench_batch(args, wl, dist, dev):
    """Heterogeneous batch: the seeded chunks of synth.draw_batch dedispersed (a) one
    plain call per chunk (Plan.run, back to back on one stream), (b) as a grouped
    batch and (c) as a persistent batch (Batch, replayed from a CUDA graph).  Chunks
    are grouped into waves that fit the HBM budget; `value` is the faster batched
    form's throughput over all chunks."""
    import torch

    from astroflow_b200.dedisp import Batch, Plan, measure_int_add_rate
    from astroflow_b200.synth import draw_batch, make_chunk_device

    f32 = np.float32
    chunks = draw_batch(wl["nchunks"], seed=wl["seed"] + dist.rank, subband_width=wl["subband_width"],
                        log2_nsamp=wl.get("log2_nsamp", (15.0, 19.0)))
    budget = wl["budget_gb"] * 1e9
    stream = torch.cuda.current_stream(dev)
    times = {"plain": 0.0, "grouped": 0.0, "persistent": 0.0}
    launches = {"plain": 0, "grouped": 0, "persistent": 0}
    units_total = adds_total = bytes_total = 0.0
    waves = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    clocks = ClockSampler(dev)
    clocks.start()
    i = 0
    while i < len(chunks):
        plans, xs, outs, used = [], [], [], 0.0
        while i < len(chunks):
            c = chunks[i]
            hdr = c.spec.header()
            for k in ("tsamp", "fch1", "foff"):
                hdr[k] = float(f32(hdr[k]))
            lo = float(f32(hdr["fch1"]))
            hi = float(f32(f32(hdr["fch1"]) + f32(hdr["nchans"] - 1) * f32(hdr["foff"])))
            plan = Plan(hdr, 0.0, c.dm_high, lo, hi, c.dm_step, c.time_downsample,
                        algorithm="subband", subband_width=c.subband_width, device=dev)
            need = (plan.info["workspace_bytes"] + plan.out_shape[0] * plan.out_shape[1] * 4 +
                    plan.in_shape[0] * plan.in_shape[1] * plan.nbits // 8)
            if plans and used + need > budget:
                plan.close()
                break
            x, _ = make_chunk_device(c.spec, dev)
            o = plan.empty_output()
            if args.autotune:  # per-plan launch shape on its own chunk (untimed)
                try:
                    plan.autotune(x, o, reps=1, stream=stream)
                except RuntimeError:  # plans on the direct kernels have no staged shape
                    pass
                need += plan.info["workspace_bytes"] - (need - o.numel() * 4 - x.numel() * x.element_size())
            plans.append(plan)
            xs.append(x)
            outs.append(o)
            used += need
            i += 1
        units = sum(p.out_shape[0] * p.out_shape[1] for p in plans)
        wave = {"chunks": len(plans), "gb": round(used / 1e9, 1), "units": units}

        def plain():
            for p, x, o in zip(plans, xs, outs):
                p.run(x, o, stream)
        wave["plain_ms"] = timed(plain)
        launches["plain"] += args.steps * sum(p.run_profiled(x, o, stream)["launches"]
                                              for p, x, o in zip(plans, xs, outs))
        for mode in ("grouped", "persistent"):
            batch = Batch(plans, use_graph=True, persistent=(mode == "persistent"))
            wave[mode + "_ms"] = timed(lambda: batch.run(xs, outs, stream))
            batch.status()
            launches[mode] += batch.info["launches"] * args.steps
            wave[mode + "_sum_launches"] = batch.info["sum_launches"]
            wave[mode + "_own_plans"] = batch.info["own_plans"]
            batch.close()
        for k in times:
            times[k] += wave[k + "_ms"]
        units_total += units
        adds_total += sum(p.info["adds_per_run"] for p in plans)
        bytes_total += sum(p.in_shape[0] * p.in_shape[1] * p.nbits / 8 + p.out_shape[0] * p.out_shape[1] * 4
                           for p in plans)
        waves.append(wave)
        for p in plans:
            p.close()
        del xs, outs
        torch.cuda.empty_cache()
    clk = clocks.stop()
    best = min(("grouped", "persistent"), key=lambda k: times[k])
    rate = dist.job_rate(units_total, times[best] * 1e-3)
    rates = {k: dist.job_rate(units_total, t * 1e-3) for k, t in times.items()}
    ms = dist.max(times[best])
    hbm_peak, peak_kind = roofline_peaks()
    add_peak = measure_int_add_rate(dev)
    t = times[best] * 1e-3
    roof_s = max(bytes_total / (hbm_peak * 1e9), adds_total / add_peak)
    if dist.rank == 0:
        line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u8/u16", "data": f"synthetic (seeded draw of {len(chunks)} chunks, generated on the GPU)",
                "config": {"workload": args.workload, "chunks": len(chunks), "batched_form": best,
                           "waves": waves, "seed": wl["seed"], "subband_width": wl["subband_width"],
                           "hbm_budget_gb": wl["budget_gb"],
                           "l2": "inputs larger than L2 per wave; no flush between steps",
                           "parallelism": f"replicas x{dist.world}"},
                "forms": {k: {"value": rates[k], "ms_per_step": times[k], "launches": launches[k]}
                          for k in times},
                "batched_over_plain": times["plain"] / times[best],
                "roofline": {"bound": "hbm", "achieved": bytes_total / t / 1e9, "peak": hbm_peak,
                             "unit": "GB/s", "frac": bytes_total / t / 1e9 / hbm_peak,
                             "peak_kind": peak_kind, "traffic": None,
                             "int_add": {"achieved": adds_total / t, "peak": add_peak, "unit": "adds/s",
                                         "frac": adds_total / t / add_peak},
                             "step_frac": roof_s / t},
                "cpu_baseline": None, "e2e": None, "gpu_launches": launches[best], "clocks": clk}
        print(json.dumps(line))


def bench_multirange(args, wl, dist, dev):
    """One resident chunk searched over several (DM range, downsampling) entries
    (MultiPlan: one upload, one plan per range).  `value` counts the output
    DM-trial*samples of all ranges per second; `e2e` adds the chunk's upload and
    every range's output download (pinned host buffers)."""
    import torch

    from astroflow_b200.dedisp import IqrmParams, MultiPlan, RfiParams, measure_int_add_rate
    from astroflow_b200.synth import ChunkSpec, make_chunk_device

    f32 = np.float32
    spec = ChunkSpec(nchans=wl["nchans"], nsamp=wl["nsamp"], nbits=wl["nbits"],
                     seed=dist.chunk_seed(4321), **wl["chunk"])
    hdr = spec.header()
    for k in ("tsamp", "fch1", "foff"):
        hdr[k] = float(f32(hdr[k]))
    lo = float(f32(hdr["fch1"]))
    hi = float(f32(f32(hdr["fch1"]) + f32(wl["nchans"] - 1) * f32(hdr["foff"])))
    r = wl["rfi"]
    rfi = RfiParams(use_mask=r["use_mask"], use_zero_dm=r["use_zero_dm"], use_iqrm=r["use_iqrm"],
                    iqrm=IqrmParams(**r["iqrm"]))
    x, _ = make_chunk_device(spec, dev)
    mp = MultiPlan(hdr, wl["ranges"], lo, hi, subband_width=wl["subband_width"], rfi=rfi,
                   device=dev)
    outs = mp.empty_outputs()
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        mp.run(x, outs, stream)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)
    dist.barrier()
    torch.cuda.synchronize(dev)
    from astroflow_b200 import _lib

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = _lib.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        mp.run(x, outs, stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    timed_launches = _lib.launch_count() - l0
    dist.barrier()
    clk = clocks.stop()
    ms_rank = e0.elapsed_time(e1) / args.steps
    units = sum(p.out_shape[0] * p.out_shape[1] for p in mp.plans)
    value = dist.job_rate(units, ms_rank * 1e-3)
    ms = dist.max(ms_rank)
    stages = [p.run_profiled(x, o, stream) for p, o in zip(mp.plans, outs)]
    adds = sum(p.info["adds_per_run"] for p in mp.plans)
    in_bytes = wl["nsamp"] * wl["nchans"] * wl["nbits"] // 8
    out_bytes = mp.output_bytes
    hbm_peak, peak_kind = roofline_peaks()
    add_peak = measure_int_add_rate(dev)
    roof_s = max((in_bytes + out_bytes) / (hbm_peak * 1e9), adds / add_peak)
    e2e = None
    if args.e2e_steps > 0:
        h_in = torch.empty(tuple(x.shape), dtype=x.dtype, pin_memory=True)
        h_in.copy_(x)
        h_outs = [torch.empty(tuple(o.shape), dtype=torch.int32, pin_memory=True) for o in outs]
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e2.record(stream)
        for _ in range(args.e2e_steps):
            x.copy_(h_in, non_blocking=True)
            mp.run(x, outs, stream)
            for o, h in zip(outs, h_outs):
                h.copy_(o.view(torch.int32), non_blocking=True)
        e3.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = e2.elapsed_time(e3) / args.e2e_steps
        e2e = {"value": dist.job_rate(units, e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(in_bytes), "d2h_bytes_per_step": int(out_bytes),
               "ms_per_step": e2e_ms}
    if dist.rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": f"u{wl['nbits']}", "data": "synthetic (seeded, generated on the GPU)",
                "config": {"workload": args.workload, "nchans": wl["nchans"], "nsamp": wl["nsamp"],
                           "ranges": wl["ranges"], "subband_width": wl["subband_width"],
                           "rfi": "iqrm + zero-DM (reference call-site semantics)",
                           "device_gb": round((mp.workspace_bytes + out_bytes + in_bytes) / 1e9, 1),
                           "l2": "inputs larger than L2", "parallelism": f"replicas x{dist.world}"},
                "ranges_ms": [{k: round(v, 2) if isinstance(v, float) else v for k, v in st.items()}
                              for st in stages],
                "roofline": {"bound": "hbm", "achieved": (in_bytes + out_bytes) / (ms * 1e-3) / 1e9,
                             "peak": hbm_peak, "unit": "GB/s",
                             "frac": (in_bytes + out_bytes) / (ms * 1e-3) / 1e9 / hbm_peak,
                             "peak_kind": peak_kind, "traffic": None,
                             "int_add": {"achieved": adds / (ms * 1e-3), "peak": add_peak,
                                         "unit": "adds/s", "frac": adds / (ms * 1e-3) / add_peak},
                             "step_frac": roof_s / (ms * 1e-3)},
                "cpu_baseline": None, "e2e": e2e,
                "gpu_launches": int(timed_launches),
                "clocks": clk}
        print(json.dumps(line))
    mp.close()


def bench_serve(args, wl, dist, dev):
    """Serving: beams stream chunks in real time and files arrive as a Poisson
    process; everything goes through astroflow_b200.serve.Server.  `value` is the
    DM-trial*samples served per second over the timed window (args.steps seconds
    after args.warmup seconds of warm-up); latencies are arrival -> DM-time ready
    (chunks: on the host, files: on the device)."""
    import torch

    from astroflow_b200.dedisp import IqrmParams, RfiParams, Stream
    from astroflow_b200.serve import Server
    from astroflow_b200.synth import ChunkSpec, make_chunk_device

    f32 = np.float32
    rng = np.random.default_rng(wl["seed"] + dist.rank)
    nch, tsamp = wl["nchans"], wl["tsamp"]
    chunk = int(wl["chunk_s"] / tsamp)
    lo_dm, hi_dm, step_dm = wl["dm"]
    rfi = RfiParams(use_zero_dm=True, use_iqrm=True,
                    iqrm=IqrmParams(mode=1, radius_frac=0.00134, nsigma=3.0, win_sec=0.0, hop_sec=0.5))

    def geometry(nchans, n):
        spec = ChunkSpec(nchans=nchans, nsamp=n, nbits=8, tsamp=tsamp, seed=int(rng.integers(1 << 30)),
                         rfi_frac=0.05, impulses=2,
                         pulses=[(float(rng.uniform(100, 2500)), 0.3 * n * tsamp, 1e-3, 12.0)])
        h = spec.header()
        for k in ("tsamp", "fch1", "foff"):
            h[k] = float(f32(h[k]))
        lo = float(f32(h["fch1"]))
        hi = float(f32(f32(h["fch1"]) + f32(nchans - 1) * f32(h["foff"])))
        return spec, h, lo, hi

    # host data: a pool of beam chunks and one long file buffer (pinned)
    pool = []
    for k in range(8):
        spec, h, lo, hi = geometry(nch, chunk)
        x, _ = make_chunk_device(spec, dev)
        pool.append(x.cpu().pin_memory())
    beam_hdr, beam_lo, beam_hi = dict(h, ndata=chunk), lo, hi
    max_file = int(wl["file_s"][1] / tsamp)
    spec, _, _, _ = geometry(4096, max_file)
    filebuf = torch.empty((max_file, 4096), dtype=torch.uint8, pin_memory=True)
    step_rows = 1 << 18
    for r0 in range(0, max_file, step_rows):
        part = ChunkSpec(nchans=4096, nsamp=min(step_rows, max_file - r0), nbits=8, tsamp=tsamp,
                         seed=wl["seed"] + r0)
        xp, _ = make_chunk_device(part, dev)
        filebuf[r0:r0 + xp.shape[0]].copy_(xp)
        del xp
    torch.cuda.synchronize(dev)

    def file_request(arrival):
        nchans = int(rng.choice(wl["file_nchans"]))
        n = int(rng.uniform(*wl["file_s"]) / tsamp)
        spec, h, lo, hi = geometry(nchans, n)
        data = filebuf.view(-1)[:n * nchans].view(n, nchans)
        kw = dict(dm_low=lo_dm, dm_high=hi_dm, freq_start=lo, freq_end=hi, dm_step=step_dm,
                  subband_width=wl["subband_width"] if nchans >= 2048 else 32, rfi=rfi)
        return data, dict(h, ndata=n), kw

    srv = Server(device=dev, hbm_budget_gb=wl["budget_gb"])
    beams = [srv.open_beam(f"beam{b}", beam_hdr, lo_dm, hi_dm, beam_lo, beam_hi, step_dm,
                           subband_width=wl["subband_width"], rfi=rfi) for b in range(wl["beams"])]
    # the plain single call: one chunk of one beam alone on the device
    solo = Stream(beam_hdr, lo_dm, hi_dm, beam_lo, beam_hi, step_dm,
                  subband_width=wl["subband_width"], rfi=rfi, device=dev)
    xs = pool[0].to(f"cuda:{dev}")
    out = solo.empty_output()
    host = torch.empty(solo.out_shape, dtype=torch.int32, pin_memory=True)
    solo_ms = []
    for _ in range(5):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        xs.copy_(pool[1], non_blocking=True)
        solo.push(xs, out)
        host.copy_(out.view(torch.int32), non_blocking=True)
        torch.cuda.synchronize(dev)
        solo_ms.append((time.perf_counter() - t0) * 1e3)
    solo.close()

    period = wl["chunk_s"]
    phase = [b * period / len(beams) for b in range(len(beams))]
    t_start = time.monotonic()
    warm_end = t_start + args.warmup
    end = warm_end + args.steps
    next_chunk = [t_start + p for p in phase]
    kchunk = [0] * len(beams)
    next_file = t_start + rng.exponential(1.0 / wl["file_rate"])
    clocks = ClockSampler(dev)
    clocks.start()
    files_submitted = 0
    while True:
        now = time.monotonic()
        if now >= end:
            break
        for b, beam in enumerate(beams):
            while next_chunk[b] <= now:
                srv.submit_chunk(beam, pool[(b + kchunk[b]) % len(pool)], arrival=next_chunk[b])
                kchunk[b] += 1
                next_chunk[b] += period
        while next_file <= now:
            srv.submit_file(*file_request(next_file), arrival=next_file)
            files_submitted += 1
            next_file += rng.exponential(1.0 / wl["file_rate"])
        srv.step()
        time.sleep(0.0002)
    # units served in the window: requests that arrived in it and finished
    srv.drain(timeout=900)
    clk = clocks.stop()
    st = srv.stats(since=warm_end)
    window = [t for t in srv.finished if warm_end <= t.arrival < end and not t.error]
    t_last = max(t.done for t in window) if window else end
    units = sum(t.units for t in window)
    rate = units / (t_last - warm_end)
    srv.close()
    if dist.rank == 0:
        chunks_lat = st["chunks"]
        line = {"metric": METRIC, "value": dist.job_rate(units, t_last - warm_end), "unit": UNIT,
                "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": (t_last - warm_end) * 1e3 / max(1, args.steps),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                "data": "synthetic (seeded, generated on the GPU, pinned host buffers)",
                "config": {"workload": args.workload, "beams": wl["beams"], "chunk_samples": chunk,
                           "dm": wl["dm"], "subband_width": wl["subband_width"],
                           "file_rate_per_s": wl["file_rate"], "file_seconds": wl["file_s"],
                           "hbm_budget_gb": wl["budget_gb"], "window_s": args.steps,
                           "step": "one second of served time",
                           "l2": "inputs larger than L2", "parallelism": f"replicas x{dist.world}"},
                "serving": {"chunk_latency": chunks_lat, "file_latency": st["files"],
                            "files_submitted": files_submitted, "errors": st["errors"][:3],
                            "plain_chunk_ms": {"p50": float(np.median(solo_ms)), "max": float(max(solo_ms))},
                            "chunk_deadline_s": period,
                            "p99_under_deadline": bool(chunks_lat.get("p99_s", 1e9) < period),
                            "served_rate": rate},
                "roofline": None, "cpu_baseline": None,
                "e2e": {"value": rate, "unit": UNIT, "note": "requests from pinned host buffers; "
                        "chunk results copied back to the host"},
                "gpu_launches": None, "clocks": clk}
        print(json.dumps(line))


def reference_gpu_arm(args, wl, spec, hdr, config, dist, dev):
    """The reference's own plain GPU call (gpucal::dedisperse_spec from
    src/core/dedispered.cu, built for sm_100a into oracle/_ref with its AF_DEBUG
    timers on) on the workload's chunk, one call per step.  `value` uses the
    reference's device-timed stages (binning, RFI, stage 1, stage 2); `e2e` the
    host time of the whole call (allocations, pageable copies, sums)."""
    from astroflow_b200.synth import make_chunk_device
    from oracle import oracle as O

    if dist.rank != 0:
        dist.close()
        return
    sbw = wl["subband_width"] if wl["algorithm"] == "subband" else None
    if sbw is None or not O.ref_gpu_timed_available(sbw):
        print(json.dumps({"impl": "reference-gpu", "unavailable": "the reference GPU path has no "
                          "brute-force kernels compiled in (AF_USE_SUBBAND), or its timing build "
                          "oracle/_ref/libref_gpu_timed_sb*.so is missing"}))
        return
    x, _ = make_chunk_device(spec, dev)
    x_host = x.cpu().numpy()
    del x
    lo, hi, step = wl["dm"]
    f32 = np.float32
    fs = float(f32(hdr["fch1"]))
    fe = float(f32(f32(hdr["fch1"]) + f32(hdr["nchans"] - 1) * f32(hdr["foff"])))
    r = wl["rfi"] or {}
    iq = None
    if r.get("use_iqrm"):
        from types import SimpleNamespace
        iq = SimpleNamespace(**r["iqrm"])

    def call():
        return O.ref_gpu_time_spec(x_host, hdr["nchans"], hdr["tsamp"], hdr["fch1"], hdr["foff"], lo,
                                   hi, fs, fe, step, wl["ds"], sb_width=sbw,
                                   use_zero_dm=r.get("use_zero_dm", False),
                                   use_iqrm=r.get("use_iqrm", False), iq=iq, device=dev)

    for _ in range(max(1, min(args.warmup, 2))):
        call()
    runs = [call() for _ in range(max(1, args.steps))]
    rows, cols = runs[0][0], runs[0][1]
    units = rows * cols
    keys = ["Time binning", "IQRM generate", "IQRM mask", "Zero-DM filtering", "Maskfile marking",
            "Stage1 (subband)", "Stage2 (subband)"]
    dev_ms = [sum(t.get(k, 0.0) for k in keys) for _, _, t in runs]
    wall_ms = [t["wall"] for _, _, t in runs]
    med = lambda v: float(np.median(v))
    timers = {k: med([t.get(k, 0.0) for _, _, t in runs]) for k in runs[0][2]}
    line = {"impl": "reference-gpu", "metric": METRIC, "value": units / (med(dev_ms) * 1e-3),
            "unit": UNIT, "n_gpus": 1, "steps": len(runs), "warmup": args.warmup,
            "ms_per_step": med(dev_ms), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": f"u{wl['nbits']}", "data": "synthetic", "config": config,
            "e2e": {"value": units / (med(wall_ms) * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": int(x_host.nbytes),
                    "d2h_bytes_per_step": int(units * 4), "ms_per_step": med(wall_ms)},
            "reference_timers_ms": timers,
            "note": "value: the reference's device-timed stages (its AF_DEBUG CUDA-event timers); "
                    "e2e: host time of the whole reference call"}
    print(json.dumps(line))


# ---------------------------------------------------------------- extras
EXTRAS = [
    # (key, bench.py arguments): short runs, each in its own process on this GPU
    ("reference-gpu", ["--impl", "reference-gpu", "--steps", "2", "--warmup", "1"]),
    # (the 256-short-chunk batch workload runs on request: --workload batched-256-short-subband32)
    ("plain-1024ch-u8-2^17-1001dm-brute", ["--workload", "plain-1024ch-u8-2^17-1001dm-brute",
                                           "--steps", "10", "--warmup", "3", "--e2e-steps", "2"]),
    ("batched-64-heterogeneous-subband32", ["--workload", "batched-64-heterogeneous-subband32",
                                            "--steps", "2", "--warmup", "1", "--no-autotune"]),
    ("large-8192ch-u16-2^21-multirange-subband64-rfi", ["--workload",
                                                       "large-8192ch-u16-2^21-multirange-subband64-rfi",
                                                       "--steps", "3", "--warmup", "3",
                                                       "--e2e-steps", "1"]),
    ("serving-19beams-4096ch-u8-3001dm-files", ["--workload",
                                                "serving-19beams-4096ch-u8-3001dm-files",
                                                "--steps", "10", "--warmup", "3"]),
]
EXTRA_KEYS = ("impl", "value", "unit", "ms_per_step", "steps", "warmup", "e2e", "cpu_baseline",
              "batched_over_plain", "forms", "serving", "clocks", "gpu_launches", "unavailable",
              "reference_timers_ms")


def run_extras(dev):
    """The other workloads and the reference's plain GPU call, run briefly after the
    headline measurement so that their numbers come from the same bench run.  Each
    runs as `bench.py --no-extras ...` in a child process on this GPU (the headline's
    buffers are released first); the child's JSON line is kept, trimmed to its
    results and roofline."""
    import subprocess

    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)))
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = {}
    for key, argv in EXTRAS:
        t = time.perf_counter()
        try:
            r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--no-extras", *argv],
                               capture_output=True, text=True, timeout=900, env=env)
            lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
            d = json.loads(lines[-1]) if lines else {"error": (r.stderr or r.stdout)[-400:]}
        except subprocess.TimeoutExpired:
            d = {"error": "timed out after 900 s"}
        res = {k: d[k] for k in EXTRA_KEYS if k in d}
        if "roofline" in d and d["roofline"]:
            res["roofline"] = {k: d["roofline"].get(k) for k in
                               ("achieved", "peak", "unit", "frac", "step_frac", "int_add", "kernel",
                                "stages_ms") if k in d["roofline"]}
        if "config" in d:
            res["config"] = d["config"]
        if "error" in d:
            res["error"] = d["error"]
        res["run_seconds"] = round(time.perf_counter() - t, 1)
        out[key] = res
    return out


# ---------------------------------------------------------------- helpers
def parity_rows(wl, plan):
    """DM rows checked against the reference build: the first two, the rows of the
    injected pulses' DMs, the middle and the last two."""
    lo, hi, step = wl["dm"]
    n = int(plan.out_shape[0])
    rows = {0, 1, n // 2, n - 2, n - 1}
    for dm, *_ in wl["chunk"].get("pulses", []):
        rows.add(int(min(n - 1, max(0, round((dm - lo) / step)))))
    return sorted(r for r in rows if 0 <= r < n)


def reference_parity(x_host, hdr, wl, rows, ours_rows, dev):
    """The timed output's rows (all columns) against the reference's own GPU path
    (gpucal::dedisperse_spec, src/core/dedispered.cu:988-1304, built from its
    sources into oracle/_ref) run on the same chunk.  A checker: it runs after the
    timed region and its time is not part of any reported number."""
    from oracle import oracle as O

    sbw = wl["subband_width"]
    if not O.ref_gpu_available(sbw):
        return None
    lo, hi, step = wl["dm"]
    f32 = np.float32
    fs = float(f32(hdr["fch1"]))
    fe = float(f32(f32(hdr["fch1"]) + f32(hdr["nchans"] - 1) * f32(hdr["foff"])))
    r = wl["rfi"] or {}
    iq = None
    if r.get("use_iqrm"):
        from types import SimpleNamespace
        iq = SimpleNamespace(**r["iqrm"])
    t = time.perf_counter()
    ref = O.ref_gpu_dedisperse_spec_rows(x_host, hdr["nchans"], hdr["tsamp"], hdr["fch1"],
                                         hdr["foff"], lo, hi, fs, fe, step, wl["ds"], rows=rows,
                                         sb_width=sbw, use_zero_dm=r.get("use_zero_dm", False),
                                         use_iqrm=r.get("use_iqrm", False), iq=iq, device=dev)
    dt = time.perf_counter() - t
    ours = ours_rows.view(__import__("torch").int32).numpy().view(np.uint32)
    bad = int((ours != ref).sum()) if ours.shape == ref.shape else -1
    return {"ok": bad == 0, "rows": rows, "columns": int(ref.shape[1]), "mismatches": bad,
            "reference": f"oracle/_ref/libref_gpu_sb{sbw}.so: the reference's gpucal::dedisperse_spec "
                         "(src/core/dedispered.cu) built from its sources for sm_100a, raw sums",
            "seconds": round(dt, 1)}


def roofline_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel: str, units_launch: float):
    """DRAM bytes (read + write) of one launch of `kernel` at this workload: the
    committed ncu capture's bytes per DM-trial*sample times the launch's units
    (profiles/traffic.txt: kernel, DRAM bytes of the captured launch, its units)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel:
            try:
                return float(parts[1]) / float(parts[2]) * units_launch
            except ValueError:
                return None
    return None


def make_plan(wl, hdr, device):
    from astroflow_b200.dedisp import IqrmParams, Plan, RfiParams

    lo, hi, step = wl["dm"]
    freq_lo = float(np.float32(np.float32(hdr["fch1"])))
    nch = hdr["nchans"]
    f32 = np.float32
    top = float(f32(f32(hdr["fch1"]) + f32(nch - 1) * f32(hdr["foff"])))
    rfi = None
    if wl["rfi"]:
        r = wl["rfi"]
        rfi = RfiParams(use_mask=r["use_mask"], use_zero_dm=r["use_zero_dm"],
                        use_iqrm=r["use_iqrm"], iqrm=IqrmParams(**r["iqrm"]))
    if wl["algorithm"] == "brute":
        return Plan(hdr, lo, hi, freq_lo, top, step, wl["ds"], hdr["nsamp_total_s"],
                    algorithm="brute", freq_mode="fil", device=device)
    return Plan(hdr, lo, hi, freq_lo, top, step, wl["ds"], algorithm="subband",
                subband_width=wl["subband_width"], rfi=rfi, device=device)


def e2e_run(plan, x, out, units, dist, dev, stream, steps, warmup):
    """The workload's metric through the host-buffer calls with pinned host buffers
    (host->device copy, run, device->host copy of every step inside the timed
    region): steps are queued back to back with dd_run_host_async, as a streaming
    caller does, so one step's output copy overlaps the next step's input copy;
    dd_run_host_join then makes the timing stream wait for the last output copy.
    Returns (e2e dict, whether the host path's first rows equal the device-resident
    run's)."""
    import torch

    h_in = torch.empty(tuple(x.shape), dtype=x.dtype, pin_memory=True)
    h_in.copy_(x)
    h_out = torch.empty(plan.out_shape, dtype=out.dtype, pin_memory=True)
    h_in_np = h_in.view(torch.uint8).numpy() if x.dtype == torch.uint8 else h_in.view(torch.int16).numpy().view(np.uint16)
    h_out_np = h_out.view(torch.int32).numpy().view(np.uint32)
    for _ in range(max(1, warmup)):  # warm-up (allocator pool, caches)
        plan.run_host(h_in_np, h_out_np, stream)
    dist.barrier()
    torch.cuda.synchronize(dev)
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(steps):
        plan.run_host_async(h_in_np, h_out_np, stream)
    plan.run_host_join(stream)
    e3.record(stream)
    torch.cuda.synchronize(dev)
    plan.run_host_join(stream, sync=True)  # device-side failures of the queued runs
    e2e_rank_ms = e2.elapsed_time(e3) / steps
    e2e_rate = dist.job_rate(units, e2e_rank_ms * 1e-3)
    e2e_ms = dist.max(e2e_rank_ms)
    e2e = {"value": e2e_rate, "unit": UNIT,
           "h2d_bytes_per_step": int(h_in.numel() * h_in.element_size()),
           "d2h_bytes_per_step": int(h_out.numel() * h_out.element_size()),
           "ms_per_step": e2e_ms,
           "calls": "dd_run_host_async per step (one step's output copy overlaps the next "
                    "step's input copy), dd_run_host_join"}
    # bit-level spot check of the host path against the device run
    same = bool(torch.equal(h_out[:4].to(dev).view(torch.int32), out[:4].view(torch.int32)))
    return e2e, same


def e2e_dropin_run(wl, hdr, x, units, dist, dev, steps, warmup, t_sample=0.5):
    """The workload's metric through the drop-in call the reference's users make,
    _astroflow_core._dedisperse_spec: a host numpy chunk in, the t_sample-second
    512x512x3 viridis images out (what the reference returns), every copy and the
    image step inside the timed region."""
    import torch

    from astroflow_b200 import _astroflow_core as C

    x_host = x.cpu().numpy()
    if wl["nbits"] == 16:
        x_host = x_host.view(np.uint16)
    header = C.Header(0.0, hdr["tsamp"], hdr["fch1"], hdr["foff"], wl["nbits"], wl["nchans"],
                      wl["nsamp"], "bench")
    r = wl["rfi"]
    rfi = C.RFIconfig()
    if r:
        q = r["iqrm"]
        rfi = C.RFIconfig(r["use_mask"], r["use_zero_dm"], r["use_iqrm"],
                          C.IQRMconfig(q["mode"], q["radius_frac"], q["nsigma"], q["geofactor"],
                                       q["win_sec"], q["hop_sec"], q["include_tail"]))
    C.SUBBAND_WIDTH = wl["subband_width"]
    lo, hi, step = wl["dm"]
    f32 = np.float32
    fs = float(f32(hdr["fch1"]))
    fe = float(f32(f32(hdr["fch1"]) + f32(wl["nchans"] - 1) * f32(hdr["foff"])))
    args = (x_host, header, lo, hi, fs, fe, step, wl["ds"], t_sample, dev, "", rfi)
    for _ in range(max(1, warmup)):  # the first call builds and caches the plan
        res = C._dedisperse_spec(*args)
    stream = torch.cuda.current_stream(dev)
    dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        res = C._dedisperse_spec(*args)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_rank = e0.elapsed_time(e1) / steps
    n = len(res.dm_times)

    # untimed: one more call's phases one at a time (synchronised between phases),
    # through the same functions the call uses
    from astroflow_b200 import postprocess

    plan = next(reversed(C._PLANS.values()))[0]  # (plan, lock); no other thread uses it
    phases = {}

    def phase(name, f):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = f()
        torch.cuda.synchronize(dev)
        phases[name] = (time.perf_counter() - t0) * 1e3
        return r

    xd = phase("to_device_ms", lambda: C._to_device(x_host, dev))
    o = phase("run_ms", lambda: plan.run(xd))
    ds = wl["ds"]
    tsamp_out = float(f32(header.tsamp * f32(ds))) if ds > 1 else header.tsamp
    phase("images_ms", lambda: postprocess.device_slice_images(o, tsamp_out, 1, t_sample))
    return {"value": dist.job_rate(units, ms_rank * 1e-3), "unit": UNIT,
            "h2d_bytes_per_step": int(x_host.nbytes), "d2h_bytes_per_step": int(n * 512 * 512 * 3),
            "ms_per_step": dist.max(ms_rank), "images": n, "t_sample": t_sample,
            "api": "_astroflow_core._dedisperse_spec: host numpy chunk in, images out",
            "phases_one_call": phases}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the plan's default launch shape")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the short runs of the other workloads and of the reference GPU "
                         "arm that the default single-GPU run adds to its line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    wl = WORKLOADS[args.workload]

    import torch

    from astroflow_b200.synth import ChunkSpec, make_chunk_device

    from astroflow_b200.replicas import Replicas

    dist = Replicas("nccl", timeout_s=300.0)
    dev = dist.local
    torch.cuda.set_device(dev)
    if wl.get("kind") == "batch":
        bench_batch(args, wl, dist, dev)
        dist.close()
        return
    if wl.get("kind") == "multirange":
        bench_multirange(args, wl, dist, dev)
        dist.close()
        return
    if wl.get("kind") == "serve":
        bench_serve(args, wl, dist, dev)
        dist.close()
        return
    spec = ChunkSpec(nchans=wl["nchans"], nsamp=wl["nsamp"], nbits=wl["nbits"], seed=dist.chunk_seed(1234),
                     **wl["chunk"])
    hdr = spec.header()
    f32 = np.float32
    # the Header the reference's _dedisperse_spec path receives holds float fields
    hdr.update(tsamp=float(f32(hdr["tsamp"])), fch1=float(f32(hdr["fch1"])),
               foff=float(f32(hdr["foff"])), nsamp_total_s=float(f32(hdr["ndata"] * hdr["tsamp"] * 0.999)))
    config = {"workload": args.workload, "nchans": wl["nchans"], "nsamp": wl["nsamp"],
              "nbits": wl["nbits"], "dm_low": wl["dm"][0], "dm_high": wl["dm"][1],
              "dm_step": wl["dm"][2], "algorithm": wl["algorithm"],
              "subband_width": wl["subband_width"] if wl["algorithm"] == "subband" else None,
              "rfi": "iqrm(std, radius 5 lags, 3 sigma) + zero-DM (reference call-site semantics)"
                     if wl["rfi"] else "off",
              "l2": "inputs larger than L2 (chunk >> 126 MB), no flush between steps",
              "parallelism": f"replicas x{dist.world} (independent chunks, no exchange)"}

    if args.impl == "reference-gpu":
        reference_gpu_arm(args, wl, spec, hdr, config, dist, dev)
        return

    if args.impl == "reference":
        if dist.rank != 0:
            dist.close()
            return
        x, _ = make_chunk_device(spec, dev)
        x_host = x.cpu().numpy()
        del x
        from oracle import oracle as O

        if not O.ref_cpu_available():
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU build "
                              "oracle/_ref/libref_cpu.so is missing (build with make -C oracle ref)"}))
            return
        for _ in range(args.warmup):
            reference_cpu_rate(x_host, hdr, wl, target_s=1.0)
        rates, secs = [], []
        for _ in range(args.steps):
            r, threads, sample, dt = reference_cpu_rate(x_host, hdr, wl, target_s=4.0)
            rates.append(r)
            secs.append(dt)
        value = float(np.median(rates))
        full_ms = 1e3 * wl["nsamp"] * O.dm_steps(*wl["dm"]) / value
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * float(np.median(secs)),
                "full_workload_ms_extrapolated": full_ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                                 "kind": "reference", "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "note": "each step times one bounded sample (a DM subsample over the whole "
                        "chunk); ms_per_step is that sample's time, full_workload_ms_extrapolated "
                        "the full workload's time at the measured rate"}
        print(json.dumps(line))
        return

    # ------------------------------------------------------------ our arm
    from astroflow_b200.dedisp import measure_int_add_rate

    x, _ = make_chunk_device(spec, dev)
    plan = make_plan(wl, hdr, dev)
    out = plan.empty_output()
    stream = torch.cuda.current_stream(dev)
    units = plan.out_shape[0] * plan.out_shape[1]
    # launch shape chosen by the library's autotuner on this chunk (untimed; results
    # do not depend on it)
    tune = plan.autotune(x, out, reps=1, stream=stream) if (
        args.autotune and wl["algorithm"] == "subband") else None
    for _ in range(args.warmup):
        plan.run(x, out)
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)
    dist.barrier()
    torch.cuda.synchronize(dev)
    from astroflow_b200 import _lib

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = _lib.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        plan.run(x, out, stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    launches = _lib.launch_count() - l0
    dist.barrier()
    clk = clocks.stop()
    ms_rank = e0.elapsed_time(e1) / args.steps
    value = dist.job_rate(units, ms_rank * 1e-3)
    ms = dist.max(ms_rank)

    # rows of the timed output, kept for the check against the reference build in the
    # cpu_baseline leg (every column, so every time tile is covered)
    check_rows = parity_rows(wl, plan) if wl["algorithm"] == "subband" else None
    ours_rows = None
    if check_rows is not None:
        ours_rows = out.index_select(0, torch.tensor(check_rows, device=out.device)).cpu()

    # per-stage breakdown: the profiled form of the run after the timed steps (its
    # stages run one after another; CUDA events on the run's stream)
    stats = [plan.run_profiled(x, out, stream) for _ in range(min(args.steps, 3))]
    st = {k: float(np.mean([s[k] for s in stats])) for k in ("total_ms", "prep_ms", "stage1_ms", "stage2_ms")}
    s1n, s2n = stats[0]["stage1_launches"], stats[0]["stage2_launches"]
    info = plan.info
    hbm_peak, peak_kind = roofline_peaks()
    add_peak = measure_int_add_rate(dev)
    bytes_per_unit = (wl["nsamp"] * wl["nchans"] * wl["nbits"] / 8 + units * 4) / units
    elem = wl["nbits"] // 8
    if wl["algorithm"] == "subband":
        tile = min(int(info["nsamp_binned"]), int(info["tile_samples"]))
        dch = info["chan_end"] - info["chan_start"] + 1
        # bytes of one subband sum: 16-bit for 8-bit samples in subbands of <= 64
        # channels, else the reference's accumulator type
        inter = 2 if (wl["nbits"] == 8 and wl["subband_width"] <= 64) else (8 if wl["nbits"] == 32 else 4)
        # stage 1 may also write a one-sample-shifted twin of its sums, which stage 2 reads
        inter *= max(1, int(info["subband_sum_copies"]))
        if st["stage1_ms"] >= st["stage2_ms"]:
            kname, kms, kn = "stage1", st["stage1_ms"], s1n
            adds_launch = info["ndm_nom"] * dch * tile
            # the tile's prepared input, read once, and its subband sums (and twin), written once
            kbytes = dch * tile * elem + info["ndm_nom"] * info["nsb"] * tile * inter
        else:
            kname, kms, kn = "stage2", st["stage2_ms"], s2n
            adds_launch = info["dm_steps"] * info["nsb"] * tile
            # the tile's subband sums (and twin), read once, and its DM-time output, written once
            kbytes = info["ndm_nom"] * info["nsb"] * tile * inter + info["dm_steps"] * tile * 4
        units_launch = info["dm_steps"] * tile
    else:
        kname, kms, kn = "brute", st["stage2_ms"], s2n
        units_launch = units / max(kn, 1)
        adds_launch = info["adds_per_run"] / max(kn, 1)
        kbytes = (wl["nsamp"] * (info["chan_end"] - info["chan_start"]) * elem + units * 4) / max(kn, 1)
    avg_launch_s = kms / max(kn, 1) * 1e-3
    achieved = units_launch * bytes_per_unit / avg_launch_s / 1e9
    adds_rate = adds_launch / avg_launch_s
    step_adds = info["adds_per_run"] / (st["total_ms"] * 1e-3)
    roof_time = max(units * bytes_per_unit / (hbm_peak * 1e9), info["adds_per_run"] / add_peak)
    roofline = {
        "bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
        "frac": achieved / hbm_peak, "peak_kind": peak_kind,
        "traffic": ncu_traffic(kname, units_launch),
        "bytes_per_unit": bytes_per_unit, "units_per_launch": units_launch,
        "avg_launch_ms": avg_launch_s * 1e3,
        # the dominant kernel's own algorithmic bytes (its inputs read once, its
        # outputs written once) against its launch time: compare with `traffic`
        "kernel_bytes_per_launch": kbytes, "kernel_achieved": kbytes / avg_launch_s / 1e9,
        "kernel_frac": kbytes / avg_launch_s / 1e9 / hbm_peak,
        "int_add": {"achieved": adds_rate, "peak": add_peak, "unit": "adds/s",
                    "frac": adds_rate / add_peak, "peak_kind": "measured live (IADD3 probe)"},
        "binding": "int_add" if info["adds_per_run"] / add_peak > units * bytes_per_unit / (hbm_peak * 1e9) else "hbm",
        "step_frac": roof_time / (st["total_ms"] * 1e-3),
        "step_adds_per_s": step_adds,
        "stages_ms": st,
    }

    # e2e: same metric through the C ABI with host buffers (pinned), copies in the timed region
    e2e, same = None, None
    if args.e2e_steps > 0:
        e2e, same = e2e_run(plan, x, out, units, dist, dev, stream, args.e2e_steps, args.warmup)

    # and through the drop-in call (its own plan and output; ours released first)
    e2e_dropin = None
    if args.e2e_steps > 0 and wl["algorithm"] == "subband":
        del out
        plan.close()
        torch.cuda.empty_cache()
        e2e_dropin = e2e_dropin_run(wl, hdr, x, units, dist, dev, args.e2e_steps, args.warmup)

    cpu = None
    parity = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        x_host = x.cpu().numpy() if x.dtype == torch.uint8 else x.view(torch.int16).cpu().numpy().view(np.uint16)
        if O.ref_cpu_available():
            rate, threads, sample, dt = reference_cpu_rate(x_host, hdr, wl, target_s=12.0)
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": sample, "seconds": dt}
        if check_rows is not None:
            parity = reference_parity(x_host, hdr, wl, check_rows, ours_rows, dev)
        del x_host
    dist.barrier()
    extras = None
    if dist.rank == 0 and dist.world == 1 and args.extras and args.workload == DEFAULT_WORKLOAD:
        # release the headline's device buffers: the children need the GPU's memory
        if not plan.closed:
            plan.close()
        out = x = None
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
        extras = run_extras(dev)
    if dist.rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": f"u{wl['nbits']}", "data": "synthetic (seeded, generated on the GPU)",
                "config": config, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "e2e_dropin": e2e_dropin, "gpu_launches": launches, "clocks": clk,
                "autotune": tune,
                "host_path_matches_device": same,
                "parity_vs_reference": None if parity is None else parity["ok"],
                "parity_vs_reference_detail": parity,
                "extras": extras}
        print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
