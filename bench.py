#!/usr/bin/env python3
"""Benchmark: G uvw x pixel terms/s of visibility generation + imaging adjoint.

Workload (one "step"): the headline configuration -- HEALPix Nside 256
(786,432 pixels), 10 satellites = 45 baselines x 8,640 snapshots = 388,800
samples at 10 MHz, Moon occultation (ray-sphere) plus an Earth cap, i.e. one
forward pass V = A(I), the shell-histogram DCF and weights, and one imaging
adjoint pass, split precision.  Terms per step = 2 x 388,800 x 786,432.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Beside the headline, the line carries "formation_mode": the same step through
the formation entry points (viss_plan_set_formation: the samples given as the
satellites' vectors, S exponentials per pixel and snapshot instead of one per
sample), with its own roofline (FP32 FMA issue) and its rel-L2 against the
direct kernels.  --formation makes that the whole run.

N > 1 runs under torchrun: every rank is an independent replica (its own
observation day, no data-path collective; weak scaling), timed on the device
and reduced as the max over ranks.  --impl reference times the FP64 CPU
restatement of the reference's kernels (the reference has no CPU path) on the
host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

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

WORKLOAD = "c3_10mhz"
WORKLOAD_TEXT = {
    "c3_10mhz": "Nside 256 (786,432 px) x 388,800 uvw samples (45 baselines x 8,640 snapshots), "
                "10 MHz, Moon + Earth occultation",
    "c3_1mhz": "Nside 256 (786,432 px) x 388,800 uvw samples (45 baselines x 8,640 snapshots), "
               "1 MHz, Moon + Earth occultation",
    "prod_1mhz": "production operating point at 1 MHz: Nside 512 (3,145,728 px) x 2,000,160 uvw samples "
                 "(45 baselines x 44,448 snapshots, one day's 4,000,320 rows with the mirror rows folded), "
                 "Moon + Earth occultation",
    "c2": "Nside 64 (49,152 px) x 20,160 uvw samples (28 baselines x 720 snapshots), 10 MHz, "
          "Moon occultation (profiling-size case)",
    "c3_small": "Nside 256 (786,432 px) x 48,600 uvw samples (45 baselines x 1,080 snapshots), "
                "10 MHz, Moon + Earth occultation (profiling-size case of the headline workload)",
    "c3_small_1mhz": "Nside 256 (786,432 px) x 48,600 uvw samples (45 baselines x 1,080 snapshots), "
                     "1 MHz, Moon + Earth occultation (profiling-size case of the gridded adjoint)",
    "c4": "batched: Nside 128 (196,608 px) x 64 channels (1-10 MHz) x 129,600 uvw samples "
          "(45 baselines x 2,880 snapshots), Moon + Earth occultation, spectral index per pixel",
    "c5": "reconstruction: Nside 128 (196,608 px) x 194,400 uvw samples (45 baselines x 4,320 "
          "snapshots), 10 MHz, Moon occultation, SNR 20, positions perturbed N(0, 5 m); 200 L-BFGS steps",
    "c1": "Nside 32 (12,288 px) x 10,080 uvw samples (28 baselines x 360 snapshots), 1 MHz, "
          "no occultation",
    "stream": "day files end to end: Nside 256 (786,432 px) x 388,800 uvw samples + 388,800 mirror "
              "rows per day, 10 MHz, Moon occultation in both passes; text drop-in vs binary streaming loop",
}
METRIC = "G uvw x pixel terms/s (vis-gen + adjoint), split precision, rel-L2<=1e-5 vs FP64"
UNIT = "Gterms/s"
MUFU_TERMS_PER_CLK_PER_SM = 8     # 16 MUFU results/clk/SM, sin + cos per term
KERNEL_SOURCES = os.path.join(ROOT, "viss_optimize_3d_b200", "csrc")
TRAFFIC_RECORD = os.path.join(ROOT, "viss_optimize_3d_b200", "ncu_traffic.json")
# workloads too large for the launch-shape sweep, the FP64 comparison and the
# formation comparison in a bench run of a few minutes
BIG_WORKLOADS = ("prod_1mhz",)


# the translation units of the kernels a traffic record measures (k_forward,
# k_adjoint, k_form_forward, k_form_adjoint) and every header they include
TRAFFIC_KERNEL_SOURCES = ("formation.cu", "visibility.cu", "visibility.cuh", "viss_common.cuh")


def kernel_sources_sha() -> str:
    """sha256 over the CUDA sources of the recorded kernels (csrc/ files in
    TRAFFIC_KERNEL_SOURCES, in name order): the key under which a measured
    DRAM traffic record is valid.  Other sources (the gridded adjoint, the
    HEALPix and staging kernels) do not enter these kernels' code."""
    import hashlib
    h = hashlib.sha256()
    for name in sorted(TRAFFIC_KERNEL_SOURCES):
        h.update(name.encode())
        with open(os.path.join(KERNEL_SOURCES, name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


FWD_INSTANCES = ["k_forward<256, 4, 2, {m}, 0>", "k_forward<256, 4, 3, {m}, 0>",
                 "k_forward<256, 2, 3, {m}, 0>", "k_forward<256, 2, 4, {m}, 0>"]
ADJ_INSTANCES = ["k_adjoint<128, 8, 4, {m}, 0, 0>", "k_adjoint<128, 8, 5, {m}, 0, 0>",
                 "k_adjoint<128, 4, 5, {m}, 0, 0>", "k_adjoint<128, 4, 6, {m}, 0, 0>"]


def measured_traffic(workload: str, kernel: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    of the kernel instance `kernel` (e.g. "k_adjoint<128, 8, 4, 1, 0, 0>", the
    launch shape the run used) on `workload`, from an ncu capture recorded by
    `bench.py --record-traffic`, or None when no capture of the current
    kernel sources exists (a record of other sources is never reported)."""
    try:
        with open(TRAFFIC_RECORD) as f:
            rec = json.load(f)
    except Exception:
        return None, "no ncu traffic record"
    if rec.get("kernel_sources_sha256") != kernel_sources_sha():
        return None, "the ncu traffic record is of other kernel sources"
    v = rec.get("bytes_per_launch", {}).get(workload, {}).get(kernel)
    if v is None:
        return None, f"no ncu traffic record of {kernel} on {workload}"
    cap = rec.get("captures", {}).get(workload, {})
    return v, f"ncu capture of these kernel sources (git {cap.get('git_commit', '?')}): {cap.get('command', '')}"


def record_traffic(csv_path: str, workload: str, command: str, commit: str = ""):
    """Write the DRAM traffic per launch of each kernel in an ncu --csv
    metrics log (dram__bytes_read.sum, dram__bytes_write.sum) into the traffic
    record, keyed by the current kernel sources' sha256."""
    import csv
    import re
    per = {}
    with open(csv_path) as f:
        lines = [ln for ln in f if ln.startswith('"')]
    for row in csv.DictReader(lines):
        name = row.get("Kernel Name", "")
        metric, val = row.get("Metric Name"), row.get("Metric Value", "").replace(",", "")
        if metric not in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            continue
        unit = row.get("Metric Unit", "byte")
        scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}.get(unit, 1)
        m = re.search(r"\b((?:k_form_forward|k_form_adjoint|k_forward|k_adjoint)<[^>]*>)", name)
        if m:
            k = m.group(1)     # the template instance, e.g. k_adjoint<128, 8, 4, 1, 0, 0>
            per.setdefault(k, {}).setdefault(row.get("ID"), 0.0)
            per[k][row.get("ID")] += float(val) * scale
    try:
        with open(TRAFFIC_RECORD) as f:
            rec = json.load(f)
    except Exception:
        rec = {}
    sha = kernel_sources_sha()
    if rec.get("kernel_sources_sha256") != sha:
        rec = {"kernel_sources_sha256": sha, "bytes_per_launch": {}}
    try:
        git = commit or subprocess.run(["git", "rev-parse", "--short", "HEAD"], cwd=ROOT,
                                       capture_output=True, text=True).stdout.strip() or "?"
    except Exception:
        git = "?"
    rec.setdefault("captures", {})[workload] = {"git_commit": git, "command": command}
    # per template instance (launch shape), the median over its launches
    rec["bytes_per_launch"][workload] = {k: int(statistics.median(v.values())) for k, v in per.items()}
    with open(TRAFFIC_RECORD, "w") as f:
        json.dump(rec, f, indent=1)
    return rec


def bench_config(args, J: int, K: int, world: int) -> dict:
    """The workload description both arms print (identical keys and values)."""
    return {"workload": WORKLOAD_TEXT.get(args.workload, args.workload)
                        + ("; formation mode" if getattr(args, "formation", False) else ""),
            "pixels": J, "samples": K, "terms_per_step": 2 * K * J,
            "l2": "GPU arm: flushed between timed steps (256 MB write)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def workload_config(name: str):
    from viss_optimize_3d_b200 import synth
    if name == "c3_small":
        return synth.scaled(synth.CONFIGS["c3_10mhz"], n_snap=1080)
    if name == "c3_small_1mhz":
        return synth.scaled(synth.CONFIGS["c3_1mhz"], n_snap=1080)
    return synth.CONFIGS[name]


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f), "measured"
    except Exception:
        return {"sm_max_mhz": 1965.0, "hbm_gbs": 6650.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
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
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    from viss_optimize_3d_b200 import api, pipeline, replicas, synth
    from viss_optimize_3d_b200._capi import check, lib
    import ctypes as C

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    if args.formation:
        return run_formation(args, rank, world, local_rank)
    cfg = workload_config(args.workload)
    if world > 1:
        import dataclasses
        # one observation day per replica, the reference's round-robin day split
        day = replicas.days_for_rank(world, rank, world)[0]
        cfg = dataclasses.replace(cfg, day=float(day - 1))
    f_hz = cfg.freqs_hz[0]
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, f_hz, device=dev)
    K, J = g.plan.K, g.plan.J
    terms_per_step = 2 * K * J
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2
    big = args.workload in BIG_WORKLOADS

    # device-resident step: forward, DCF + weights, adjoint
    def step():
        V = g.plan.forward(g.sky)
        return pipeline.dirty_image(g, V)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    V0 = g.plan.forward(g.sky)
    gs0, _c0, dcf0 = api.dcf(g.bll, g.nr, multiplicity=2)
    coef0 = api.scale_coef(api.weights(g.w, g.bll, gs0, dcf0, g.nr)[1], V0)
    sweep = {"forward_ms": [], "adjoint_ms": []}
    if big:
        # the shapes the tuner picks at the headline size; a sweep here would
        # take longer than the timed run
        g.plan.set_shapes(0, 0)
        shapes = (0, 0)
    else:
        # launch-shape sweep (recorded) and the plan's own tuner (chooses)
        for shape in range(4):
            g.plan.set_shapes(shape, shape)
            for key, fn in (("forward_ms", lambda: g.plan.forward(g.sky)),
                            ("adjoint_ms", lambda: g.plan.adjoint(coef0, scale=2.0, mask=cfg.imaging_mask))):
                fn()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                sweep[key].append(round(e0.elapsed_time(e1), 3))
        shapes = g.plan.tune(g.sky, coef0, mask=cfg.imaging_mask)
    torch.cuda.synchronize()
    fwd_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    adj_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    step_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
    # this rank's day images summed on the device (FP64, non-finite as 0), and
    # over the ranks by one NCCL all-reduce at the end of the timed region:
    # the day-summed image of the reference's notebooks, replacing its
    # round-robin days with a host sum (vissgen3d_blockage.cu:271-279)
    day_sum = torch.zeros(J, dtype=torch.float64, device=dev)
    clocks = ClockSampler(local_rank)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        flush.fill_(float(i))                                  # evict L2 between steps
        step_ev[i][0].record(stream)
        fwd_ev[i][0].record(stream)
        V = g.plan.forward(g.sky)
        fwd_ev[i][1].record(stream)
        gs, _c, dcf = api.dcf(g.bll, g.nr, multiplicity=2)
        _dg, wt = api.weights(g.w, g.bll, gs, dcf, g.nr)
        coef = api.scale_coef(wt, V)
        adj_ev[i][0].record(stream)
        img = g.plan.adjoint(coef, scale=2.0, mask=cfg.imaging_mask)
        adj_ev[i][1].record(stream)
        replicas.add_day_image(day_sum, img)
        if i == args.steps - 1:
            replicas.sum_images(day_sum)
        step_ev[i][1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        torch.distributed.barrier()
    step_ms = [a.elapsed_time(b) for a, b in step_ev]
    fwd_ms = [a.elapsed_time(b) for a, b in fwd_ev]
    adj_ms = [a.elapsed_time(b) for a, b in adj_ev]
    total_s = sum(step_ms) / 1e3
    # culled fraction of the last forward/adjoint (device counters); also
    # raises if a bounded device-side wait gave up in either kernel
    g.plan.forward(g.sky)
    ev_f, mx_f, tot = g.plan.last_stats()
    g.plan.adjoint(coef, scale=2.0, mask=cfg.imaging_mask)
    ev_a, mx_a, _ = g.plan.last_stats()
    day_sum_ok = bool(torch.isfinite(day_sum).all().item())

    # end to end through the public API from pinned host buffers: every step
    # uploads a new observation's inputs (sky, uvw, satellite positions, the
    # Earth rows, occulter refs), builds the occulter rows on the device
    # (viss_occulters), stages the samples, runs forward + DCF + adjoint and
    # reads V and the image back
    sky_h = torch.from_numpy(obs.sky_at(f_hz).astype(np.float32) * np.float32(4 * math.pi / J)).pin_memory()
    uvw_h = torch.from_numpy(obs.uvw(f_hz)).pin_memory()
    masked = obs.refs is not None
    refs_h = torch.from_numpy(obs.refs).pin_memory() if masked else None
    P_h = torch.from_numpy(np.ascontiguousarray(obs.occ_sat_positions)).pin_memory() if masked else None
    earth_h = (torch.from_numpy(np.ascontiguousarray(obs.earth_rows)).pin_memory()
               if masked and obs.earth_rows is not None else None)
    img_h = torch.empty(J, dtype=torch.float32).pin_memory()
    V_h = torch.empty(K, dtype=torch.complex64).pin_memory()
    sky_d = torch.empty_like(g.sky)
    uvw_d = torch.empty_like(g.uvw)
    refs_d = torch.empty_like(g.refs) if masked else None
    P_d = torch.empty(P_h.shape, dtype=torch.float64, device=dev) if masked else None
    occ_d = torch.empty_like(g.occ) if masked else None
    n_sat_rows = P_h.shape[0] if masked else 0

    def e2e_step():
        sky_d.copy_(sky_h, non_blocking=True)
        uvw_d.copy_(uvw_h, non_blocking=True)
        st = C.c_void_p(stream.cuda_stream)
        if masked:
            refs_d.copy_(refs_h, non_blocking=True)
            P_d.copy_(P_h, non_blocking=True)
            check(lib.viss_occulters(n_sat_rows, C.c_void_p(P_d.data_ptr()), synth.R_MOON, 0, 0.0,
                                     C.c_void_p(occ_d.data_ptr()), st), "viss_occulters")
            if earth_h is not None:
                occ_d[n_sat_rows:].copy_(earth_h, non_blocking=True)
        check(lib.viss_plan_set_samples(g.plan._h, K, C.c_void_p(uvw_d.data_ptr()), None,
                                        C.c_void_p(refs_d.data_ptr()) if masked else None,
                                        occ_d.shape[0] if masked else 0,
                                        C.c_void_p(occ_d.data_ptr()) if masked else None, st),
              "set_samples")
        Vd = g.plan.forward(sky_d)
        imgd = pipeline.dirty_image(g, Vd)
        V_h.copy_(Vd, non_blocking=True)
        img_h.copy_(imgd, non_blocking=True)

    e2e_steps = 1 if big else max(1, min(args.steps, 3))
    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = e0.elapsed_time(e1) / 1e3
    h2d = J * 4 + K * 24
    if masked:
        h2d += K * 12 + P_h.numel() * 8 + (earth_h.numel() * 8 if earth_h is not None else 0)
    d2h = J * 4 + K * 8

    # max over ranks (device-timed seconds)
    total_s, e2e_s = replicas.max_over_ranks([total_s, e2e_s], device=dev)
    if rank != 0:
        return None

    # the plain FP64 path on the same step (the split path's >= 3x target):
    # one warm-up, then the mean of three timed repeats
    fp64 = None
    if args.fp64_compare and not big:
        reps = 3
        g.plan.forward(g.sky, fp64=True)
        g.plan.adjoint(coef, scale=2.0, mask=cfg.imaging_mask, fp64=True)
        torch.cuda.synchronize()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(reps)]
        for r in range(reps):
            flush.fill_(float(r))
            ev[r][0].record(stream)
            Vd = g.plan.forward(g.sky, fp64=True)
            ev[r][1].record(stream)
            g.plan.adjoint(coef, scale=2.0, mask=cfg.imaging_mask, fp64=True)
            ev[r][2].record(stream)
        torch.cuda.synchronize()
        g.plan.last_stats()
        fp64_fwd = statistics.mean(e[0].elapsed_time(e[1]) for e in ev) / 1e3
        fp64_adj = statistics.mean(e[1].elapsed_time(e[2]) for e in ev) / 1e3
        split_fwd, split_adj = statistics.mean(fwd_ms) / 1e3, statistics.mean(adj_ms) / 1e3
        Vs = g.plan.forward(g.sky).to(torch.complex128)
        rel = (torch.linalg.norm(Vs - Vd.to(torch.complex128)) / torch.linalg.norm(Vd.to(torch.complex128))).item()
        fp64 = {"value": round(terms_per_step / (fp64_fwd + fp64_adj) / 1e9, 3), "unit": UNIT,
                "forward_ms": round(fp64_fwd * 1e3, 2), "adjoint_ms": round(fp64_adj * 1e3, 2),
                "timed_repeats": reps, "warmup": 1,
                "split_speedup": round((fp64_fwd + fp64_adj) / (split_fwd + split_adj), 2),
                "forward_rel_l2_split_vs_fp64": float(f"{rel:.3e}")}

    pk, pk_kind = peaks()
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_terms = MUFU_TERMS_PER_CLK_PER_SM * nsm * pk["sm_max_mhz"] * 1e6
    fwd_s = statistics.mean(fwd_ms) / 1e3
    adj_s = statistics.mean(adj_ms) / 1e3
    dom = "forward" if fwd_s >= adj_s else "adjoint"
    dom_s = max(fwd_s, adj_s)
    dom_eval = (ev_f if dom == "forward" else ev_a)
    achieved = K * J / dom_s
    value = terms_per_step * args.steps * world / total_s / 1e9
    G = g.occ.shape[0] if g.occ is not None else 0
    # algorithmic bytes of one launch: each input record read once, each
    # output written once (pixel records 32 B, sample records 32 B + refs
    # 16 B, occulter rows 32 B + 16 B, V 8 B / coefficients 8 B, image 4 B)
    alg_bytes = {"forward": J * 32 + K * 48 + G * 48 + K * 8,
                 "adjoint": J * 32 + K * 48 + G * 48 + K * 8 + J * 4}[dom]
    masked = 1 if obs.refs is not None else 0
    inst = (FWD_INSTANCES[shapes[0]] if dom == "forward" else ADJ_INSTANCES[shapes[1]]).format(m=masked)
    traffic, traffic_src = measured_traffic(args.workload, inst)
    res = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_s / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64-phase/f32-sincos",
        "data": "synthetic (seeded lunar-orbit formation and log-normal sky, see synth.py)",
        "config": bench_config(args, J, K, world),
        "e2e": {"value": round(terms_per_step * e2e_steps / e2e_s / 1e9 * world, 3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "pinned host sky/uvw/refs/satellite positions/Earth rows -> viss_occulters -> "
                        "viss_plan_set_samples -> viss_forward -> viss_dcf/viss_weights -> viss_adjoint "
                        "-> pinned host V/image"},
        "roofline": {"bound": "sfu", "kernel": f"k_{dom}",
                     "achieved": round(achieved / 1e9, 2), "peak": round(peak_terms / 1e9, 1),
                     "unit": "Gterms/s", "frac": round(achieved / peak_terms, 4),
                     "peak_source": f"8 terms/clk/SM x {nsm} SMs x sm_max_mhz ({pk_kind})",
                     "evaluated_frac": round(dom_eval / (K * J), 4),
                     "frac_of_evaluated": round(dom_eval / dom_s / peak_terms, 4),
                     "algorithmic_bytes": alg_bytes,
                     "traffic": traffic, "traffic_unit": "DRAM bytes per launch",
                     "traffic_source": traffic_src, "instance": inst},
        "kernel_ms": {"forward": round(fwd_s * 1e3, 3), "adjoint": round(adj_s * 1e3, 3)},
        "culling": {"forward_evaluated": round(ev_f / tot, 4), "forward_mixed": round(mx_f / tot, 4),
                    "adjoint_evaluated": round(ev_a / tot, 4), "adjoint_mixed": round(mx_a / tot, 4)},
        "day_sum": {"ranks": world, "reduction": "NCCL all-reduce (SUM) of the FP64 day sums"
                    if world > 1 else "single rank: device day sum only", "finite": day_sum_ok},
        "gpu_launches": 11 * args.steps,
        "fp64_path": fp64,
        "tuning": {"chosen": {"forward": shapes[0], "adjoint": shapes[1]},
                   "forward_shapes": "(samples/thread, CTAs/SM) = (4,2) (4,3) (2,3) (2,4)",
                   "adjoint_shapes": "(pixels/lane, CTAs/SM), 128-thread CTAs = (8,4) (8,5) (4,5) (4,6)",
                   **({"note": "fixed at the headline size's choice (no sweep at this size)"} if big else sweep)},
        "clocks": clk,
    }
    if args.cpu_baseline:
        res["cpu_baseline"] = cpu_baseline(obs, f_hz, budget_s=args.cpu_seconds)
    return res


# ------------------------------------------------------ formation mode
FORM_FFMA_PER_TERM = 4   # one complex multiply-accumulate G_a conj(F_b) per (pair, pixel)


def run_formation(args, rank, world, local_rank):
    """The same step through the formation entry points: the samples given as
    satellite vectors U (T x S x 3), S exponentials per pixel and snapshot,
    the S(S-1)/2 pair sums as FP32 complex multiply-accumulates."""
    import numpy as np
    import torch
    from viss_optimize_3d_b200 import api, pipeline, replicas, synth
    from viss_optimize_3d_b200._capi import check, lib
    import ctypes as C

    dev = torch.device("cuda", local_rank)
    if args.workload in ("c1", "c2", "c3_10mhz", "c3_1mhz", "c3_small", "prod_1mhz"):
        cfg = workload_config(args.workload)
    else:
        raise SystemExit(f"--formation covers the single-channel workloads, not {args.workload}")
    if world > 1:
        import dataclasses
        day = replicas.days_for_rank(world, rank, world)[0]
        cfg = dataclasses.replace(cfg, day=float(day - 1))
    f_hz = cfg.freqs_hz[0]
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, f_hz, device=dev)
    U, occ_sat, occ_snap = pipeline.formation_inputs(obs, f_hz, device=dev, occ=g.occ)
    plan = g.plan
    plan.set_formation(U, None, occ_sat, occ_snap)
    K, J = plan.form_T * plan.form_B, plan.J
    terms_per_step = 2 * K * J
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def image(V):
        gs, _c, dcf = api.dcf(g.bll, g.nr, multiplicity=2)
        _dg, wt = api.weights(g.w, g.bll, gs, dcf, g.nr)
        return plan.adjoint_formation(api.scale_coef(wt, V), scale=2.0, mask=cfg.imaging_mask)

    for _ in range(args.warmup):
        image(plan.forward_formation(g.sky))
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        flush.fill_(float(i))
        ev[i][0].record(stream)
        V = plan.forward_formation(g.sky)
        ev[i][1].record(stream)
        gs, _c, dcf = api.dcf(g.bll, g.nr, multiplicity=2)
        _dg, wt = api.weights(g.w, g.bll, gs, dcf, g.nr)
        coef = api.scale_coef(wt, V)
        ev[i][2].record(stream)
        plan.adjoint_formation(coef, scale=2.0, mask=cfg.imaging_mask)
        ev[i][3].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        torch.distributed.barrier()
    total_s = sum(e[0].elapsed_time(e[3]) for e in ev) / 1e3
    fwd_s = statistics.mean(e[0].elapsed_time(e[1]) for e in ev) / 1e3
    adj_s = statistics.mean(e[2].elapsed_time(e[3]) for e in ev) / 1e3
    plan.forward_formation(g.sky)
    ev_f, mx_f, tot = plan.last_stats()
    plan.adjoint_formation(coef, scale=2.0, mask=cfg.imaging_mask)
    ev_a, mx_a, _ = plan.last_stats()
    # parity of this step against the direct kernels on the same plan
    Vd = plan.forward(g.sky).to(torch.complex128)
    Vf = plan.forward_formation(g.sky).to(torch.complex128)
    rel_v = (torch.linalg.norm(Vf - Vd) / torch.linalg.norm(Vd)).item()

    # end to end: every step uploads a new observation's inputs from pinned
    # host memory (sky, satellite positions, the Earth rows), forms the
    # satellite vectors U = (P - centre) / lambda and the Moon occulter rows
    # (viss_occulters) on the device, stages the formation, runs forward +
    # DCF + adjoint and reads V and the image back
    sky_h = torch.from_numpy(obs.sky_at(f_hz).astype(np.float32) * np.float32(4 * math.pi / J)).pin_memory()
    P_h = torch.from_numpy(np.ascontiguousarray(obs.positions, dtype=np.float64)).pin_memory()
    earth_h = torch.from_numpy(np.ascontiguousarray(obs.earth_rows)).pin_memory() if occ_snap is not None else None
    P_d, sky_d = torch.empty(P_h.shape, dtype=torch.float64, device=dev), torch.empty_like(g.sky)
    osat_d = torch.empty_like(occ_sat) if occ_sat is not None else None
    osnap_d = torch.empty_like(occ_snap) if occ_snap is not None else None
    img_h = torch.empty(J, dtype=torch.float32).pin_memory()
    V_h = torch.empty(K, dtype=torch.complex64).pin_memory()
    lam = synth.C_LIGHT / f_hz

    def e2e_step():
        st = C.c_void_p(stream.cuda_stream)
        sky_d.copy_(sky_h, non_blocking=True)
        P_d.copy_(P_h, non_blocking=True)
        U_d = ((P_d - P_d.mean(dim=1, keepdim=True)) / lam).contiguous()
        if osat_d is not None:
            check(lib.viss_occulters(P_d.shape[0] * P_d.shape[1], C.c_void_p(P_d.data_ptr()), synth.R_MOON,
                                     0, 0.0, C.c_void_p(osat_d.data_ptr()), st), "viss_occulters")
        if osnap_d is not None:
            osnap_d.copy_(earth_h, non_blocking=True)
        check(lib.viss_plan_set_formation(plan._h, plan.form_T, plan.form_S, C.c_void_p(U_d.data_ptr()),
                                          None, None if osat_d is None else C.c_void_p(osat_d.data_ptr()),
                                          None if osnap_d is None else C.c_void_p(osnap_d.data_ptr()), st),
              "viss_plan_set_formation")
        Vd_ = plan.forward_formation(sky_d)
        imgd = image(Vd_)
        V_h.copy_(Vd_, non_blocking=True)
        img_h.copy_(imgd, non_blocking=True)

    e2e_steps = 1 if args.workload in BIG_WORKLOADS else max(1, min(args.steps, 3))
    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = e0.elapsed_time(e1) / 1e3
    h2d = J * 4 + P_h.numel() * 8 + (earth_h.numel() * 8 if earth_h is not None else 0)
    total_s, e2e_s = replicas.max_over_ranks([total_s, e2e_s], device=dev)
    if rank != 0:
        return None
    traffic, traffic_src = measured_traffic(
        args.workload, f"k_form_{'forward' if fwd_s >= adj_s else 'adjoint'}<{plan.form_S}>")
    pk, pk_kind = peaks()
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_terms = 128 / FORM_FFMA_PER_TERM * nsm * pk["sm_max_mhz"] * 1e6
    dom = "forward" if fwd_s >= adj_s else "adjoint"
    dom_s = max(fwd_s, adj_s)
    dom_eval = ev_f if dom == "forward" else ev_a
    achieved = K * J / dom_s
    res = {
        "metric": METRIC,
        "value": round(terms_per_step * args.steps * world / total_s / 1e9, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_s / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64-phase/f32-sincos/f32-pair-products",
        "data": "synthetic (seeded lunar-orbit formation and log-normal sky, see synth.py)",
        "config": {**bench_config(args, J, K, world), "satellites": plan.form_S, "snapshots": plan.form_T},
        "e2e": {"value": round(terms_per_step * e2e_steps / e2e_s / 1e9 * world, 3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": J * 4 + K * 8,
                "path": "pinned host sky/satellite positions/Earth rows -> U and viss_occulters on the "
                        "device -> viss_plan_set_formation -> viss_forward_formation -> "
                        "viss_dcf/viss_weights -> viss_adjoint_formation -> pinned host V/image"},
        "roofline": {"bound": "fp32", "kernel": f"k_form_{dom}",
                     "achieved": round(achieved / 1e9, 2), "peak": round(peak_terms / 1e9, 1),
                     "unit": "Gterms/s", "frac": round(achieved / peak_terms, 4),
                     "peak_source": f"128 FP32 lanes/clk/SM / {FORM_FFMA_PER_TERM} FFMA per term x {nsm} SMs "
                                    f"x sm_max_mhz ({pk_kind})",
                     "evaluated_frac": round(dom_eval / (K * J), 4),
                     "traffic": traffic, "traffic_unit": "DRAM bytes per launch",
                     "traffic_source": traffic_src},
        "kernel_ms": {"forward": round(fwd_s * 1e3, 3), "adjoint": round(adj_s * 1e3, 3)},
        "culling": {"forward_evaluated": round(ev_f / tot, 4), "forward_general_path": round(mx_f / tot, 4),
                    "adjoint_evaluated": round(ev_a / tot, 4), "adjoint_general_path": round(mx_a / tot, 4)},
        "forward_rel_l2_vs_direct": float(f"{rel_v:.3e}"),
        "gpu_launches": 10 * args.steps,
        "clocks": clk,
    }
    return res


# ------------------------------------------------------- batched channels
def run_batched(args):
    """All channels in one launch per kernel (CUDA-graph replay) against one
    launch per channel, forward + adjoint."""
    import numpy as np
    import torch
    from viss_optimize_3d_b200 import api, pipeline, synth

    dev = torch.device("cuda", 0)
    cfg = synth.CONFIGS["c4"]
    obs = synth.make_observation(cfg)
    C, K, J = len(cfg.freqs_hz), cfg.n_samples, cfg.npix
    lmn = api.pix2lmn(cfg.nside, "ring", device=dev)
    occ = pipeline.build_occulters(obs, dev)
    refs = torch.as_tensor(obs.refs, device=dev)
    uvw = [torch.as_tensor(obs.uvw(f), device=dev) for f in cfg.freqs_hz]
    sky = torch.stack([torch.as_tensor(obs.sky_at(f) * 4 * math.pi / J, dtype=torch.float32, device=dev)
                       for f in cfg.freqs_hz])
    stream = torch.cuda.current_stream(dev)
    terms = 2 * C * K * J

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / steps

    batched = api.Plan(lmn, torch.cat(uvw), None, refs.repeat(C, 1), occ, channels=C)
    coef = batched.forward(sky)
    shapes = batched.tune(sky, coef)
    out_V = torch.empty(C * K, dtype=torch.complex64, device=dev)
    out_I = torch.empty((C, J), dtype=torch.float32, device=dev)

    def step_batched():
        batched.forward(sky, out=out_V)
        batched.adjoint(coef, out=out_I)

    t_batched = timed(step_batched, args.steps, args.warmup)
    graph = torch.cuda.CUDAGraph()
    step_batched()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        step_batched()
    t_graph = timed(graph.replay, args.steps, 1)

    singles = []
    for c in range(C):
        pl = api.Plan(lmn, uvw[c], None, refs, occ)
        pl.set_shapes(*shapes)
        singles.append(pl)
    outs = [(torch.empty(K, dtype=torch.complex64, device=dev), torch.empty(J, dtype=torch.float32, device=dev))
            for _ in range(C)]

    def step_per_channel():
        for c, pl in enumerate(singles):
            pl.forward(sky[c], out=outs[c][0])
            pl.adjoint(coef[c * K:(c + 1) * K], out=outs[c][1])

    t_single = timed(step_per_channel, max(1, args.steps // 2), 1)
    g2 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g2):
        step_per_channel()
    t_single_graph = timed(g2.replay, max(1, args.steps // 2), 1)
    ok = all(torch.allclose(out_I[c], outs[c][1], rtol=1e-4, atol=1e-5 * outs[c][1].abs().max().item())
             for c in range(C))
    del singles, outs
    form = None
    if args.formation_compare or args.formation:
        # the same channels through the formation entry points: U (C, T, S, 3),
        # one launch per kernel for all channels, graph replay
        U = torch.stack([pipeline.formation_inputs(obs, f, device=dev, occ=occ)[0] for f in cfg.freqs_hz])
        _u, occ_sat, occ_snap = pipeline.formation_inputs(obs, cfg.freqs_hz[0], device=dev, occ=occ)
        fplan = api.Plan(lmn)
        fplan.set_formation(U, None, occ_sat, occ_snap)
        fV = torch.empty(C * K, dtype=torch.complex64, device=dev)
        fI = torch.empty((C, J), dtype=torch.float32, device=dev)

        def step_formation():
            fplan.forward_formation(sky, out=fV)
            fplan.adjoint_formation(coef, out=fI)

        t_fstream = timed(step_formation, args.steps, args.warmup)
        fg = torch.cuda.CUDAGraph()
        step_formation()
        torch.cuda.synchronize()
        with torch.cuda.graph(fg):
            step_formation()
        t_fgraph = timed(fg.replay, args.steps, 1)
        rel_V = float(torch.linalg.norm((fV - out_V).to(torch.complex128)) / torch.linalg.norm(out_V.to(torch.complex128)))
        rel_I = float(torch.linalg.norm((fI - out_I).double()) / torch.linalg.norm(out_I.double()))
        form = {"value": round(terms / t_fgraph / 1e9, 3), "unit": UNIT, "graph_ms": round(t_fgraph * 1e3, 2),
                "stream_ms": round(t_fstream * 1e3, 2), "launches_per_step": 2,
                "V_rel_l2_vs_direct": float(f"{rel_V:.3e}"), "image_rel_l2_vs_direct": float(f"{rel_I:.3e}"),
                "entry_points": "viss_plan_set_formation (U: C x T x S x 3), viss_plan_set_formation_channels, "
                                "viss_forward_formation, viss_adjoint_formation"}
        del fg
    res = {
        "metric": METRIC, "value": round(terms / t_graph / 1e9, 3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_graph * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64-phase/f32-sincos", "data": "synthetic (seeded, see synth.py)",
        "config": {"workload": WORKLOAD_TEXT["c4"], "pixels": J, "samples_per_channel": K,
                   "channels": C, "terms_per_step": terms},
        "batched": {"graph_ms": round(t_graph * 1e3, 2), "stream_ms": round(t_batched * 1e3, 2),
                    "launches_per_step": 2, "shapes": list(shapes)},
        "per_channel": {"stream_ms": round(t_single * 1e3, 2), "graph_ms": round(t_single_graph * 1e3, 2),
                        "launches_per_step": 2 * C},
        "speedup_batched_graph_vs_per_channel": round(t_single / t_graph, 3),
        "images_agree": bool(ok),
    }
    if form is not None:
        res["formation_mode"] = form
    del graph, g2
    return res


# ------------------------------------------------------- reconstruction
def run_reconstruction(args):
    """Loss + gradient through the differentiable operator, gradient accuracy
    (split vs FP64), and 200 L-BFGS steps beside the DCF dirty image."""
    import torch
    from viss_optimize_3d_b200 import reconstruct, synth

    dev = torch.device("cuda", 0)
    cfg = synth.CONFIGS["c5"]
    p = reconstruct.make_problem(cfg, device=dev, seed=0, formation=args.formation)
    p64 = reconstruct.make_problem(cfg, device=dev, seed=0, fp64=True)
    stream = torch.cuda.current_stream(dev)
    K, J = cfg.n_samples, cfg.npix
    x = p.x_true * 0.9
    d = torch.zeros_like(p.delta_true)

    def evaluate(prob):
        xx = x.clone().requires_grad_(True)
        dd = d.clone().requires_grad_(True)
        L = reconstruct.loss(prob, xx, dd)
        L.backward()
        return xx.grad.double(), dd.grad.double()

    for _ in range(2):
        evaluate(p)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    gx, gd = evaluate(p)
    e1.record(stream)
    torch.cuda.synchronize()
    t_eval = e0.elapsed_time(e1) / 1e3
    gx64, gd64 = evaluate(p64)
    dirty = reconstruct.dirty_image(p)
    torch.cuda.synchronize()
    e0.record(stream)
    xr, dr, hist = reconstruct.reconstruct(p, iters=200)
    e1.record(stream)
    torch.cuda.synchronize()
    t_lbfgs = e0.elapsed_time(e1) / 1e3
    c = lambda t: t - t.mean(dim=0, keepdim=True)
    # one evaluation = forward + adjoint + 3-channel phase-derivative forward
    terms_eval = 5 * K * J
    return {
        "metric": METRIC, "value": round(terms_eval / t_eval / 1e9, 3), "unit": UNIT, "n_gpus": 1,
        "steps": 1, "warmup": 2, "ms_per_step": round(t_eval * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64-phase/f32-sincos",
        "data": "synthetic (seeded, see synth.py)",
        "config": {"workload": WORKLOAD_TEXT["c5"] + ("; formation mode" if args.formation else ""),
                   "pixels": J, "samples": K, "terms_per_evaluation": terms_eval,
                   "operator": "FormationModel (viss_*_formation)" if args.formation
                               else "VisibilityModel (viss_forward / viss_adjoint)"},
        "gradient": {"sky_rel_err_split_vs_fp64": float(f"{float((gx - gx64).norm() / gx64.norm()):.3e}"),
                     "positions_rel_err_split_vs_fp64": float(f"{float((gd - gd64).norm() / gd64.norm()):.3e}")},
        "lbfgs": {"iterations": 200, "evaluations": len(hist), "seconds": round(t_lbfgs, 2),
                  "loss_first": float(f"{hist[0]:.4e}"), "loss_last": float(f"{hist[-1]:.4e}"),
                  "chi2_per_dof_last": round(hist[-1] / (2 * K), 3),
                  "image_rel_l2": round(reconstruct.rel_l2(xr, p.x_true), 4),
                  "dirty_image_rel_l2": round(reconstruct.rel_l2(dirty, p.x_true), 4),
                  "position_error_m_before": round(float(c(p.delta_true).norm()), 3),
                  "position_error_m_after": round(float((c(dr) - c(p.delta_true)).norm()), 3)},
    }


# ---------------------------------------------------------- CPU baseline
class CpuSampler:
    """The FP64 CPU restatement (oracle/) on all host cores, timed on bounded
    samples of a workload: n_f samples x all pixels (forward) and n_a pixels
    x all samples (adjoint), sized from a calibrated rate to a time budget."""

    def __init__(self, obs, f_hz):
        import numpy as np
        from oracle import oracle as O

        O.build()
        self.O = O
        self.cores = O.max_threads()
        _, _, xyz = O.pix2ang(obs.cfg.nside)
        self.lmn = O.lmn_from_xyz(xyz)
        self.uvw = obs.uvw(f_hz)
        self.sky = obs.sky_at(f_hz) * (4 * math.pi / obs.cfg.npix)
        self.refs, self.occ = obs.refs, None
        if self.refs is not None:
            self.occ = O.occulters(obs.occ_sat_positions, 1737.4e3, 0)
            if obs.earth_rows is not None:
                self.occ = np.concatenate([self.occ, obs.earth_rows])
        self.K, self.J = self.uvw.shape[0], self.lmn.shape[0]
        # calibrate on slices that grow until one takes >= 0.5 s (a tiny slice
        # measures thread start-up more than the sum)
        n_cal = self.cores
        while True:
            t0 = time.perf_counter()
            O.forward(self.uvw[:n_cal], self.lmn, self.sky, self._sel(slice(0, n_cal)), self.occ,
                      nthreads=self.cores)
            dt = time.perf_counter() - t0
            if dt >= 0.5 or n_cal >= self.K:
                break
            n_cal = min(self.K, n_cal * 4)
        self.rate = n_cal * self.J / max(dt, 1e-6)            # terms/s

    def _sel(self, idx):
        return None if self.refs is None else self.refs[idx]

    def sample(self, budget_s: float, seed: int = 0) -> dict:
        import numpy as np
        K, J, cores = self.K, self.J, self.cores
        n_f = int(max(cores, min(K, 0.5 * budget_s * self.rate / J)))
        n_a = int(max(cores, min(J, 0.5 * budget_s * self.rate / K)))
        rng = np.random.default_rng(seed)
        ks = np.sort(rng.choice(K, n_f, replace=False))
        js = np.sort(rng.choice(J, n_a, replace=False))
        a = np.ones(K, dtype=np.complex128)
        t0 = time.perf_counter()
        self.O.forward(self.uvw[ks], self.lmn, self.sky, self._sel(ks), self.occ, nthreads=cores)
        t1 = time.perf_counter()
        self.O.adjoint(self.uvw, a, self.lmn[js], self.refs, self.occ, nthreads=cores)
        t2 = time.perf_counter()
        return {"terms": n_f * J + n_a * K, "seconds": t2 - t0,
                "sample": f"{n_f} samples x {J} pixels (forward) + {n_a} pixels x {K} samples "
                          f"(adjoint), FP64 oracle, OpenMP"}


def cpu_baseline(obs, f_hz, budget_s: float = 15.0):
    """One bounded sample of the workload through the FP64 CPU restatement."""
    smp = CpuSampler(obs, f_hz)
    r = smp.sample(budget_s)
    return {"value": round(r["terms"] / r["seconds"] / 1e9, 5), "unit": UNIT, "cores": smp.cores,
            "kind": "port", "sample": r["sample"], "seconds": round(r["seconds"], 2)}


# ---------------------------------------------------------- reference arm
def run_gridded(args):
    """The imaging adjoint two ways on one workload, unmasked (computeC of the
    noblockage programs) and occulted (of the blockage programs): the direct
    kernel (viss_adjoint) and per-facet type-3 NUFFTs (viss_adjoint_gridded,
    facet size chosen by the library; occulted: the pairs whose facet the
    sample sees wholly gridded, the rest direct).  CUDA events around each
    call, rel-L2 between the images."""
    import torch
    from viss_optimize_3d_b200 import pipeline, synth

    dev = torch.device("cuda", 0)
    name = args.workload
    cfg = workload_config(name)
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, cfg.freqs_hz[0], device=dev)
    K, J = g.plan.K, g.plan.J
    gen = torch.Generator(device=dev).manual_seed(1)
    a = torch.complex(torch.randn(K, device=dev, generator=gen), torch.randn(K, device=dev, generator=gen))
    stream = torch.cuda.current_stream(dev)
    steps = max(1, min(args.steps, 3))
    warm = max(1, min(args.warmup, 2))

    def timed(fn):
        for _ in range(warm):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ts = []
        for _ in range(steps):
            torch.cuda.synchronize()
            e0.record(stream)
            out = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return sorted(ts)[len(ts) // 2], out

    terms = K * J
    res = {"metric": "G uvw x pixel terms/s, occulted imaging adjoint (computeC), rel-L2<=1e-5", "unit": UNIT,
           "n_gpus": 1, "steps": steps, "warmup": warm, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64-phase/f32-grid", "data": "synthetic (seeded, see synth.py)",
           "config": {"workload": WORKLOAD_TEXT.get(name, name), "pixels": J, "samples": K,
                      "coefficients": "complex normal (seeded)"}}
    for label, mask in (("unmasked", False), ("occulted", True)):
        t_direct, direct = timed(lambda: g.plan.adjoint(a, mask=mask))
        t_grid, grid = timed(lambda: g.plan.adjoint_gridded(a, mask=mask))
        info = g.plan.gridded_info()
        err = float(torch.linalg.norm((grid - direct).double()) / torch.linalg.norm(direct.double()))
        res[label] = {
            "direct": {"entry_point": "viss_adjoint" + ("" if mask else " (VISS_NO_MASK)"),
                       "ms": round(t_direct * 1e3, 2), "value": round(terms / t_direct / 1e9, 3)},
            "gridded": {"entry_point": "viss_adjoint_gridded" + ("" if mask else " (VISS_NO_MASK)"),
                        "ms": round(t_grid * 1e3, 2), "value": round(terms / t_grid / 1e9, 3),
                        "facet_pixels": info["facet_pixels"], "facets": -(-J // info["facet_pixels"]),
                        "grid": list(info["grid"]), "hbm_spread_blocks": info["hbm_blocks"]},
            "speedup_gridded_vs_direct": round(t_direct / t_grid, 3),
            "image_rel_l2_gridded_vs_direct": float(f"{err:.3e}"),
        }
    res["value"] = res["occulted"]["gridded"]["value"]
    res["ms_per_step"] = res["occulted"]["gridded"]["ms"]
    return res


def run_stream(args):
    """Observation days from files to images, wall clock, three ways on the same
    synthetic days: the text drop-in executable (the reference's interface and
    file formats, one day after another), the binary streaming loop, and the
    loop with --fold-mirrors.  Terms per day are counted in the headline unit
    (forward + adjoint over the unique samples)."""
    import dataclasses
    import shutil
    import subprocess
    import tempfile

    import numpy as np
    from viss_optimize_3d_b200 import api, dayfile, synth

    cfg = synth.CONFIGS["c3_10mhz"]
    f_hz, ndays = 1e7, args.stream_days
    bindir = os.path.join(ROOT, "viss_optimize_3d_b200", "bin")
    work = tempfile.mkdtemp(prefix="viss_stream_")
    try:
        th, ph, _ = api.pix2ang(cfg.nside, "ring")
        th, ph = th.cpu().numpy().astype(np.float32), ph.cpu().numpy().astype(np.float32)
        sky = synth.make_observation(cfg).sky.astype(np.float32)
        tdir, bdir = os.path.join(work, "earth_10Mhz"), os.path.join(work, "bin")
        for d in (tdir, bdir, os.path.join(work, "out_text")):
            os.makedirs(d)
        dayfile.write_sky(os.path.join(bdir, "sky.vsky"), sky, th, ph)
        with open(os.path.join(tdir, "B_10Mhz.txt"), "w") as fh:
            fh.write(f"{sky.size}\n")
            np.savetxt(fh, sky, fmt="%.9g")
        np.savetxt(os.path.join(tdir, "theta_heal_10Mhz.txt"), th, fmt="%.9g")
        np.savetxt(os.path.join(tdir, "phi_heal_10Mhz.txt"), ph, fmt="%.9g")
        n_unique = 0
        for d in range(1, ndays + 1):
            rows = dayfile.observation_rows(
                synth.make_observation(dataclasses.replace(cfg, day=float(d - 1))), f_hz)
            n_unique = rows.uvw.shape[0] // 2
            dayfile.write_day(dayfile.day_path(bdir, d), rows, day=d, frequency=f_hz)
            for name, arr in (("uvw", rows.uvw), ("xyza", rows.xyza), ("xyzb", rows.xyzb)):
                with open(os.path.join(tdir, f"{name}{d}day1M.txt"), "w") as fh:
                    fh.write("0 0 0\n")
                    np.savetxt(fh, arr, fmt="%.9g")
            with open(os.path.join(tdir, f"bll{d}day1M.txt"), "w") as fh:
                fh.write("0\n")
                np.savetxt(fh, rows.bll, fmt="%.9g")

        def timed(cmd):
            t0 = time.perf_counter()
            r = subprocess.run(cmd, cwd=work, capture_output=True, text=True, timeout=3600)
            dt = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError(f"{cmd[0]} failed: {r.stderr[-2000:]}")
            return dt, r.stdout

        t_text, _ = timed([os.path.join(bindir, "vissgen3d_blockage_10m"), "--days", str(ndays),
                           "--data-dir", tdir, "--out-dir", os.path.join(work, "out_text")])
        base = [os.path.join(bindir, "vissgen_stream"), "--sky", os.path.join(bdir, "sky.vsky"),
                "--days-dir", bdir, "--days", str(ndays), "--frequency", str(f_hz), "--blockage", "1"]
        t_bin, out_bin = timed(base + ["--sum-out", os.path.join(work, "sum.vimg")])
        t_fold, out_fold = timed(base + ["--fold-mirrors", "--sum-out", os.path.join(work, "sum_fold.vimg")])
        # the same work: day sums of the three runs agree
        text_sum = sum(np.loadtxt(os.path.join(work, "out_text", f"C{d}day1M.txt"))
                       for d in range(1, ndays + 1))
        s_bin = dayfile.read_image(os.path.join(work, "sum.vimg"))[0]
        s_fold = dayfile.read_image(os.path.join(work, "sum_fold.vimg"))[0]
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        terms_day = 2 * n_unique * cfg.npix
        info_bin = json.loads(out_bin.strip().splitlines()[-1])
        info_fold = json.loads(out_fold.strip().splitlines()[-1])

        def line(t):
            return {"days_per_s": round(ndays / t, 4), "s_per_day": round(t / ndays, 4),
                    "gterms_per_s_e2e": round(terms_day * ndays / t / 1e9, 2)}
        return {"metric": "observation days/s, files to images (wall clock)", "unit": "days/s",
                "value": round(ndays / t_fold, 4), "higher_is_better": True, "n_gpus": 1,
                "days": ndays, "data": "synthetic (seeded lunar-orbit formation, see synth.py)",
                "config": {"workload": WORKLOAD_TEXT["stream"], "pixels": cfg.npix,
                           "unique_samples_per_day": n_unique, "terms_per_day": terms_day},
                "text_drop_in": line(t_text), "binary_stream": line(t_bin),
                "binary_stream_fold_mirrors": line(t_fold),
                "stream_gpu_ms_per_day": round(info_bin["gpu_ms_total"] / ndays, 2),
                "stream_fold_gpu_ms_per_day": round(info_fold["gpu_ms_total"] / ndays, 2),
                "day_sum_rel_l2": {"binary_vs_text": rel(s_bin, text_sum),
                                   "fold_vs_binary": rel(s_fold, s_bin)},
                "speedup_vs_text": round(t_text / t_fold, 2)}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def run_reference(args, rank, world):
    """The reference arm: the reference's path on the host cores.  The
    reference has no CPU implementation (its kernels are CUDA only), so this
    is the FP64 restatement of its kernels (oracle/) on every host thread.
    Each step is one bounded sample of the workload (a seeded subset of
    samples x all pixels for the forward and of pixels x all samples for the
    adjoint), sized so that warm-up + timed steps take about
    --reference-seconds in all; ms_per_step is the measured time of one such
    sample and value the terms it evaluated per second."""
    if rank != 0:
        return None
    from viss_optimize_3d_b200 import synth
    if args.workload in ("c1", "c2", "c3_10mhz", "c3_1mhz", "c3_small", "prod_1mhz"):
        cfg = workload_config(args.workload)
    else:
        return {"impl": "reference", "unavailable": f"workload {args.workload} has no reference "
                "counterpart (batched channels, reconstruction and day files are this repository's)"}
    obs = synth.make_observation(cfg)
    f_hz = cfg.freqs_hz[0]
    smp = CpuSampler(obs, f_hz)
    budget = min(args.cpu_seconds, max(1.0, args.reference_seconds / max(1, args.steps + args.warmup)))
    runs = [smp.sample(budget, seed=i) for i in range(args.warmup + args.steps)][args.warmup:]
    terms = sum(r["terms"] for r in runs)
    secs = sum(r["seconds"] for r in runs)
    v = terms / secs / 1e9
    return {
        "impl": "reference",
        "metric": METRIC, "value": round(v, 5), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(secs / len(runs) * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (same generator and seed as our arm)",
        "config": bench_config(args, obs.cfg.npix, obs.cfg.n_samples, world),
        "step": "one bounded sample of the workload per step (the reference has no CPU "
                "implementation; this is the FP64 restatement of its kernels, oracle/)",
        "cpu_baseline": {"value": round(v, 5), "unit": UNIT, "cores": smp.cores,
                         "kind": "port", "sample": runs[-1]["sample"] + " per step"},
        "e2e": {"value": round(v, 5), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-fp64-compare", dest="fp64_compare", action="store_false",
                    help="skip timing the plain FP64 path on the same step")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="time budget of the CPU baseline's bounded sample (and the cap per step of "
                         "the reference arm)")
    ap.add_argument("--reference-seconds", type=float, default=150.0,
                    help="reference arm: about this many seconds for warm-up + timed steps in all")
    ap.add_argument("--record-traffic", metavar="NCU_CSV",
                    help="store the DRAM bytes per launch of an ncu --csv metrics log of this "
                         "workload as the traffic record of the current kernel sources, and exit")
    ap.add_argument("--record-command", default="", help="the ncu command line, stored with the record")
    ap.add_argument("--record-commit", default="", help="the commit the capture ran on (default: HEAD)")
    ap.add_argument("--workload", default=WORKLOAD, choices=sorted(WORKLOAD_TEXT),
                    help="benchmark configuration (default: the headline one)")
    ap.add_argument("--formation", action="store_true",
                    help="run the step through the formation entry points (satellite vectors)")
    ap.add_argument("--no-formation-compare", dest="formation_compare", action="store_false",
                    help="skip timing the formation entry points beside the headline step")
    ap.add_argument("--stream-days", type=int, default=4,
                    help="days of the stream workload")
    ap.add_argument("--gridded", action="store_true",
                    help="time the imaging adjoint (unmasked and occulted) direct vs gridded (per-facet NUFFT) "
                         "on --workload")
    args = ap.parse_args()
    if args.record_traffic:
        print(json.dumps(record_traffic(args.record_traffic, args.workload, args.record_command,
                                        args.record_commit)))
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus != world and world > 1:
        print(f"warning: --gpus {args.gpus} but WORLD_SIZE {world}", file=sys.stderr)
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == "c4":
            print(json.dumps(run_batched(args)), flush=True)
            return
        if args.workload == "c5":
            print(json.dumps(run_reconstruction(args)), flush=True)
            return
        if args.workload == "stream":
            print(json.dumps(run_stream(args)), flush=True)
            return
        if args.gridded:
            if rank == 0:
                print(json.dumps(run_gridded(args)), flush=True)
            return
        res = run_ours(args, rank, world, local_rank)
        if not args.formation and args.formation_compare and args.workload in ("c1", "c2", "c3_10mhz", "c3_1mhz", "c3_small"):  # noqa: E501
            # the same step through the formation entry points (satellite vectors
            # instead of per-sample uvw), reported beside the headline
            f = run_formation(args, rank, world, local_rank)
            if res is not None and f is not None:
                res["formation_mode"] = {k: f[k] for k in ("value", "unit", "ms_per_step", "e2e", "roofline",
                                                           "kernel_ms", "culling", "forward_rel_l2_vs_direct",
                                                           "clocks")}
                res["formation_mode"]["entry_points"] = ("viss_plan_set_formation, viss_forward_formation, "
                                                         "viss_adjoint_formation")
        if res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
