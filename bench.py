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
    "c2": "Nside 64 (49,152 px) x 20,160 uvw samples (28 baselines x 720 snapshots), 10 MHz, "
          "Moon occultation (profiling-size case)",
    "c3_small": "Nside 256 (786,432 px) x 48,600 uvw samples (45 baselines x 1,080 snapshots), "
                "10 MHz, Moon + Earth occultation (profiling-size case of the headline workload)",
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
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# tuned shapes, from the one-pass ncu capture of this bench command recorded in
# profiles/dram_c3_10mhz.md; bench.py cannot read DRAM counters itself.
NCU_TRAFFIC = {"c3_10mhz": {"k_forward": 56540672 + 45793024, "k_adjoint": 60630784 + 45324032}}
NCU_TRAFFIC_SOURCE = "profiles/dram_c3_10mhz.md (ncu, one pass, full-size workload)"
FORM_NCU_TRAFFIC = {"c3_10mhz": {"k_form_forward": 32984064 + 449792, "k_form_adjoint": 36857344 + 32256}}
FORM_NCU_TRAFFIC_SOURCE = "profiles/launches_bench_formation_c3_10mhz.md (ncu, one pass, full-size workload)"


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

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    if args.formation:
        return run_formation(args, rank, world, local_rank)
    if args.workload == "c3_small":
        cfg = synth.scaled(synth.CONFIGS["c3_10mhz"], n_snap=1080)
    else:
        cfg = synth.CONFIGS[args.workload]
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

    # device-resident step: forward, DCF + weights, adjoint
    def step():
        V = g.plan.forward(g.sky)
        return pipeline.dirty_image(g, V)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # launch-shape sweep (recorded) and the plan's own tuner (chooses)
    V0 = g.plan.forward(g.sky)
    gs0, _c0, dcf0 = api.dcf(g.bll, g.nr, multiplicity=2)
    coef0 = api.scale_coef(api.weights(g.w, g.bll, gs0, dcf0, g.nr)[1], V0)
    sweep = {"forward_ms": [], "adjoint_ms": []}
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
        step_ev[i][1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        torch.distributed.barrier()
    step_ms = [a.elapsed_time(b) for a, b in step_ev]
    fwd_ms = [a.elapsed_time(b) for a, b in fwd_ev]
    adj_ms = [a.elapsed_time(b) for a, b in adj_ev]
    total_s = sum(step_ms) / 1e3
    # culled fraction of the last forward/adjoint (device counters)
    g.plan.forward(g.sky)
    ev_f, mx_f, tot = g.plan.last_stats()
    g.plan.adjoint(coef, scale=2.0, mask=cfg.imaging_mask)
    ev_a, mx_a, _ = g.plan.last_stats()

    # end to end through the public API from pinned host buffers
    sky_h = torch.from_numpy(obs.sky_at(f_hz).astype(np.float32) * np.float32(4 * math.pi / J)).pin_memory()
    uvw_h = torch.from_numpy(obs.uvw(f_hz)).pin_memory()
    masked = obs.refs is not None
    refs_h = torch.from_numpy(obs.refs).pin_memory() if masked else None
    img_h = torch.empty(J, dtype=torch.float32).pin_memory()
    V_h = torch.empty(K, dtype=torch.complex64).pin_memory()
    sky_d = torch.empty_like(g.sky)
    uvw_d = torch.empty_like(g.uvw)
    refs_d = torch.empty_like(g.refs) if masked else None
    from viss_optimize_3d_b200._capi import check, lib
    import ctypes as C

    def e2e_step():
        sky_d.copy_(sky_h, non_blocking=True)
        uvw_d.copy_(uvw_h, non_blocking=True)
        if masked:
            refs_d.copy_(refs_h, non_blocking=True)
        check(lib.viss_plan_set_samples(g.plan._h, K, C.c_void_p(uvw_d.data_ptr()), None,
                                        C.c_void_p(refs_d.data_ptr()) if masked else None,
                                        g.occ.shape[0] if masked else 0,
                                        C.c_void_p(g.occ.data_ptr()) if masked else None,
                                        C.c_void_p(stream.cuda_stream)), "set_samples")
        Vd = g.plan.forward(sky_d)
        imgd = pipeline.dirty_image(g, Vd)
        V_h.copy_(Vd, non_blocking=True)
        img_h.copy_(imgd, non_blocking=True)

    e2e_steps = max(1, min(args.steps, 3))
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
    h2d = J * 4 + K * 24 + (K * 12 if masked else 0)
    d2h = J * 4 + K * 8

    # max over ranks (device-timed seconds)
    total_s, e2e_s = replicas.max_over_ranks([total_s, e2e_s], device=dev)
    if rank != 0:
        return None

    # the plain FP64 path on the same step (the split path's >= 3x target)
    fp64 = None
    if args.fp64_compare:
        f0, f1, f2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        f0.record(stream)
        Vd = g.plan.forward(g.sky, fp64=True)
        f1.record(stream)
        g.plan.adjoint(coef, scale=2.0, mask=cfg.imaging_mask, fp64=True)
        f2.record(stream)
        torch.cuda.synchronize()
        fp64_fwd, fp64_adj = f0.elapsed_time(f1) / 1e3, f1.elapsed_time(f2) / 1e3
        split_fwd, split_adj = statistics.mean(fwd_ms) / 1e3, statistics.mean(adj_ms) / 1e3
        Vs = g.plan.forward(g.sky).to(torch.complex128)
        rel = (torch.linalg.norm(Vs - Vd.to(torch.complex128)) / torch.linalg.norm(Vd.to(torch.complex128))).item()
        fp64 = {"value": round(terms_per_step / (fp64_fwd + fp64_adj) / 1e9, 3), "unit": UNIT,
                "forward_ms": round(fp64_fwd * 1e3, 2), "adjoint_ms": round(fp64_adj * 1e3, 2),
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
        "config": {"workload": WORKLOAD_TEXT.get(args.workload, args.workload),
                   "pixels": J, "samples": K, "terms_per_step": terms_per_step,
                   "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": {"value": round(terms_per_step * e2e_steps / e2e_s / 1e9 * world, 3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "pinned host sky/uvw/refs -> viss_plan_set_samples -> viss_forward -> "
                        "viss_dcf/viss_weights -> viss_adjoint -> pinned host V/image"},
        "roofline": {"bound": "sfu", "kernel": f"k_{dom}",
                     "achieved": round(achieved / 1e9, 2), "peak": round(peak_terms / 1e9, 1),
                     "unit": "Gterms/s", "frac": round(achieved / peak_terms, 4),
                     "peak_source": f"8 terms/clk/SM x {nsm} SMs x sm_max_mhz ({pk_kind})",
                     "evaluated_frac": round(dom_eval / (K * J), 4),
                     "frac_of_evaluated": round(dom_eval / dom_s / peak_terms, 4),
                     "traffic": NCU_TRAFFIC.get(args.workload, {}).get(f"k_{dom}"),
                     "traffic_unit": "bytes per launch",
                     "traffic_source": NCU_TRAFFIC_SOURCE if args.workload in NCU_TRAFFIC else None},
        "kernel_ms": {"forward": round(fwd_s * 1e3, 3), "adjoint": round(adj_s * 1e3, 3)},
        "culling": {"forward_evaluated": round(ev_f / tot, 4), "forward_mixed": round(mx_f / tot, 4),
                    "adjoint_evaluated": round(ev_a / tot, 4), "adjoint_mixed": round(mx_a / tot, 4)},
        "gpu_launches": 10 * args.steps,
        "fp64_path": fp64,
        "tuning": {"chosen": {"forward": shapes[0], "adjoint": shapes[1]},
                   "forward_shapes": "(samples/thread, CTAs/SM) = (4,2) (4,3) (2,3) (2,4)",
                   "adjoint_shapes": "(pixels/lane, CTAs/SM), 128-thread CTAs = (8,4) (8,5) (4,5) (4,6)", **sweep},
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
    if args.workload == "c3_small":
        cfg = synth.scaled(synth.CONFIGS["c3_10mhz"], n_snap=1080)
    elif args.workload in ("c1", "c2", "c3_10mhz", "c3_1mhz"):
        cfg = synth.CONFIGS[args.workload]
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

    # end to end: pinned host sky and satellite vectors -> image and V on the host
    sky_h = torch.from_numpy(obs.sky_at(f_hz).astype(np.float32) * np.float32(4 * math.pi / J)).pin_memory()
    U_h = U.cpu().pin_memory()
    U_d, sky_d = torch.empty_like(U), torch.empty_like(g.sky)
    img_h = torch.empty(J, dtype=torch.float32).pin_memory()
    V_h = torch.empty(K, dtype=torch.complex64).pin_memory()
    os_p = C.c_void_p(occ_sat.data_ptr()) if occ_sat is not None else None
    on_p = C.c_void_p(occ_snap.data_ptr()) if occ_snap is not None else None

    def e2e_step():
        sky_d.copy_(sky_h, non_blocking=True)
        U_d.copy_(U_h, non_blocking=True)
        check(lib.viss_plan_set_formation(plan._h, plan.form_T, plan.form_S, C.c_void_p(U_d.data_ptr()),
                                          None, os_p, on_p, C.c_void_p(stream.cuda_stream)),
              "viss_plan_set_formation")
        Vd_ = plan.forward_formation(sky_d)
        imgd = image(Vd_)
        V_h.copy_(Vd_, non_blocking=True)
        img_h.copy_(imgd, non_blocking=True)

    e2e_steps = max(1, min(args.steps, 3))
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
    total_s, e2e_s = replicas.max_over_ranks([total_s, e2e_s], device=dev)
    if rank != 0:
        return None
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
        "config": {"workload": WORKLOAD_TEXT.get(args.workload, args.workload) + "; formation mode",
                   "pixels": J, "samples": K, "satellites": plan.form_S, "snapshots": plan.form_T,
                   "terms_per_step": terms_per_step, "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": {"value": round(terms_per_step * e2e_steps / e2e_s / 1e9 * world, 3), "unit": UNIT,
                "h2d_bytes_per_step": J * 4 + U.numel() * 8, "d2h_bytes_per_step": J * 4 + K * 8,
                "path": "pinned host sky/U -> viss_plan_set_formation -> viss_forward_formation -> "
                        "viss_dcf/viss_weights -> viss_adjoint_formation -> pinned host V/image"},
        "roofline": {"bound": "fp32", "kernel": f"k_form_{dom}",
                     "achieved": round(achieved / 1e9, 2), "peak": round(peak_terms / 1e9, 1),
                     "unit": "Gterms/s", "frac": round(achieved / peak_terms, 4),
                     "peak_source": f"128 FP32 lanes/clk/SM / {FORM_FFMA_PER_TERM} FFMA per term x {nsm} SMs "
                                    f"x sm_max_mhz ({pk_kind})",
                     "evaluated_frac": round(dom_eval / (K * J), 4),
                     "traffic": FORM_NCU_TRAFFIC.get(args.workload, {}).get(f"k_form_{dom}"),
                     "traffic_unit": "bytes per launch",
                     "traffic_source": FORM_NCU_TRAFFIC_SOURCE if args.workload in FORM_NCU_TRAFFIC else None},
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
def cpu_baseline(obs, f_hz, budget_s: float = 15.0):
    """The FP64 CPU restatement (oracle/) on all host cores, on a bounded
    sample: n_f samples x all pixels (forward) and n_a pixels x all samples
    (adjoint), sized to about budget_s seconds."""
    import numpy as np
    from oracle import oracle as O

    O.build()
    cores = O.max_threads()
    _, _, xyz = O.pix2ang(obs.cfg.nside)
    lmn = O.lmn_from_xyz(xyz)
    uvw = obs.uvw(f_hz)
    sky = obs.sky_at(f_hz) * (4 * math.pi / obs.cfg.npix)
    refs, occ = obs.refs, None
    if refs is not None:
        occ = O.occulters(obs.occ_sat_positions, 1737.4e3, 0)
        if obs.earth_rows is not None:
            occ = np.concatenate([occ, obs.earth_rows])
    sel = (lambda r, idx: None if r is None else r[idx])
    K, J = uvw.shape[0], lmn.shape[0]
    # calibrate on slices that grow until one takes >= 0.5 s (a tiny slice
    # measures thread start-up more than the sum)
    n_cal = cores
    while True:
        t0 = time.perf_counter()
        O.forward(uvw[:n_cal], lmn, sky, sel(refs, slice(0, n_cal)), occ, nthreads=cores)
        dt = time.perf_counter() - t0
        if dt >= 0.5 or n_cal >= K:
            break
        n_cal = min(K, n_cal * 4)
    rate = n_cal * J / max(dt, 1e-6)                              # terms/s
    n_f = int(max(cores, min(K, 0.5 * budget_s * rate / J)))
    n_a = int(max(cores, min(J, 0.5 * budget_s * rate / K)))
    rng = np.random.default_rng(0)
    ks = np.sort(rng.choice(K, n_f, replace=False))
    js = np.sort(rng.choice(J, n_a, replace=False))
    a = np.ones(K, dtype=np.complex128)
    t0 = time.perf_counter()
    O.forward(uvw[ks], lmn, sky, sel(refs, ks), occ, nthreads=cores)
    t1 = time.perf_counter()
    O.adjoint(uvw, a, lmn[js], refs, occ, nthreads=cores)
    t2 = time.perf_counter()
    terms = n_f * J + n_a * K
    return {"value": round(terms / (t2 - t0) / 1e9, 5), "unit": UNIT, "cores": cores,
            "kind": "port",
            "sample": f"{n_f} samples x {J} pixels (forward) + {n_a} pixels x {K} samples "
                      f"(adjoint), FP64 oracle, OpenMP",
            "seconds": round(t2 - t0, 2)}


# ---------------------------------------------------------- reference arm
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
    if rank != 0:
        return None
    from viss_optimize_3d_b200 import synth
    if args.workload == "c3_small":
        cfg = synth.scaled(synth.CONFIGS["c3_10mhz"], n_snap=1080)
    elif args.workload in ("c1", "c2", "c3_10mhz", "c3_1mhz"):
        cfg = synth.CONFIGS[args.workload]
    else:
        return {"impl": "reference", "unavailable": f"workload {args.workload} has no reference "
                "counterpart (batched channels, reconstruction and day files are this repository's)"}
    obs = synth.make_observation(cfg)
    f_hz = cfg.freqs_hz[0]
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(obs, f_hz, budget_s=args.cpu_seconds)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.mean(x["value"] for x in vals)
    last = vals[-1]
    terms = 2 * obs.cfg.n_samples * obs.cfg.npix
    return {
        "impl": "reference",
        "metric": METRIC, "value": round(v, 5), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(terms / (v * 1e9) * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (same generator and seed as our arm)",
        "config": {"workload": WORKLOAD_TEXT.get(args.workload, args.workload),
                   "pixels": obs.cfg.npix, "samples": obs.cfg.n_samples, "terms_per_step": terms,
                   "note": "the reference has no CPU implementation; this is the FP64 "
                           "restatement of its kernels (oracle/), timed on a bounded sample"},
        "cpu_baseline": {"value": round(v, 5), "unit": UNIT, "cores": last["cores"],
                         "kind": "port", "sample": last["sample"]},
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
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--workload", default=WORKLOAD, choices=sorted(WORKLOAD_TEXT),
                    help="benchmark configuration (default: the headline one)")
    ap.add_argument("--formation", action="store_true",
                    help="run the step through the formation entry points (satellite vectors)")
    ap.add_argument("--no-formation-compare", dest="formation_compare", action="store_false",
                    help="skip timing the formation entry points beside the headline step")
    ap.add_argument("--stream-days", type=int, default=4,
                    help="days of the stream workload")
    args = ap.parse_args()

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
        res = run_ours(args, rank, world, local_rank)
        if not args.formation and args.formation_compare and args.workload in ("c1", "c2", "c3_10mhz", "c3_1mhz", "c3_small"):
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
