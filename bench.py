#!/usr/bin/env python
"""Throughput of the FMM force pass on B200 at 1e-6 relative force error
(particles per second), tensor-core translations against the plain FP32 GPU
FMM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step is one force evaluation of the whole system: tree build (the
reference's Tree::init_tree) and every FMM pass, the work of the
reference's FMM::update (src/system_updaters/FMM.cpp:9-12).  Workload: a 3D
Plummer sphere of N = 2^20 particles (scale radius 1, truncated at 20, seed
2, equal masses summing to 1), leaf capacity 64, forces in FP32 from FP64
positions, G = 1, at expansion order p = 12: the lowest order whose relative
L2 force error against the FP64 direct sum is <= 1e-6 on this input
(p = 11 gives 1.06e-6, p = 12 8.6e-7).  M2L, M2M and L2L run on the tensor
cores (tcgen05, 3xBF16 split, FP32 accumulation); interaction-list pairs with
n_T * n_S <= direct_max are summed directly.

value: N * K / (sum of the K per-step device times), inputs resident in HBM,
       timed with CUDA events on the launching stream; a 256 MiB buffer is
       written between steps (outside the event pair) to flush L2.  With N
       GPUs each rank runs its own replica (the single-system pass does not
       shard), value sums the particles of all ranks over the slowest rank.
order: the tensor-core tiles take the orders the learned MLP picks
       (FMM_ORDER_LEARNED); the judge (512 targets against the FP64 direct
       sum, budget 1e-6, fixed-order fallback) checks the first and then every
       8th evaluation, inside the timed steps.  The first evaluation runs at
       p (warm-up).
tc_fixed_order, plain: the same workload and maximum order through the
       tensor cores at fixed p, and through the plain FP32 GPU FMM (SIMT
       contractions, FMM_M2L_FP32), timed the same way; speedup_vs_plain is
       the headline against the latter at equal error.
e2e:   the headline configuration through the public C ABI with pinned host
       buffers (fmm_evaluate: host-to-device copy of positions and masses,
       the pass, device-to-host copy of accelerations), wall clock per call.
autotune: before timing, fmm_autotune times the candidate direct-pair
       thresholds on this input and keeps the fastest (setup, not timed).
roofline: the dominant kernel by live-measured time, and both of the two
       largest: the tensor-core M2L (algorithmic FLOPs 2 K^2 per
       interaction-list pair, K = (p+1)^2, against the measured sustained
       BF16 peak) and the direct far field (20 FLOPs per particle pair,
       against the FP32 peak derived from the SM count and clock).
cpu_baseline: the reference itself (compiled from its sources into
       oracle/_ref) timing FMM::update on a bounded Plummer sample, 1 thread.
--impl reference: the reference's CPU FMM on all host cores (one process per
       core, each a bounded sample of the same workload), rank 0 only.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nbody-fmm_b200"))

METRIC = "3D FMM particles/s at 1e-6 rel force err: learned+TC vs plain GPU FMM"
UNIT = "particles/s"
REF_SAMPLE_N = 512           # particles per reference process per step (about 2 s at p = 12)
CPU_SAMPLE_N = 2048     # single-thread CPU baseline sample (about 20 s at p = 12)


def workload_desc(n, p, leaf, m2l, direct_max=None, mixture=False):
    inputs = (f"3D clustered mixture N={n} (32 Plummer spheres, scale radii log-uniform in [0.01, 0.1], "
              f"centres uniform in [0,1]^3, equal mass per sphere, seed 5)" if mixture
              else f"3D Plummer sphere N={n} (a=1, r<=20, seed 2)")
    return {
        "workload": f"{inputs}, p={p}, leaf capacity {leaf}, "
                    f"one force evaluation (tree build + all FMM passes) per step",
        "n": n, "p": p, "leaf_cap": leaf, "m2l": m2l, "direct_max": direct_max, "positions": "f64",
        "forces": "f32", "l2": "256 MiB buffer written between steps (outside the timed events)",
        "parallelism": "replicas",
    }


def max_over_ranks(x, world, dev):
    """The largest x over the ranks (the slowest rank's time); x on one rank."""
    if world <= 1:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def min_over_ranks(x, world, dev):
    """The smallest x over the ranks (the slowest rank's rate); x on one rank."""
    if world <= 1:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MIN)
    return float(t.item())


def job_rate(particles_per_rank, steps, world, seconds):
    """Whole-job particles/s: the particles of every rank's steps over the
    slowest rank's time."""
    return particles_per_rank * steps * world / seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"fmm_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


# ---------------------------------------------------------------- ours
def _timed(ctx, n, d_pos, d_mass, d_acc, stream, flush, steps, warmup, barrier):
    """Runs warmup + steps passes; returns per-step device ms and stats."""
    import torch

    sp = stream.cuda_stream
    for _ in range(warmup):
        flush.zero_()
        ctx.evaluate_device(n, d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), None, sp)
        ctx.synchronize()
    barrier()
    step_ms, stats = [], []
    l0 = ctx.launch_count()
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.evaluate_device(n, d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), None, sp)
        e1.record(stream)
        ctx.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        stats.append(ctx.stats())
    launches = ctx.launch_count() - l0
    barrier()
    return step_ms, stats, launches


def _error(ctx, n, d_pos, d_mass, d_acc, d_pot, stream, dev, judge):
    """Relative force and potential errors on 4096 sampled targets against
    the FP64 direct sum on the GPU."""
    import torch

    d_tg, ra, rp = judge
    ctx.evaluate_device(n, d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr(), stream.cuda_stream)
    ctx.synchronize()
    a = d_acc[d_tg].cpu().numpy()
    ph = d_pot[d_tg].cpu().numpy()
    return {
        "targets": int(d_tg.numel()), "vs": "FP64 direct sum on the GPU",
        "force_rel_l2": float(np.linalg.norm(a - ra) / np.linalg.norm(ra)),
        "force_max_rel": float((np.linalg.norm(a - ra, axis=1) / np.linalg.norm(ra, axis=1)).max()),
        "pot_rel_l2": float(np.linalg.norm(ph - rp) / np.linalg.norm(rp)),
        "pot_max_rel": float((np.abs(ph - rp) / np.abs(rp)).max()),
    }


def _phases(stats):
    keys = ("ms_tree", "ms_upward", "ms_m2l", "ms_downward", "ms_p2p", "ms_far_direct", "ms_total")
    return {k: float(np.mean([s[k] for s in stats])) for k in keys}


def run_ours(args, world, rank, local):
    import torch

    import fmmgpu
    from fmmgpu import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    n, p, leaf = args.n, args.p, args.leaf
    mixture = args.workload == "mixture"
    tune_leaf = mixture  # the mixture's configuration leaves the leaf capacity open
    mode = fmmgpu.FMM_M2L_TC if args.m2l == "tc" else fmmgpu.FMM_M2L_FP32
    pos, mass = workloads.plummer_mixture(n, seed=5) if mixture else workloads.plummer(n, seed=2)
    d_pos = torch.from_numpy(pos).to(dev)
    d_mass = torch.from_numpy(mass).to(dev)
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
    d_pot = torch.empty((n,), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # a stream of our own (torch's default stream has handle 0, which the C
    # ABI reads as "the context's stream")
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    # the judge: FP64 direct sum on 4096 sampled targets (8192 on the mixture)
    rng = np.random.default_rng(7)
    tg = np.sort(rng.choice(n, size=min(8192 if mixture else 4096, n), replace=False)).astype(np.int64)
    d_tg = torch.from_numpy(tg).to(dev)
    r_acc = torch.empty((len(tg), 3), dtype=torch.float64, device=dev)
    r_pot = torch.empty((len(tg),), dtype=torch.float64, device=dev)
    with fmmgpu.Context(dim=3, G=1.0, device=local) as jc:
        jc.direct_device(n, d_pos.data_ptr(), d_mass.data_ptr(), len(tg), d_tg.data_ptr(), r_acc.data_ptr(),
                         r_pot.data_ptr(), stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    judge = (d_tg, r_acc.cpu().numpy(), r_pot.cpu().numpy())

    # headline: the chosen M2L mode
    learned = args.order == "learned" and mode == fmmgpu.FMM_M2L_TC
    okw = dict(order_mode=fmmgpu.FMM_ORDER_LEARNED, judge_samples=args.judge, judge_budget=1e-6,
               judge_every=args.judge_every) if learned else {}
    ctx = fmmgpu.Context(dim=3, p=p, leaf_cap=leaf, m2l_mode=mode, G=1.0, device=local, direct_max=args.direct_max,
                         adaptive_leaf=args.adaptive, **okw)
    tune = None
    if args.autotune and args.direct_max < 0:
        # the autotuner picks the direct-pair threshold on this input (setup, outside the timed steps)
        t0 = time.perf_counter()
        cands, best = ctx.autotune(n, d_pos.data_ptr(), d_mass.data_ptr(), tune_leaf=tune_leaf,
                                   stream=stream.cuda_stream)
        tune = {"seconds": time.perf_counter() - t0, "chosen_direct_max": best["direct_max"],
                "chosen_leaf_cap": best["leaf_cap"],
                "candidates": [[x["leaf_cap"], x["direct_max"], round(x["ms"], 3)] for x in cands]}
        leaf = best["leaf_cap"]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    step_ms, stats, launches = _timed(ctx, n, d_pos, d_mass, d_acc, stream, flush, args.steps, args.warmup, barrier)
    clocks = sampler.stop()
    total_ms = max_over_ranks(float(sum(step_ms)), world, dev)
    value = job_rate(n, args.steps, world, total_ms / 1e3)
    err = _error(ctx, n, d_pos, d_mass, d_acc, d_pot, stream, dev, judge)

    # end to end through the C ABI with pinned host buffers
    h_pos = torch.from_numpy(pos).pin_memory()
    h_mass = torch.from_numpy(mass).pin_memory()
    h_acc = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    hp, hm, ha = h_pos.numpy(), h_mass.numpy(), h_acc.numpy()
    ctx.evaluate(hp, hm, out=ha)
    e2e_steps = max(3, args.steps // 2)
    e2e_s = 0.0
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        ctx.evaluate(hp, hm, out=ha)
        e2e_s += time.perf_counter() - t0
    e2e_val = min_over_ranks(job_rate(n, e2e_steps, 1, e2e_s), world, dev) * world
    ctx.close()

    # rooflines of the two largest kernels, from the live event timings
    pk = peaks()
    sm_max = float(pk.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12
    tc_peak = pk.get("bf16_tflops_sustained")
    tc_src = "MEASURED_PEAKS.json bf16_tflops_sustained (cuBLAS bf16, seconds-long loop)"
    if tc_peak is None:
        tc_peak, tc_src = 1400.0, "fallback sustained bf16 figure (MEASURED_PEAKS.json absent)"
    K = (p + 1) ** 2
    ph = _phases(stats)
    s_last = stats[-1]
    m2l_flops = 2.0 * K * K * s_last["m2l_pairs"]
    far_flops = 20.0 * s_last["far_direct_pairs"]
    traffic = load_traffic()
    roofs = {
        "m2l_tc" if mode == fmmgpu.FMM_M2L_TC else "m2l_fp32": {
            "kernel": "k_tc_translate (M2L: tcgen05 3xBF16, FP32 accumulation)" if mode == fmmgpu.FMM_M2L_TC
            else "k_contract (M2L, FP32 SIMT)",
            "bound": "tensor" if mode == fmmgpu.FMM_M2L_TC else "fp32", "unit": "TFLOP/s",
            "achieved": m2l_flops / (ph["ms_m2l"] / 1e3) / 1e12 if ph["ms_m2l"] > 0 else None,
            "peak": tc_peak if mode == fmmgpu.FMM_M2L_TC else fp32_peak,
            "peak_source": tc_src if mode == fmmgpu.FMM_M2L_TC else f"derived: 148 SM x 128 FP32 lanes x 2 x {sm_max:.0f} MHz",
            "flops_per_launch": m2l_flops, "pairs": int(s_last["m2l_pairs"]), "tiles": int(s_last["m2l_tiles"]),
            "ms_per_launch": ph["ms_m2l"],
            "traffic": traffic.get("m2l_tc" if mode == fmmgpu.FMM_M2L_TC else "m2l_fp32"),
        },
        "far_direct": {
            "kernel": "k_direct_far (interaction-list pairs summed directly, FP32)", "bound": "fp32",
            "unit": "TFLOP/s", "achieved": far_flops / (ph["ms_far_direct"] / 1e3) / 1e12 if ph["ms_far_direct"] > 0 else None,
            "peak": fp32_peak, "peak_source": f"derived: 148 SM x 128 FP32 lanes x 2 x {sm_max:.0f} MHz "
                                              "(no FP32 figure in MEASURED_PEAKS.json)",
            "flops_per_launch": far_flops, "pairs": int(s_last["far_direct_pairs"]),
            "ms_per_launch": ph["ms_far_direct"], "traffic": traffic.get("far_direct"),
        },
    }
    for r in roofs.values():
        r["frac"] = r["achieved"] / r["peak"] if r["achieved"] else None
    dominant = max(roofs, key=lambda k: roofs[k]["ms_per_launch"])
    roof = dict(roofs[dominant], name=dominant)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": f"synthetic (seeded {'Plummer mixture' if mixture else 'Plummer sphere'})",
        "impl": "fmmgpu",
        "config": dict(workload_desc(n, p, leaf, args.m2l, s_last.get("direct_max"), mixture),
                       adaptive_leaf=args.adaptive),
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(n * 3 * 8 + n * 8),
                "d2h_bytes_per_step": int(n * 3 * 8)},
        "roofline": roof, "rooflines": roofs, "error": err, "phases_ms": ph,
        "tree": {"depth": s_last["depth"], "leaves": s_last["n_leaves"], "cells": s_last["n_cells"],
                 "p2p_pairs": s_last["p2p_pairs"], "far_direct_pairs": s_last["far_direct_pairs"],
                 "m2l_pairs": s_last["m2l_pairs"]},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if tune:
        line["autotune"] = tune

    if learned:
        line["order"] = {"mode": "learned (M2L tile orders from the MLP in fmmgpu/order_model.npy)",
                         "judge_samples": args.judge, "judge_budget": 1e-6, "judge_every": args.judge_every,
                         "fallbacks_in_timed_steps": int(sum(s["order_fallbacks"] for s in stats)),
                         "judged_in_timed_steps": int(sum(1 for s in stats if s["judge_rel_l2"] > 0)),
                         "judge_rel_l2_max": float(max([s["judge_rel_l2"] for s in stats] + [0.0])),
                         "m2l_width_mean": stats[-1]["m2l_width_sum"] / max(1, stats[-1]["m2l_tiles"])}

    # comparisons at the same order: tensor cores at fixed p, and the plain
    # FP32 GPU FMM (the method without tensor cores and learned orders)
    def compare(m2l_mode, label):
        pc = fmmgpu.Context(dim=3, p=p, leaf_cap=args.leaf, m2l_mode=m2l_mode, G=1.0, device=local,
                            direct_max=args.direct_max, adaptive_leaf=args.adaptive)
        chosen = None
        if args.autotune and args.direct_max < 0:  # tuned the same way as the headline
            b = pc.autotune(n, d_pos.data_ptr(), d_mass.data_ptr(), tune_leaf=tune_leaf,
                            stream=stream.cuda_stream)[1]
            chosen = {"direct_max": b["direct_max"], "leaf_cap": b["leaf_cap"]}
        psteps = max(3, args.steps // 2)
        pms, pst, _ = _timed(pc, n, d_pos, d_mass, d_acc, stream, flush, psteps, max(1, args.warmup), barrier)
        ptot = max_over_ranks(float(sum(pms)), world, dev)
        perr = _error(pc, n, d_pos, d_mass, d_acc, d_pot, stream, dev, judge)
        pc.close()
        return {"m2l": label, "value": job_rate(n, psteps, world, ptot / 1e3), "unit": UNIT, "steps": psteps,
                "ms_per_step": ptot / psteps, "error": perr, "phases_ms": _phases(pst), "tuned": chosen}

    if not args.no_plain and mode == fmmgpu.FMM_M2L_TC:
        if learned:
            line["tc_fixed_order"] = compare(fmmgpu.FMM_M2L_TC, "tensor cores, fixed p")
        line["plain"] = compare(fmmgpu.FMM_M2L_FP32, "fp32 SIMT, fixed p")
        line["speedup_vs_plain"] = value / line["plain"]["value"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p, leaf, mixture)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_frames(args, world, rank, local):
    """Frame output around the force pass: per-step device time of a loop
    of passes on the 2^20 Plummer sphere (tensor cores, fixed p) without
    frames and with a device frame (fmm_frames_write_device) every
    `frames_every` steps into a temporary directory, the final flush
    included; and the host path's write rate."""
    import tempfile

    import torch

    import fmmgpu
    from fmmgpu import workloads

    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    pos, mass = workloads.plummer(n, seed=2)
    d_pos = torch.from_numpy(pos).to(dev)
    d_mass = torch.from_numpy(mass).to(dev)
    d_vel = torch.zeros_like(d_pos)
    d_acc = torch.empty_like(d_pos)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    ctx = fmmgpu.Context(dim=3, p=args.p, leaf_cap=args.leaf, G=1.0, device=local, m2l_mode=fmmgpu.FMM_M2L_TC)
    out = tempfile.mkdtemp()

    def loop(steps, frames):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for s in range(steps):
            ctx.evaluate_device(n, d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), None, sp)
            if frames is not None and s % args.frames_every == 0:
                frames.write_device(n, d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), s, 1e-3 * s,
                                    acc_ptr=d_acc.data_ptr(), stream=sp)
        ctx.synchronize()
        if frames is not None:
            frames.flush()
        return (time.perf_counter() - t0) / steps * 1e3

    loop(args.warmup, None)
    plain = loop(args.steps, None)
    with fmmgpu.Frames(os.path.join(out, "device")) as fr:
        loop(args.warmup, fr)
        framed = loop(args.steps, fr)
    acc = d_acc.cpu().numpy()
    vel = np.zeros_like(pos)
    with fmmgpu.Frames(os.path.join(out, "host")) as fh:
        t0 = time.perf_counter()
        for s in range(3):
            fh.write(pos, vel, mass, s, 1e-3 * s, acc=acc)
        host_ms = (time.perf_counter() - t0) / 3 * 1e3
    ctx.close()
    shutil.rmtree(out, ignore_errors=True)
    print(json.dumps({"mode": "frames", "n": n, "frame_bytes": 80 * n, "frames_every": args.frames_every,
                      "steps": args.steps, "ms_per_step_without_frames": plain, "ms_per_step_with_frames": framed,
                      "host_write_ms_per_frame": host_ms, "host_write_GBps": 80 * n / host_ms / 1e6}), flush=True)


def run_ensemble(args, world, rank, local):
    """The batched-ensemble configuration: 256 independent Plummer spheres,
    N per system log-uniform in [1024, 65536] (seed 4), p = 8, leaf 64, all
    evaluated by one fmm_evaluate_batched call (concurrent worker streams);
    aggregate particles/s over the wall clock of the call, per-system error
    against the FP64 direct sum on up to 64 sampled targets per system."""
    import torch

    import fmmgpu
    from fmmgpu import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sizes = workloads.ensemble_sizes(256, 1024, 65536, seed=4)
    pos, mass = [], []
    for k, n in enumerate(sizes):
        p_, m_ = workloads.plummer(int(n), seed=1000 + k)
        pos.append(p_)
        mass.append(m_)
    pos, mass = np.concatenate(pos), np.concatenate(mass)
    off = np.r_[0, np.cumsum(sizes)].astype(np.int64)
    ntot = int(off[-1])
    d_pos, d_m = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    d_acc = torch.empty((ntot, 3), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    res = {}
    with fmmgpu.Context(dim=3, p=8, leaf_cap=64, G=1.0, m2l_mode=fmmgpu.FMM_M2L_TC, device=local) as c:
        for label, workers in (("concurrent", 0), ("one_stream", 1)):
            for _ in range(max(1, args.warmup)):
                c.evaluate_batched(off, d_pos.data_ptr(), d_m.data_ptr(), d_acc.data_ptr(), None, workers)
            steps = max(2, args.steps // 4)
            t0 = time.perf_counter()
            for _ in range(steps):
                c.evaluate_batched(off, d_pos.data_ptr(), d_m.data_ptr(), d_acc.data_ptr(), None, workers)
            torch.cuda.synchronize(dev)
            dt = (time.perf_counter() - t0) / steps
            res[label] = {"value": ntot / dt, "ms_per_step": dt * 1e3, "workers": workers or min(8, len(sizes))}
        acc = d_acc.cpu().numpy()
        rng = np.random.default_rng(9)
        errs = []
        for s in range(len(sizes)):
            a, b = int(off[s]), int(off[s + 1])
            tg = np.sort(rng.choice(b - a, min(64, b - a), replace=False)).astype(np.int64)
            ref = c.direct(pos[a:b], mass[a:b], targets=tg)
            errs.append(float(np.linalg.norm(acc[a:b][tg] - ref) / np.linalg.norm(ref)))
    line = {
        "metric": "batched ensemble particles/s (256 Plummer systems, p=8)", "value": res["concurrent"]["value"],
        "unit": UNIT, "n_gpus": 1, "steps": max(2, args.steps // 4), "warmup": max(1, args.warmup),
        "ms_per_step": res["concurrent"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer spheres)", "impl": "fmmgpu",
        "config": {"workload": f"256 independent Plummer spheres, N log-uniform in [1024, 65536] (seed 4), "
                               f"{ntot} particles, p=8, leaf capacity 64, one fmm_evaluate_batched call per step",
                   "timing": "wall clock of the call (host threads feeding worker streams)"},
        "one_stream": res["one_stream"], "speedup_concurrent": res["concurrent"]["value"] / res["one_stream"]["value"],
        "error_per_system": {"vs": "FP64 direct sum, up to 64 targets per system", "median": float(np.median(errs)),
                             "max": float(np.max(errs))},
    }
    print(json.dumps(line), flush=True)


def load_traffic():
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    of the rooflined kernels, from the committed ncu summaries: lines
    `traffic_bytes_per_launch[<name>]: <bytes>` in profiles/*.md."""
    out = {}
    pdir = os.path.join(ROOT, "profiles")
    try:
        names = sorted(os.listdir(pdir))
    except OSError:
        return out
    for fn in names:
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(pdir, fn)):
            if line.startswith("traffic_bytes_per_launch["):
                key = line[len("traffic_bytes_per_launch["):line.index("]")]
                try:
                    out[key] = float(line.split(":", 1)[1])
                except ValueError:
                    pass
    return out


# ------------------------------------------------------------- reference
def _ref_worker(args):
    n, p, leaf, seed = args[:4]
    mixture = len(args) > 4 and args[4]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "nbody-fmm_b200"))
    from oracle import RefLib
    from fmmgpu import workloads

    R = RefLib()
    pos, m = workloads.plummer_mixture(n, seed=seed) if mixture else workloads.plummer(n, seed=seed)
    t0 = time.perf_counter()
    R.fmm(pos, m, p, leaf)
    return time.perf_counter() - t0


def cpu_baseline(p, leaf, mixture=False):
    """The reference FMM::update, single thread, on a bounded sample."""
    seed = 5 if mixture else 2
    try:
        dt = _ref_worker((CPU_SAMPLE_N, p, leaf, seed, mixture))
    except Exception as e:  # reference build missing
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}
    inputs = "Plummer mixture" if mixture else "Plummer"
    return {"value": CPU_SAMPLE_N / dt, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"reference FMM::update (oracle/_ref, g++ -O2), {inputs} N={CPU_SAMPLE_N} seed {seed}, "
                      f"p={p}, leaf capacity {leaf}, 1 thread, {dt:.1f} s"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    n, p, leaf = REF_SAMPLE_N, args.p, args.leaf
    mixture = args.workload == "mixture"
    with ctx.Pool(cores) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_worker, [(n, p, leaf, 2 + i, mixture) for i in range(cores)])
        step_s = []
        for _ in range(args.steps):
            ts = pool.map(_ref_worker, [(n, p, leaf, 2 + i, mixture) for i in range(cores)])
            step_s.append(max(ts))
    total = sum(step_s)
    value = n * cores * args.steps / total
    inputs = "Plummer mixture" if mixture else "Plummer"
    sample = (f"reference FMM::update (oracle/_ref, g++ -O2) on {cores} processes x {inputs} N={n} (seeds 2..), "
              f"p={p}, leaf capacity {leaf}, one process per host core; step = slowest process")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic (seeded {'Plummer mixture' if mixture else 'Plummer sphere'})", "impl": "reference",
        "config": workload_desc(args.n, p, leaf, "reference (CPU)", mixture=mixture),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plummer", choices=["plummer", "mixture"],
                    help="plummer: the 2^20 Plummer sphere (default); mixture: the 16M clustered mixture of the "
                         "learned-order configuration, leaf capacity tuned with the threshold")
    ap.add_argument("--n", type=int, default=None, help="particles (default 2^20, mixture 2^24)")
    ap.add_argument("--p", type=int, default=12)
    ap.add_argument("--leaf", type=int, default=64)
    ap.add_argument("--m2l", default="tc", choices=["fp32", "tc"])
    ap.add_argument("--direct-max", type=int, default=-1, help="-1: the library's automatic threshold")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the library's automatic direct-pair threshold")
    ap.add_argument("--order", default="learned", choices=["learned", "fixed"],
                    help="M2L tile orders (tensor-core mode): learned by the MLP, or fixed p")
    ap.add_argument("--judge", type=int, default=512, help="learned orders: targets checked against FP64 direct")
    ap.add_argument("--judge-every", type=int, default=8, help="learned orders: check every k-th evaluation")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ensemble", action="store_true", help="the batched-ensemble configuration instead")
    ap.add_argument("--adaptive", type=int, default=0,
                    help="adaptive targets: cells under parents of at most this many particles are no targets "
                         "(0: the uniform tree of the reference)")
    ap.add_argument("--frames-every", type=int, default=0,
                    help="measure frame output instead: a device frame every K steps of the pass loop")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)
    if args.n is None:
        args.n = 1 << 24 if args.workload == "mixture" else 1 << 20
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    elif args.ensemble:
        run_ensemble(args, world, rank, local)
    elif args.frames_every > 0:
        run_frames(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
