#!/usr/bin/env python3
"""Benchmark of the exact part field's narrow-band brick bake on B200.

Workload (one step): the level bake of the brick cache (the reference's
PartCache::level, crates/icam-sim/src/partcache.rs:433) of the freeform-top part —
a 120 x 120 x 50 mm block whose top is a clamped bicubic rational B-spline with
16 x 16 control points (8 seeded Gaussian bumps, weights in [0.8, 1.2]) — at
h = 0.1 mm with a narrow band of +-2 mm (the clamp: every node within 2 mm of the
surface exact, the rest clamped), over the part's box grown by the band. A voxel is
a cell of a brick the bake reads (512 a brick). Under torchrun each rank bakes its
own part (seed = rank): weak scaling, no collective on the data path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision learned|mixed|fp64]

The headline arm (default: mixed precision with the seed network's Newton starts) is
timed beside the plain FP64 kernel and the mixed form without the network on the same
level; the line carries all three, the speed-up over FP64, and the headline level's
error against the f64 oracle (its decision whole, sampled nodes and distances).
    python bench.py --impl reference ...   # the reference's CPU path (the oracle port)

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "narrow-band SDF voxels/s, mixed+learned vs plain FP64 kernel, err ≤1e-7·diag"
H = 0.1
BAND = 2.0
# algorithmic FLOPs a node spends on one candidate of each kind (analytic face,
# B-spline span, line or arc edge, spline edge piece, vertex): foot + uv + one parity
# leg; 6 Newton steps of 750 + trim 200; closed-form foot; 6 steps of 120; a distance
FLOPS_PER_CANDIDATE = np.array([80.0, 6 * 750.0 + 200.0, 40.0, 6 * 120.0, 10.0])
# DRAM bytes the brick kernel moves a read brick: one ncu capture of the same kernel
# (mixed + learned) on the same part's level at h = 0.2 mm, 7x smaller (dram__bytes_read.sum
# 19.39 MB + dram__bytes_write.sum 49.57 MB over the 74,588 bricks that bake reads),
# scaled by the bricks read
TRAFFIC_PER_READ_BRICK = (19.390720e6 + 49.571328e6) / 74588
# the seed network's training: 50M pairs from the exact evaluator, before any timing
SEEDNET_STEPS, SEEDNET_BATCH = 12208, 4096


def set_level(h, band):
    global H, BAND
    H, BAND = h, band


def workload(seed: int, kind: str = "freeform"):
    """The part and its level's (lo, nb), over the part's whole box: the freeform top,
    or the mold cavity (its block, the pocket's floor of 500 B-spline faces, the bosses
    on its rim)."""
    from implicitcam_b200 import parts

    if kind == "mold":
        b = parts.mold(seed=seed)
        pts = np.asarray(b.verts)  # the block's corners and the bosses' caps bound it
        lo, hi = pts.min(0), pts.max(0)
    else:
        b = parts.freeform_top(seed=seed)
        # the part's box: the control net's box (the top is within its control points)
        pts = np.asarray(b.verts)
        net = np.concatenate([np.asarray(p).reshape(-1, 4) for p in b.patches])
        xyz = net[:, :3] / net[:, 3:]
        lo = np.minimum(pts.min(0), xyz.min(0))
        hi = np.maximum(pts.max(0), xyz.max(0))
    lo = lo - BAND
    nb = np.ceil((hi + BAND - lo) / (8 * H)).astype(np.int64)
    return b, lo, nb


def newton_figures(st):
    """The mixed forms' in-bake Newton work from a bake's stats: solves of sub-patches
    at the nodes, evaluations a solve (its iterations), nodes and box centres read again
    in double precision."""
    solves = st.get("newton_solves", 0)
    return {"newton_solves": solves,
            "newton_iters_per_solve": st.get("newton_evals", 0) / solves if solves else None,
            "nodes_double": st.get("nodes_double", 0), "centres_double": st.get("centres_double", 0)}


# FLOPs of one float patch evaluation and Newton step (eval_bicubic_f: the rows' and
# columns' Bernstein sums of the point and its first and second derivatives, ~600; the
# rational quotients, ~50; the 2 x 2 Newton step, ~50)
FLOPS_PER_FLOAT_EVAL = 700.0


def hbm_figure(traffic, node_ms):
    """The brick kernel's DRAM traffic over its time against the measured copy bandwidth
    (MEASURED_PEAKS.json hbm_gbs): the path is not bound by HBM; reported beside the
    FP32/FP64 roofline."""
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    gbs = traffic / (node_ms * 1e-3) / 1e9
    return {"achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak if peak else None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peak else None}


def executed_roofline(st, node_ms, peak):
    """The work the mixed walk did in the bake: its float patch evaluations (counted by
    the kernel) at FLOPS_PER_FLOAT_EVAL each, over the node phase's time, against the
    FP32 probe (None for the FP64 arm, whose evaluations are not counted)."""
    ev = st.get("newton_evals", 0)
    if not ev:
        return None
    f = FLOPS_PER_FLOAT_EVAL * ev
    return {"flops_per_launch": f, "achieved": f / (node_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
            "frac": f / (node_ms * 1e-3) / peak,
            "note": "float patch evaluations the kernel counted x 700 FLOPs, over the node phase"}


def over_ranks(dist, device, ms, voxels=None):
    """The job's figures over the ranks: the slowest rank's time (max) and every rank's
    voxels (sum); as given on one process. Every rank calls it at the same point."""
    if dist is None:
        return ms, voxels
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if voxels is None:
        return float(t.item()), None
    v = torch.tensor([voxels], device=device, dtype=torch.float64)
    dist.all_reduce(v)
    return float(t.item()), float(v.item())


def workload_name(kind):
    if kind == "mold":
        return (f"mold cavity level bake over the whole block (500 B-spline floor faces of 8x8-24x24 control "
                f"points), h={H} mm, band +-{BAND} mm")
    return f"freeform-top level bake, h={H} mm, band +-{BAND} mm"


def level_config(args, nb):
    """The level both arms (the GPU bake and the CPU reference) measure: the same dict in
    both lines. precision names the GPU line's headline arm; the CPU arm is f64 (its dtype)."""
    return {"workload": workload_name(args.workload), "part": "mold" if args.workload == "mold" else "freeform_top",
            "seed": "rank", "h_mm": H, "band_mm": BAND, "nb": [int(x) for x in nb], "precision": args.precision,
            "l2": "flushed (256 MB write) before every step"}


def sample_clocks(path):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except OSError:
        return None


def read_clocks(path, device):
    sm, mx, reasons = [], 0.0, set()
    try:
        for line in open(path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or f[0] != str(device):
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], f[5:9]):
                if v.lower() in ("active", "0x1", "1"):
                    reasons.add(name)
    except OSError:
        pass
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
            "samples": len(sm)}


def cpu_level_sample(seed, kind="freeform", target_s=8.0, threads=None, region=16):
    """The reference's CPU bake of the level (PartCache::level on the exact source:
    decide, then exact_brick for every brick to read; partcache.rs:226-331, 979-1058) as
    the oracle restates it, timed on all host cores over a random sample of the level.
    The level is cut into regions of region^3 bricks on its box grid; a region whose
    centre lies farther from the surface than its half-diagonal plus twice the band
    holds no brick to read. Regions are drawn at random from both kinds, near first,
    until target_s of CPU time is spent; in each, the oracle's decision is timed whole
    and exact_brick over up to 24 of its bricks to read, drawn uniformly; each kind's
    time and bricks to read are extrapolated to all regions of that kind. Voxels are
    counted as the GPU arm counts them: 512 for every brick the decision reads.
    Returns (voxels/s, cores, sample text)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import icam_oracle

    b, lo, nb = workload(seed, kind)
    o = icam_oracle.Oracle(b, threads=threads)
    rng = np.random.default_rng(seed + 1)
    nr = -(-nb // region)
    grid = np.stack(np.meshgrid(*[np.arange(k) for k in nr], indexing="ij"), -1).reshape(-1, 3)
    side = 8 * H * region
    centres = lo + side * (grid + 0.5)
    dcen = o.sdf(centres)[0]
    near = np.abs(dcen) <= 0.5 * side * np.sqrt(3.0) + 2 * BAND
    strata = {"near": rng.permutation(np.nonzero(near)[0]), "far": rng.permutation(np.nonzero(~near)[0])}
    acc = {k: [0.0, 0.0, 0] for k in strata}  # seconds, bricks to read, regions
    origin = lo + H  # the level's box grid (the oracle's default for the whole level)
    spent, turn = 0.0, 0
    t_start = time.perf_counter()
    while spent < target_s and any(acc[k][2] < len(strata[k]) for k in strata):
        k = "near" if (turn % 3 != 2 and acc["near"][2] < len(strata["near"])) or acc["far"][2] >= len(strata["far"]) else "far"
        turn += 1
        r = strata[k][acc[k][2]]
        lo_r = lo + side * grid[r]
        nb_r = np.minimum(region, nb - region * grid[r]).astype(np.int64)
        t0 = time.perf_counter()
        _, idx, _ = o.decide(H, lo_r, nb_r, BAND, origin=origin)
        t_dec = time.perf_counter() - t0
        t_brk = 0.0
        if len(idx):
            pick = rng.choice(idx, min(24, len(idx)), replace=False)
            firsts = lo_r + 8 * H * np.stack([pick % nb_r[0], (pick // nb_r[0]) % nb_r[1],
                                              pick // (nb_r[0] * nb_r[1])], 1)
            t0 = time.perf_counter()
            o.bricks(firsts, H, BAND)
            t_brk = (time.perf_counter() - t0) * len(idx) / len(pick)
        acc[k][0] += t_dec + t_brk
        acc[k][1] += len(idx)
        acc[k][2] += 1
        spent = time.perf_counter() - t_start
    T = sum(len(strata[k]) / a[2] * a[0] for k, a in acc.items() if a[2])
    R = sum(len(strata[k]) / a[2] * a[1] for k, a in acc.items() if a[2])
    text = (f"oracle decide + exact_brick over random {region}^3-brick regions of the level (h={H}, band={BAND}): "
            f"{acc['near'][2]} of {len(strata['near'])} near the surface, {acc['far'][2]} of {len(strata['far'])} "
            f"away from it, up to 24 bricks to read timed in each, extrapolated per region ({spent:.1f} s; "
            f"estimated {T:.0f} s for the level's ~{R:.0f} bricks to read)")
    return 512.0 * R / T, o.threads, text, T


def run_reference(args, rank, world):
    if rank != 0:
        return
    vals = []
    per_step = max(2.0, min(8.0, 100.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_level_sample(0, kind=args.workload, target_s=per_step)
    sample = ""
    bake_s = []
    for _ in range(args.steps):
        v, cores, sample, t_level = cpu_level_sample(0, kind=args.workload, target_s=per_step)
        vals.append(v)
        bake_s.append(t_level)
    value = float(np.mean(vals))
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world,
        # a step is one whole level bake, estimated from the step's sample
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(bake_s)),
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": level_config(args, workload(0, kind=args.workload)[2]),
        "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": cores, "kind": "port",
                         "sample": f"each step: {sample}"},
        "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="learned", choices=["fp64", "mixed", "learned"],
                    help="the headline arm; the plain FP64 arm is timed beside it")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--h", type=float, default=None, help="cell side (mm); smaller cases for profiling")
    ap.add_argument("--band", type=float, default=None, help="narrow band half-width (mm), the clamp")
    ap.add_argument("--workload", default="freeform", choices=["freeform", "batch", "mold", "block"],
                    help="freeform: the headline (h 0.1 mm, band 2 mm); mold: the mold cavity's pocket "
                         "(h 0.05 mm, band 1 mm); batch: 64 seeded uneven parts at h = 0.2 mm baked together; "
                         "block: the block with a hole's point queries and levels")
    ap.add_argument("--shard", action="store_true",
                    help="under torchrun: the ranks bake ONE level together (each rank a box of it, maps and "
                         "atlases all-gathered over NCCL; strong scaling) instead of a part each")
    ap.add_argument("--seednet-steps", type=int, default=SEEDNET_STEPS,
                    help="training steps of the seed network (fewer only for profiling captures)")
    args = ap.parse_args()
    dh, db = (0.05, 1.0) if args.workload == "mold" else (H, BAND)
    set_level(args.h if args.h is not None else dh, args.band if args.band is not None else db)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batch":
        return run_batch(args, rank, world)
    if args.workload == "block":
        return run_block(args, rank, world)
    if args.shard:
        return run_shard(args, rank, world, local)

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from implicitcam_b200 import part_gpu

    prec = {"fp64": part_gpu.FP64, "mixed": part_gpu.MIXED, "learned": part_gpu.MIXED_LEARNED}[args.precision]
    b, lo, nb = workload(seed=rank, kind=args.workload)
    need = BAND + 8 * H * np.sqrt(3.0)
    g = part_gpu.PartGpu(b, need=need, device=local)
    stream = torch.cuda.ExternalStream(g.stream(), device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # > L2 (126 MB)
    # the level's narrow band as the reference's decision defines it (the bricks its box
    # rule reads, partcache.rs:226-331): the voxel count of every arm and of the CPU
    # reference, read once before any timing; a bake's tighter rule reads fewer of them
    # (bricks_read_bake) with the same map and atlas
    band_bricks = int(g.decide(H, lo, nb, BAND, precision=part_gpu.FP64)[3]["bricks_read"])
    seednet = None
    if prec == part_gpu.MIXED_LEARNED:  # trained before any timing: 50M pairs from the exact evaluator
        t0 = time.perf_counter()
        loss = g.seednet_train(args.seednet_steps, batch=SEEDNET_BATCH, seed=rank, need=need)
        torch.cuda.synchronize()
        seednet = {"train_pairs": args.seednet_steps * SEEDNET_BATCH, "train_s": time.perf_counter() - t0,
                   "final_loss": float(loss[-50:].mean()), "ab": g.seednet_ab(1 << 20, seed=rank + 7, need=need)}

    def step(p, device_only=True, host=None):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if device_only:
            _, _, ns, st = g.level_device(H, lo, nb, BAND, precision=p)
        else:
            m, a = host
            ns, st = g.level_into(H, lo, nb, BAND, m, a, precision=p)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), ns, st

    def arm(p):
        """W warm-up steps, then K timed steps between barriers: (ms max over ranks,
        voxels over ranks, stats of each step)."""
        for _ in range(args.warmup):
            step(p)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms, stats = [], []
        for _ in range(args.steps):
            t, ns, st = step(p)
            ms.append(t)
            stats.append(st)
        torch.cuda.synchronize()
        total_ms, voxels = over_ranks(dist, f"cuda:{local}", float(sum(ms)), 512.0 * band_bricks)
        if dist:
            dist.barrier()
        return total_ms, voxels, stats

    clk_path = os.path.join(tempfile.gettempdir(), f"icam_clocks_{os.getpid()}.csv")
    smi = sample_clocks(clk_path) if rank == 0 else None
    total_ms, voxels, stats = arm(prec)
    # the other arms on the same level: the plain FP64 kernel (the metric's reference) and,
    # beside the learned arm, the mixed form without the seed network (what the net gains)
    others = {}
    for name, p in (("fp64", part_gpu.FP64), ("mixed", part_gpu.MIXED)):
        if p == prec or (name == "mixed" and prec != part_gpu.MIXED_LEARNED):
            continue
        o_ms, o_vox, o_stats = arm(p)
        others[name] = {"value": o_vox * args.steps / (o_ms * 1e-3), "ms_per_step": o_ms / args.steps,
                        "stage_ms": {"decide": float(np.mean([x["ms_decide"] for x in o_stats])),
                                     "nodes": float(np.mean([x["ms_nodes"] for x in o_stats])),
                                     "assemble": float(np.mean([x["ms_post"] for x in o_stats]))},
                        **newton_figures(o_stats[-1])}
    if smi:
        smi.terminate()
        smi.wait()
    value = voxels * args.steps / (total_ms * 1e-3)
    # end to end through the C ABI: the map and atlas read back into pinned host memory
    m_host = torch.empty(int(np.prod(nb)), dtype=torch.int32, pin_memory=True)
    a_host = torch.empty((max(stats[-1]["bricks_words"], 1) * part_gpu.WORDS,), dtype=torch.int32, pin_memory=True)
    e2e_ms = []
    for _ in range(max(1, args.steps)):
        t, ns, st_e = step(prec, device_only=False, host=(m_host, a_host))
        e2e_ms.append(t)
    e2e_total, _ = over_ranks(dist, f"cuda:{local}", float(sum(e2e_ms)))
    e2e_value = voxels * len(e2e_ms) / (e2e_total * 1e-3)
    m_arm = m_host.numpy().view(np.uint32).copy()
    a_arm = a_host.numpy().view(np.uint32)[: ns * part_gpu.WORDS].reshape(-1, part_gpu.WORDS).copy()
    error = None
    if rank == 0 and not args.no_cpu:
        # the checker (outside every timed region): the headline arm's level against the
        # f64 oracle, with the oracle's own decision of the whole level
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import icam_oracle

        t0 = time.perf_counter()
        orc = icam_oracle.Oracle(b)
        om, _, _ = orc.decide(H, lo, nb, BAND)
        error = verify_against_oracle(g, orc, part_gpu, lo, nb, H, BAND, prec, m_arm, a_arm, decision=om)
        if prec != part_gpu.FP64:
            m64, _, _ = g.level(H, lo, nb, BAND, precision=part_gpu.FP64, atlas=False)
            error["map_equal_to_fp64_kernel"] = bool((m64 == m_arm).all())
        error["check_s"] = time.perf_counter() - t0
    if rank == 0:
        st = stats[-1]
        node_ms = float(np.mean([s["ms_nodes"] for s in stats]))
        census = np.array(st["census"], dtype=np.float64)
        flops = 729.0 * float(census @ FLOPS_PER_CANDIDATE)
        peak = g.probe_fma(part_gpu.FP64 if prec == part_gpu.FP64 else part_gpu.MIXED)
        achieved = flops / (node_ms * 1e-3)
        cpu = None
        if not args.no_cpu and world == 1:
            v, cores, sample, _ = cpu_level_sample(0, kind=args.workload, target_s=12.0)
            cpu = {"value": v, "unit": "voxels/s", "cores": cores, "kind": "port", "sample": sample}
        clocks = read_clocks(clk_path, local)
        out = {
            "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == part_gpu.FP64 else "f32+f64",
            "data": "synthetic",
            "config": level_config(args, nb),
            "speedup_vs_fp64": value / others["fp64"]["value"] if "fp64" in others else None,
            "fp64": others.get("fp64"), "mixed": others.get("mixed"), "error_vs_oracle": error, "seednet": seednet,
            "bricks_read": band_bricks, "bricks_read_bake": st["bricks_read"], "bricks_stored": st["bricks_words"],
            "bricks_settled": st["bricks_settled"],
            "nodes_exact": st["nodes_exact"], "nodes_undecided": st["nodes_undecided"],
            **newton_figures(st),
            "nodes_exact_per_s": st["nodes_exact"] * args.steps / (total_ms * 1e-3),
            "stage_ms": {"decide": st["ms_decide"], "nodes": st["ms_nodes"], "assemble": st["ms_post"]},
            "gpu_launches": int(st["kernel_launches"]) * args.steps,
            "e2e": {"value": e2e_value, "unit": "voxels/s", "h2d_bytes_per_step": st_e["h2d_bytes"],
                    "d2h_bytes_per_step": st_e["d2h_bytes"]},
            "roofline": {"bound": "fp64" if prec == part_gpu.FP64 else "fp32", "kernel": "k_bricks",
                         "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": TRAFFIC_PER_READ_BRICK * st["bricks_read"],
                         "traffic_source": "ncu dram bytes of k_bricks at h = 0.2 mm, scaled by bricks read",
                         "peak_source": "measured FMA probe of this run (MEASURED_PEAKS.json holds no FP64/FP32 figure)",
                         "algorithmic_flops_per_launch": flops,
                         "executed": executed_roofline(st, node_ms, peak),
                         "hbm": hbm_figure(TRAFFIC_PER_READ_BRICK * st["bricks_read"], node_ms)},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    g.close()
    if dist:
        dist.destroy_process_group()


def run_shard(args, rank, world, local):
    """One level (the freeform part of seed 0 or the mold's pocket) baked by all ranks
    together (implicitcam_b200/shard.py): the level cut once into a box a rank by k-d
    bisection of its first-box tiles weighted by the surface within their reach; each
    step every rank bakes its box, reads it into device tensors, all-gathers the maps and
    atlases over NCCL and assembles the whole level. Strong scaling: the level is fixed.
    The step's time is the slowest rank's, CUDA events around the step on torch's stream
    (the bake itself returns when its stream is done)."""
    import datetime

    import torch
    import torch.distributed as dist

    from implicitcam_b200 import part_gpu, shard

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    prec = {"fp64": part_gpu.FP64, "mixed": part_gpu.MIXED, "learned": part_gpu.MIXED_LEARNED}[args.precision]
    b, lo, nb = workload(seed=0, kind=args.workload)
    need = BAND + 8 * H * np.sqrt(3.0)
    g = part_gpu.PartGpu(b, need=need, device=local)
    if prec == part_gpu.MIXED_LEARNED:  # every rank trains the same net (same seed)
        g.seednet_train(args.seednet_steps, batch=SEEDNET_BATCH, seed=0, need=need)
    size, start, dims = shard.tile_grid(H, lo, nb)
    w = shard.tile_weights(lambda p: g.points(p)[0], H, lo, nb, BAND)
    boxes = shard.plan(w, size, start, nb, world)
    org = shard.level_origin(H, lo)
    lo_r, nb_r = shard.sub_level(H, lo, boxes[rank])
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if (nb_r > 0).all():
            mr, ar = g.level_torch(H, lo_r, nb_r, BAND, origin=org, precision=prec)
        else:
            mr = torch.zeros(0, dtype=torch.int32, device=dev)
            ar = torch.zeros((0, part_gpu.WORDS), dtype=torch.int32, device=dev)
        if world > 1:
            maps, atlases = shard.exchange(dist, boxes, mr, ar)
        else:
            maps, atlases = [mr], [ar]
        M, A = shard.assemble(nb, boxes, maps, atlases)
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1), M, A

    for _ in range(args.warmup):
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms = 0.0
    for _ in range(args.steps):
        t, M, A = step()
        ms += t
    torch.cuda.synchronize()
    bricks_read = int(g.decide(H, lo, nb, BAND, precision=prec)[3]["bricks_read"])
    total_ms, _ = over_ranks(dist if world > 1 else None, dev, ms)
    if rank == 0:
        out = {"metric": METRIC, "value": 512.0 * bricks_read * args.steps / (total_ms * 1e-3), "unit": "voxels/s",
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
               "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
               "dtype": "f64" if prec == part_gpu.FP64 else "f32+f64", "data": "synthetic",
               "config": {"workload": workload_name(args.workload) + ", one level over all ranks",
                          "h_mm": H, "band_mm": BAND, "nb": nb.tolist(), "precision": args.precision,
                          "parallelism": f"level cut into {world} boxes, maps and atlases all-gathered",
                          "l2": "flushed (256 MB write) before every step"},
               "boxes": [[b0.tolist(), b1.tolist()] for b0, b1 in boxes],
               "stored_bricks": int(A.shape[0]), "gpu_launches": None}
        print(json.dumps(out), flush=True)
    g.close()
    if world > 1:
        dist.destroy_process_group()


def batch_parts(seed0=0, count=64):
    """Uneven seeded parts of four families, a quarter each: blocks with rational
    B-spline tops of 4 x 4 to 32 x 32 control points, degree 2 or 3, weights U[0.7, 1.3],
    cut along their knot lines into 1 to 19 faces a side (6 to 366 faces), 20-120 mm
    sides; plates with one to four filleted bosses (cylinder, torus fillet, plane cap;
    9 to 18 faces); blocks with countersunk holes (cylinder and cone; 8 faces); plates with
    one to four spherical domes (cylinder under a hemisphere; 8 to 14 faces).
    Returns [(family, solid)]."""
    from implicitcam_b200 import parts

    out = []
    for k in range(count):
        f = k % 4
        s = seed0 + k
        if f == 0:  # the j-th of the family: control points and faces grow with j
            j = k // 4
            n = 4 + (28 * j) // 15
            deg = 2 + j % 2
            out.append(("freeform_top", parts.freeform_patches(
                seed=s, n=n, size=20.0 + (37 * k) % 100, base=10.0 + (13 * k) % 40, bumps=2 + k % 7, degree=deg,
                faces=1 + (18 * j) // 15)))
        elif f == 1:
            m = 1 + (k // 4) % 4
            out.append(("boss", parts.bodies_on_plate(seed=s, kind="boss", count=m,
                                                      plate=(12.0 * m + (3 * k) % 10, 14.0 + (5 * k) % 9, 4.0 + k % 5))))
        elif f == 2:
            X, Y, Z = 20.0 + (11 * k) % 80, 15.0 + (7 * k) % 50, 10.0 + (5 * k) % 30
            r = 0.12 * min(X, Y)
            out.append(("countersunk_block", parts.countersunk_block(
                size=(X, Y, Z), center=(X / 2, Y / 2), r=r, sink=min(0.4 * r, 0.3 * Z))))
        else:
            m = 1 + (k // 4) % 4
            out.append(("dome", parts.bodies_on_plate(seed=s, kind="dome", count=m,
                                                      plate=(12.0 * m + (3 * k) % 10, 14.0 + (5 * k) % 9, 4.0 + k % 5))))
    return out


def run_batch(args, rank, world):
    """64 uneven parts at h = 0.2 mm, band 1 mm, baked as one batch (one brick launch,
    a replayed graph, autotuned tiling) in each arithmetic (FP64, mixed, mixed with the
    seed network's starts, each part's net trained briefly first), and the headline arm
    one part at a time; wall time of the synchronous calls. The headline arm's maps and
    atlases of one part of each family are checked against the f64 oracle."""
    import torch

    from implicitcam_b200 import part_gpu

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    h, band = 0.2, 1.0
    precs = {"fp64": part_gpu.FP64, "mixed": part_gpu.MIXED, "learned": part_gpu.MIXED_LEARNED}
    prec = precs[args.precision]
    gs, levels, faces, fams, solids = [], [], [], [], []
    for fam, solid in batch_parts(seed0=64 * rank):
        # certificates for points within the band (a node reads a sub-patch only nearer
        # than the clamp); the brick-wide margin would split these curved tops far deeper
        g = part_gpu.PartGpu(solid, need=band)
        lo, hi = g.box()
        lo2 = lo - band
        nb = np.ceil((hi - lo + 2 * band) / (8 * h)).astype(np.int64)
        gs.append(g)
        levels.append((h, lo2, nb, band))
        faces.append(g.info()["faces"])
        fams.append(fam)
        solids.append(solid)
    t0 = time.perf_counter()
    for i, g in enumerate(gs):  # the seed networks, before any timing (1500 steps of 2048 pairs)
        if g.info()["subs"] > 0:  # a part without B-spline faces has nothing to seed
            g.seednet_train(1500, batch=2048, seed=i, need=band)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    batch = part_gpu.Batch(gs)
    # the parts' narrow bands as the reference's decision defines them (their voxel count)
    band_bricks = sum(int(g.decide(*L, precision=part_gpu.FP64)[3]["bricks_read"]) for g, L in zip(gs, levels))

    def timed(p):
        for _ in range(args.warmup):
            batch.bake(levels, precision=p, read=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            st, _ = batch.bake(levels, precision=p, read=False)
        return (time.perf_counter() - t0) / args.steps, st

    arms = {}
    for name, p in precs.items():
        t, st = timed(p)
        arms[name] = {"ms_per_step": 1e3 * t, "value": 512.0 * band_bricks / t,
                      "ms_decide": st["ms_decide"], "ms_bricks": st["ms_bricks"], "warps": st["warps"],
                      "graph_replayed": st["graph_replayed"]}
    t_batch, st = timed(prec)
    for g, L in zip(gs, levels):  # one part at a time, warm
        g.level_device(*L, precision=prec)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    per_part = []
    for _ in range(args.steps):
        for g, L in zip(gs, levels):
            _, _, _, s1 = g.level_device(*L, precision=prec)
            if len(per_part) < len(gs):
                per_part.append(s1["bricks_read"])
    t_alone = (time.perf_counter() - t0) / args.steps
    voxels = 512.0 * band_bricks
    error = None
    if rank == 0 and not args.no_cpu:
        # the checker, outside every timed region: one part of each family
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import icam_oracle

        _, res = batch.bake(levels, precision=prec, read=True)
        error = {}
        for fam in sorted(set(fams)):
            i = fams.index(fam)
            orc = icam_oracle.Oracle(solids[i])
            hh, lo2, nb, clamp = levels[i]
            om, _, _ = orc.decide(hh, lo2, nb, clamp)
            m, a = res[i]
            r = verify_against_oracle(gs[i], orc, part_gpu, lo2, nb, hh, clamp, prec, m, a, n_bricks=200,
                                      n_centres=100, decision=om)
            error[fam] = {k: r[k] for k in ("i16_max_step_diff", "sign_flips", "distance_max_over_diag",
                                           "decided_entries_differ", "stored_outside_read_set",
                                           "air_solid_centres_wrong", "nodes_checked") if k in r}
            error[fam]["part"] = i
    if rank == 0:
        out = {"metric": "batched uneven parts: narrow-band SDF voxels/s", "value": voxels / t_batch,
               "unit": "voxels/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": 1e3 * t_batch, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64" if prec == part_gpu.FP64 else "f32+f64", "data": "synthetic",
               "timing": "wall time of the synchronous bake calls",
               "config": {"workload": f"64 seeded uneven parts, h={h} mm, band +-{band} mm", "parts": len(gs),
                          "faces_min_max": [min(faces), max(faces)],
                          "bricks_read_min_max": [min(per_part), max(per_part)], "precision": args.precision},
               "arms": arms, "speedup_vs_fp64": arms["fp64"]["ms_per_step"] / (1e3 * t_batch),
               "seednet_train_s": train_s,
               "one_part_at_a_time": {"value": voxels / t_alone, "ms_per_step": 1e3 * t_alone},
               "speedup_vs_one_at_a_time": t_alone / t_batch,
               "families": {fam: {"parts": fams.count(fam),
                                  "faces": sum(n for n, f in zip(faces, fams) if f == fam),
                                  "bricks_read": sum(n for n, f in zip(per_part, fams) if f == fam)}
                            for fam in sorted(set(fams))},
               "error_vs_oracle": error,
               "batch_stats": {k: st[k] for k in ("bricks_read", "bricks_words", "warps", "graph_replayed",
                                                  "tune_ms", "ms_decide", "ms_bricks", "kernel_launches")}}
        print(json.dumps(out), flush=True)
    batch.close()
    for g in gs:
        g.close()


def run_block(args, rank, world):
    """The block with a hole (100 x 60 x 40 mm minus a 20 mm hole): 10^6 point queries
    uniform over the box grown by 10 mm (the reference checker's generator, seed 0)
    through icam_points, and the level over the part's box from (0, 0, 0) at h = 0.5 mm
    (25 x 15 x 10 bricks) and h = 1 mm, clamp a cell's diagonal; the oracle on the host's
    cores beside them. One process (the part is small)."""
    import torch

    from implicitcam_b200 import part_gpu, parts

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import icam_oracle

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    prec = {"fp64": part_gpu.FP64, "mixed": part_gpu.MIXED, "learned": part_gpu.MIXED}[args.precision]
    b = parts.block_with_hole()
    g = part_gpu.PartGpu(b)
    rng = parts.Rng(0)
    n = 1_000_000
    lo_q, hi_q = np.array([-10.0, -10.0, -10.0]), np.array([110.0, 70.0, 50.0])
    q = np.array([[rng.uniform(lo_q[k], hi_q[k]) for k in range(3)] for _ in range(n)])
    stream = torch.cuda.ExternalStream(g.stream())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    for _ in range(args.warmup):
        g.points(q[:100000])
    ms = [timed(lambda: g.points(q))[0] for _ in range(args.steps)]
    q_per_s = n / (np.mean(ms) * 1e-3)
    bakes = {}
    for h in (0.5, 1.0):
        nb = np.ceil(np.array([100.0, 60.0, 40.0]) / (8 * h)).astype(np.int64)
        lo = np.zeros(3)
        for _ in range(args.warmup):
            g.level_device(h, lo, nb, precision=prec)
        res = [timed(lambda: g.level_device(h, lo, nb, precision=prec)) for _ in range(args.steps)]
        t = float(np.mean([r[0] for r in res]))
        st = res[-1][1][3]
        bakes[f"h{h}"] = {"nb": nb.tolist(), "bricks": int(np.prod(nb)), "bricks_read": st["bricks_read"],
                          "bricks_stored": st["bricks_words"], "ms": t,
                          "voxels_per_s": 512.0 * st["bricks_read"] / (t * 1e-3),
                          "level_cells_per_s": 512.0 * float(np.prod(nb)) / (t * 1e-3)}
    o = icam_oracle.Oracle(b)
    sample = q[:: n // 20000]
    t0 = time.perf_counter()
    o.sdf(sample)
    cpu_q = len(sample) / (time.perf_counter() - t0)
    nb1 = np.ceil(np.array([100.0, 60.0, 40.0]) / 8.0).astype(np.int64)
    t0 = time.perf_counter()
    om, idx, dc = o.decide(1.0, np.zeros(3), nb1, np.sqrt(3.0))
    firsts = np.stack([8.0 * (idx % nb1[0]), 8.0 * ((idx // nb1[0]) % nb1[1]), 8.0 * (idx // (nb1[0] * nb1[1]))], 1)
    o.bricks(firsts.astype(np.float64), 1.0, np.sqrt(3.0))
    cpu_bake = time.perf_counter() - t0
    if rank == 0:
        print(json.dumps({
            "metric": "block with hole: exact signed-distance point queries/s (end to end through icam_points)",
            "value": q_per_s, "unit": "queries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == part_gpu.FP64 else "f32+f64", "data": "synthetic",
            "config": {"workload": "block 100x60x40 mm minus a 20 mm hole: 1e6 uniform queries over the box "
                                   "grown by 10 mm (seed 0), levels at h 0.5 and 1 mm", "precision": args.precision,
                       "l2": "flushed (256 MB write) before every step"},
            "e2e": {"value": q_per_s, "unit": "queries/s", "h2d_bytes_per_step": n * 24,
                    "d2h_bytes_per_step": n * 9},
            "bakes": bakes,
            "cpu_baseline": {"queries_per_s": cpu_q, "cores": o.threads, "kind": "port",
                             "sample": f"{len(sample)} of the queries; the h = 1 mm level (decision and every read "
                                       f"brick) in {cpu_bake:.2f} s",
                             "level_h1_s": cpu_bake},
        }), flush=True)
    g.close()


def brick_firsts(ids, lo, nb, h):
    """First nodes of bricks given by level index (x fastest)."""
    ids = np.asarray(ids, dtype=np.int64)
    return np.stack([lo[0] + 8 * h * (ids % nb[0]), lo[1] + 8 * h * ((ids // nb[0]) % nb[1]),
                     lo[2] + 8 * h * (ids // (nb[0] * nb[1]))], 1)


def node_points(ids, nodes, lo, nb, h):
    """Positions of nodes (0..728, x fastest) of bricks given by level index."""
    f = brick_firsts(ids, lo, nb, h)
    nodes = np.asarray(nodes, dtype=np.int64)
    return f + h * np.stack([nodes % 9, (nodes // 9) % 9, nodes // 81], 1)


def verify_against_oracle(g, oracle, part_gpu, lo, nb, h, clamp, precision, m, a, n_bricks=1000, every=29,
                          n_centres=300, seed=0, decision=None):
    """A baked level against the f64 oracle, as the reference's PartCache::verify does
    it (partcache.rs:508-543; every 29th node, icam-sim main.rs:959): every `every`th
    node of n_bricks random stored bricks, plus every node of every stored brick whose
    i16 value lies within one step of zero (where the signs are decided), plus the
    centres of random air and material bricks; the distances before quantisation of the
    sampled bricks' nodes (icam_bricks in the same precision) against the oracle's.
    With `decision` (the oracle's map from its decide), the bake's air and material
    entries outside the read set are checked against it whole."""
    rng = np.random.default_rng(seed)
    diag = float(np.linalg.norm(np.asarray(oracle.bbox()[1]) - np.asarray(oracle.bbox()[0])))
    stored = np.nonzero(m < 0xFFFFFFF0)[0]
    out = {"stored_bricks": int(len(stored))}
    # every node within one i16 step of zero, over every stored brick (chunks of the atlas)
    near_ids, near_nodes, near_q = [], [], []
    for c0 in range(0, len(stored), 20000):
        ids = stored[c0:c0 + 20000]
        q = part_gpu.unpack_atlas(a[m[ids]]).astype(np.int64)
        bi, ni = np.nonzero(np.abs(q) <= 1)
        near_ids.append(ids[bi])
        near_nodes.append(ni)
        near_q.append(q[bi, ni])
    near_ids, near_nodes, near_q = (np.concatenate(x) if x else np.zeros(0, np.int64)
                                    for x in (near_ids, near_nodes, near_q))
    pick = rng.choice(stored, min(n_bricks, len(stored)), replace=False) if len(stored) else stored
    nodes = np.arange(0, 729, every)
    s_ids = np.repeat(pick, len(nodes))
    s_nodes = np.tile(nodes, len(pick))
    s_q = part_gpu.unpack_atlas(a[m[pick]]).astype(np.int64)[:, nodes].reshape(-1) if len(pick) else s_ids
    ids = np.concatenate([near_ids, s_ids])
    nn = np.concatenate([near_nodes, s_nodes])
    qs = np.concatenate([near_q, s_q])
    d = oracle.sdf(node_points(ids, nn, lo, nb, h))[0] if len(ids) else np.zeros(0)
    qo = np.round(np.clip(d / clamp, -1.0, 1.0) * 32767.0).astype(np.int64)
    off = np.abs(qo - qs)
    flips = int(((qs > 0) & (qo < 0)).sum() + ((qs < 0) & (qo > 0)).sum())
    out.update({"nodes_checked": int(len(ids)), "nodes_near_zero": int(len(near_ids)),
                "i16_max_step_diff": int(off.max()) if len(off) else 0, "i16_nodes_off": int((off > 0).sum()),
                "sign_flips": flips})
    # distances before quantisation on the sampled bricks
    if len(pick):
        sub = pick[: min(len(pick), 256)]
        vals, dg = g.bricks(brick_firsts(sub, lo, nb, h), h, clamp, precision=precision)
        do = oracle.sdf(node_points(np.repeat(sub, len(nodes)), np.tile(nodes, len(sub)), lo, nb, h))[0]
        dgs = dg[:, nodes].reshape(-1)
        fl = vals[:, nodes, 1].reshape(-1)
        ex = fl == 0
        err = np.abs(dgs[ex] - do[ex])
        sg = ex & (np.abs(do) > 1e-9)  # signs above double rounding
        out.update({"distance_max_abs_mm": float(err.max()) if len(err) else 0.0,
                    "distance_max_over_diag": float(err.max() / diag) if len(err) else 0.0,
                    "distance_sign_flips": int(((dgs[sg] > 0) & (do[sg] < 0)).sum() + ((dgs[sg] < 0) & (do[sg] > 0)).sum()),
                    "flags_past_clamp_ok": bool((np.abs(do[fl == 1]) >= clamp * (1 - 1e-12)).all()),
                    "flags_undecided": int((fl == 2).sum())})
    # air and material bricks: the centre on the right side
    bad = 0
    for val in (part_gpu.AIR, part_gpu.SOLID):
        cand = np.nonzero(m == val)[0]
        if len(cand):
            ids2 = rng.choice(cand, min(n_centres, len(cand)), replace=False)
            dc = oracle.sdf(brick_firsts(ids2, lo, nb, h) + 4 * h)[0]
            bad += int(((dc > 0) != (val == part_gpu.AIR)).sum())
    out["air_solid_centres_wrong"] = bad
    if decision is not None:
        dec = decision != part_gpu.READ
        out["decided_entries_differ"] = int((m[dec] != decision[dec]).sum())
        out["stored_outside_read_set"] = int((m[dec] < 0xFFFFFFF0).sum())
    out["sample"] = (f"every {every}th node of {len(pick)} random stored bricks, every node within an i16 step "
                     f"of zero ({len(near_ids)}), {n_centres} centres of air and of material bricks; distances on "
                     f"{min(len(pick), 256)} of the sampled bricks")
    return out


if __name__ == "__main__":
    main()
