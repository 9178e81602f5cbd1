#!/usr/bin/env python3
"""Benchmark: Mrays/s and build+trace+shade ms/frame on one B200 per rank.

Workload (default): the animated 64-part scene (~200k triangles) at 1280x720.
One step = one animation frame through the engine: rigid transform + scene
box + triangle records, GPU SAH KD-tree build, primary rays, shadow rays,
shading -- captured once as a CUDA graph and replayed per frame with that
frame's matrices. Rays counted = primary + shadow rays traced.

value   : device time (CUDA events on the frame's stream), scene resident in
          HBM, L2 flushed (256 MB write) between frames.
e2e     : the same frames through the C ABI with host inputs, timed by the
          host clock: per frame a synchronise, then the call (part matrices,
          camera and lights copied from pinned host memory), the image read
          back to pinned host memory and a final synchronise, all inside the
          timed span; the L2 flush stays outside it.
compare : the metric's comparison, on rank 0 over the same frames: the GPU
          engine with the 32-bin binned SAH (the headline), with the learned
          split proposer, and with the exact SAH on nodes of up to 1024
          references ("exact"), each with build ms, trace + shade ms, ms per
          frame and the SAH cost of one frame's tree (hk_tree_cost), against
          the cost of the reference's own SAH-NlogN tree of that frame (the
          compiled reference with the same constants, from the CPU-baseline
          leg), plus learned_speedup_vs_exact and learned_cost_vs_exact.
roofline: the trace kernel (primary rays) on the last frame's tree:
          algorithmic bytes per ray 32 + 8 + 8 N_node + 4 N_ref + 36 N_tri with
          the per-ray counts measured by the kernel's counting mode.
Multi-GPU: frames are sharded across ranks (rank r renders frames r, r+N, ...)
with no data-path collective; the barrier / max-over-ranks timing uses NCCL.

--impl reference: the reference's own CPU path (KDTreeCPU SAH-NlogN build +
checkCollision shading loop, compiled from its sources into oracle/_ref) on the
host cores for the same frames.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="animated", choices=["animated", "static_small", "static_large", "aff"])
    ap.add_argument("--aff", help="aff workload: an AFF (BART) scene file, animated on the reference's fixed-tick clock")
    ap.add_argument("--mode", default="binned", choices=["binned", "learned"])
    ap.add_argument("--variant", default="auto",
                    help="traversal variant, or auto: hk_autotune picks variant, block size and stack depth")
    ap.add_argument("--exact-max", type=int, default=0,
                    help="exact SAH on nodes of at most this many references (0: 32-bin binned SAH everywhere)")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "hulktracer_b200",
                                                      "weights", "proposer.bin"),
                    help="trained proposer weights (learned mode)")
    ap.add_argument("--layout", type=int, nargs=3, metavar=("SUBTREE_MAX", "SUBTREE_DEPTH", "LEVEL_STREAMS"),
                    help="builder layout (hk_config subtree_max, subtree_depth, level_streams) instead of "
                         "hk_autotune_build")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the learned / exact comparison arms")
    ap.add_argument("--cost-frame", type=int, default=17, help="frame whose trees are costed in the comparison")
    ap.add_argument("--cpu-frames", type=int, default=2)
    ap.add_argument("--split", default="frames", choices=["frames", "rays"],
                    help="multi-GPU split: whole frames per rank (default), or row bands of every frame "
                         "gathered over NCCL (the build replicated on every rank)")
    return ap.parse_args()


def make_scene(name, aff_path=None):
    from hulktracer_b200 import scenes
    if name == "aff":
        if not aff_path:
            raise SystemExit("--workload aff needs --aff <scene file>")
        return scenes.from_aff(aff_path)
    if name == "animated":
        return scenes.animated_parts()
    if name == "static_small":
        return scenes.static_small()
    return scenes.static_large()


def workload_name(sc):
    rays = "primary+mirror+shadow" if "mirror" in sc.extra else "primary+shadow"
    return "%s %d tris %dx%d %s" % (sc.name, sc.ntris, sc.width, sc.height, rays)


def traffic_tag(sc):
    return {"animated_parts_200k": "animated200k"}.get(sc.name, sc.name)


def frame_mats(sc, f):
    from hulktracer_b200 import scenes
    if sc.part_center is None:
        return None
    return scenes.part_matrices(sc, f)


def frame_cam(sc, f):
    from hulktracer_b200 import scenes
    return scenes.frame_camera(sc, f)


def data_desc(sc):
    if "aff" in sc.extra:
        return "AFF scene file %s (keyframes on the fixed-tick clock)" % sc.name[4:]
    return "synthetic (seeded procedural scene)"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.rows.append([x.strip() for x in ln.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference compiled from its sources
# ---------------------------------------------------------------------------
def reference_frame(R, O, sc, f, prim, nthreads):
    """One frame of the reference CPU visitor (GLVisitorCPUTrace::traverseBegin):
    rigid transform of the vertices, KDTreeCPU::buildKDTree, traceScene.
    Returns (seconds, rays)."""
    t0 = time.perf_counter()
    if prim is None:   # a moving camera
        from oracle.oracle import NORM_IEEE
        prim = O.camera_rays(frame_cam(sc, f), sc.width, sc.height, NORM_IEEE)
    mats = frame_mats(sc, f)
    if mats is not None:
        verts = O.transform(sc.rest_verts, sc.part_of_vertex, mats)
    else:
        verts = sc.verts
    box = O.scene_box(verts)
    R.set_vertices(verts, box)
    R.build()
    img = R.render(prim, sc.width, sc.height, sc.lights, nthreads=nthreads)
    dt = time.perf_counter() - t0
    nhit = int((img != 0).sum())
    npoint = int((sc.lights[:, 3] == 1.0).sum())
    return dt, sc.width * sc.height + nhit * npoint


def reference_tree(sc, frame):
    """The reference's own SAH-NlogN tree of one frame, built by the compiled
    reference with the benchmark constants (Ct 1, Ci 1.5, depth 24, leaves of
    at most 4, no subsampling): (nodes4, refs, verts, box), or None."""
    from oracle.oracle import Oracle, Reference
    if not Reference.available(cfg=True):
        return None
    O = Oracle()
    mats = frame_mats(sc, frame)
    verts = O.transform(sc.rest_verts, sc.part_of_vertex, mats) if mats is not None else sc.verts
    box = O.scene_box(verts)
    R = Reference(cfg=True)
    R.load(verts, sc.tris, box)
    nodes, refs, _ = R.build()
    return nodes, refs, verts, box


def cpu_baseline(sc, frames, nthreads):
    from oracle.oracle import NORM_IEEE, Oracle, Reference
    O = Oracle()
    if Reference.available():
        R = Reference()
        kind = "reference"
    else:
        return None
    prim = None if "aff" in sc.extra else O.camera_rays(sc.camera, sc.width, sc.height, NORM_IEEE)
    R.load(sc.verts, sc.tris, sc.scene_box())
    reference_frame(R, O, sc, 0, prim, nthreads)   # warm-up (page-in, OpenMP pool)
    tot_t, tot_r = 0.0, 0
    for f in range(frames):
        dt, r = reference_frame(R, O, sc, f + 1, prim, nthreads)
        tot_t += dt
        tot_r += r
    return {"value": tot_r / tot_t / 1e6, "unit": "Mrays/s", "cores": nthreads, "kind": kind,
            "sample": "%d full frames (CPU transform + SAH-NlogN build + shaded trace), %d threads" % (frames, nthreads),
            "ms_per_frame": 1000.0 * tot_t / frames}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc = make_scene(args.workload, args.aff)
    nthreads = os.cpu_count() or 1
    from oracle.oracle import NORM_IEEE, Oracle, Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent when building)"}))
        return
    O = Oracle()
    R = Reference()
    prim = None if "aff" in sc.extra else O.camera_rays(sc.camera, sc.width, sc.height, NORM_IEEE)
    R.load(sc.verts, sc.tris, sc.scene_box())
    for f in range(args.warmup):
        reference_frame(R, O, sc, f, prim, nthreads)
    tot_t, tot_r = 0.0, 0
    for i in range(args.steps):
        dt, r = reference_frame(R, O, sc, args.warmup + i, prim, nthreads)
        tot_t += dt
        tot_r += r
    v = tot_r / tot_t / 1e6
    line = {"metric": "Mrays/s (build+trace+shade per frame)", "value": v, "unit": "Mrays/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * tot_t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": data_desc(sc),
            "config": {"workload": workload_name(sc), "build": "reference SAH-NlogN (CPU)",
                       "parallelism": "OpenMP rows, %d threads" % nthreads},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": nthreads, "kind": "reference",
                             "sample": "%d full frames per step" % 1},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our engine
# ---------------------------------------------------------------------------
def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def run_ours(args):
    import torch
    import torch.distributed as dist
    import hulktracer_b200 as hk
    from hulktracer_b200.shard import frames_for_rank, gather_rows, reduce_job, rows_for_rank

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    sc = make_scene(args.workload, args.aff)
    W, H = sc.width, sc.height
    variant = hk.VARIANTS.get(args.variant, hk.ROPES)
    mode = hk.BUILD_LEARNED if args.mode == "learned" else hk.BUILD_BINNED
    stream = torch.cuda.Stream()
    ctx = hk.Context(device=local, exact_max=args.exact_max)
    ctx.set_stream(stream.cuda_stream)
    if mode == hk.BUILD_LEARNED:
        ctx.mlp_load(args.weights)
    ctx.upload(sc.verts, sc.tris)
    animated = sc.part_of_vertex is not None
    if animated:
        ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    if "mirror" in sc.extra:
        # the large static scene: one mirror bounce on 30% of the triangles
        ctx.set_mirrors(sc.extra["mirror"])
        ctx.set_frame_shading(hk.SHADE_MIRROR)
    tuned = None
    if args.variant == "auto":
        # hk_autotune (untimed setup): traversal layout, block size and stack
        # depth timed on the first frame's primary rays of this scene and tree
        m0 = frame_mats(sc, 0)
        if m0 is not None:
            ctx.transform(m0)
        else:
            ctx.precompute()
        ctx.build(mode)
        d_rays = torch.from_numpy(ctx.camera_rays(frame_cam(sc, 0), W, H)).cuda()
        tuned = ctx.autotune(d_rays.data_ptr(), W * H)
        variant = tuned["variant"]
        del d_rays
    # hk_autotune_build (untimed setup): the builder layout on this scene
    m0 = frame_mats(sc, 0)
    if m0 is not None:
        ctx.transform(m0)
    else:
        ctx.precompute()
    if args.layout:
        ctx.set_build_layout(*args.layout)
        build_tuned = dict(zip(("subtree_max", "subtree_depth", "level_streams"), args.layout), tried=0)
    else:
        build_tuned = ctx.autotune_build(mode)
    rgba = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    rays_split = args.split == "rays"
    # rays split: every rank takes part in every frame with its band of rows
    frames = frames_for_rank(args.warmup, args.steps, 0 if rays_split else rank, 1 if rays_split else world)
    y0, y1 = rows_for_rank(H, rank, world) if rays_split else (0, H)
    band = torch.zeros(W * (y1 - y0), dtype=torch.int32, device="cuda")
    mats_all = {f: frame_mats(sc, f) for f in list(range(args.warmup)) + frames}
    # pinned host inputs / outputs for the e2e leg
    pin_mats = {f: (torch.from_numpy(m).pin_memory() if m is not None else None) for f, m in mats_all.items()}
    pin_img = torch.empty(W * H, dtype=torch.int32).pin_memory()

    def do_frame(f, use_graph=True):
        m = pin_mats[f]
        if not rays_split:
            ctx.frame(m.numpy() if m is not None else None, frame_cam(sc, f), sc.lights, W, H, rgba.data_ptr(), mode,
                      variant, use_graph)
            return
        # this rank's band of the frame on its own replica, then the gather
        if m is not None:
            ctx.transform(m.numpy())
        ctx._check(ctx.L.hk_build(ctx.h, mode, None))
        ctx.render_rows_device(frame_cam(sc, f), sc.lights, W, H, y0, y1, band.data_ptr(), variant,
                               hk.SHADE_MIRROR if "mirror" in sc.extra else hk.SHADE_CPU)
        rgba.copy_(gather_rows(band, rank, world, W, H))

    with torch.cuda.stream(stream):
        for f in range(args.warmup):
            do_frame(f)
        stream.synchronize()
        ctx.synchronize()
        kern_nodes, all_nodes = ctx.graph_info()
        # ---- device-timed frames ----
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in frames]
        rays = 0
        for (e0, e1), f in zip(ev, frames):
            flush.zero_()
            e0.record(stream)
            do_frame(f)
            e1.record(stream)
            p, s = ctx.ray_counts()   # synchronises after the end event (outside the timed span)
            rays += p + s
        torch.cuda.synchronize()
        cl = clocks.stop()
        t_dev = sum(e0.elapsed_time(e1) for e0, e1 in ev) / 1000.0
        # ---- e2e: host inputs in, image out, through the C ABI, host clock ----
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t_e2e = 0.0
        for f in frames:
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            do_frame(f)
            pin_img.copy_(rgba, non_blocking=True)
            stream.synchronize()
            t_e2e += time.perf_counter() - t0

    # ---- max over ranks ----
    (t_dev, t_e2e), total_rays = reduce_job([t_dev, t_e2e], rays, world, device="cuda")

    # ---- roofline of the trace kernel (rank 0) ----
    roof = None
    if rank == 0:
        roof = trace_roofline(ctx, sc, stream, variant)

    base = None
    ref_cost = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(sc, args.cpu_frames, os.cpu_count() or 1)
        if args.workload == "animated" and not args.no_compare:
            rt = reference_tree(sc, args.cost_frame)
            if rt is not None:
                ref_cost = reference_tree_cost(hk, rt, local)

    compare = None
    if rank == 0 and not args.no_compare and args.workload == "animated":
        compare = compare_arms(args, sc, local, ref_cost, variant, tuned)

    if rank == 0:
        nl = sc.lights.shape[0]
        h2d = (0 if not animated else sc.part_center.shape[0] * 48) + 64 + nl * 32
        line = {
            "metric": "Mrays/s (build+trace+shade per frame)", "value": total_rays / t_dev / 1e6, "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "strong" if rays_split else "weak",
            "vs_baseline": None, "dtype": "f32", "data": data_desc(sc),
            "config": {"workload": workload_name(sc), "build": "GPU %s SAH (32 bins/axis%s), per frame" % (
                           args.mode, ", exact on nodes <= %d refs" % args.exact_max if args.exact_max else ""),
                       "traversal": {v: k for k, v in hk.VARIANTS.items()}[variant],
                       "autotune": tuned,
                       "build_layout": build_tuned,
                       "graph": "stages launched per frame (row bands)" if rays_split else "one CUDA graph per frame",
                       "l2": "flushed (256 MB write) between frames",
                       "parallelism": ("row bands of every frame over %d GPU(s), framebuffer all_gather" % world)
                       if rays_split else "frames sharded over %d GPU(s)" % world},
            "e2e": {"value": total_rays / t_e2e / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": W * H * 4, "ms_per_step": 1000.0 * t_e2e / args.steps,
                    "timing": "host clock per frame (synchronise, call, image read-back, synchronise)"},
            "gpu_launches": int(kern_nodes) * args.steps,
            "clocks": cl,
            "roofline": roof,
            "build_roofline": build_roofline(compare, args.mode),
            "cpu_baseline": base,
            "compare": compare,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def build_roofline(compare, mode):
    """The builder against HBM: its algorithmic bytes (per level, every
    reference's index and clipped box read and its next-level slot written,
    plus the tree written) over its measured time, for the headline's build."""
    arm = (compare or {}).get("learned" if mode == "learned" else "binned") or {}
    if "build_gbs" not in arm:
        return None
    peak, src = measured_peak()
    return {"bound": "hbm", "achieved": arm["build_gbs"], "peak": peak, "unit": "GB/s",
            "frac": arm["build_gbs"] / peak, "peak_source": src, "bytes_per_build": arm["build_bytes"],
            "build_ms": arm["build_ms"],
            "bytes": "sum over levels of references x 36 B + deferred-subtree root references x 28 B + "
                     "nodes x 8 B + leaf references x 4 B"}


def reference_tree_cost(hk, rt, device):
    """SAH cost (hk_tree_cost, benchmark constants) of the reference's tree,
    imported onto its own frame's scene."""
    nodes, refs, verts, box = rt
    from hulktracer_b200 import scenes
    sc = scenes.animated_parts()
    c = hk.Context(device=device)
    c.upload(verts, sc.tris)
    c.set_box(box)
    c.import_tree(nodes, refs)
    cost = c.tree_cost(1.0, 1.5)
    c.close()
    return cost


ARMS = (("binned", "binned", 0), ("learned", "learned", 0), ("exact", "binned", 1024))


def compare_arms(args, sc, device, ref_cost, variant, tuned):
    """The metric's comparison on this GPU: the same frames through the same
    engine with each build (binned 32-bin SAH, learned proposer, exact SAH on
    nodes of up to 1024 references). Per arm: ms per frame (one CUDA graph per
    frame, device time, L2 flushed between frames), build ms and trace + shade
    ms (the stages timed apart, no graph, medians), rays, and the SAH cost of
    the tree of frame --cost-frame."""
    import torch

    import hulktracer_b200 as hk
    W, H = sc.width, sc.height
    cfg = {"block_size": tuned["block_size"], "short_stack": tuned["short_stack"]} if tuned else {}
    out = {}
    frames = list(range(args.warmup, args.warmup + args.steps))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for name, mode_s, exact_max in ARMS:
        mode = hk.BUILD_LEARNED if mode_s == "learned" else hk.BUILD_BINNED
        stream = torch.cuda.Stream()
        ctx = hk.Context(device=device, exact_max=exact_max, **cfg)
        ctx.set_stream(stream.cuda_stream)
        if mode == hk.BUILD_LEARNED:
            if not os.path.exists(args.weights):
                out[name] = {"unavailable": "no trained proposer weights"}
                ctx.close()
                continue
            ctx.mlp_load(args.weights)
        ctx.upload(sc.verts, sc.tris)
        ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
        rgba = torch.zeros(W * H, dtype=torch.int32, device="cuda")
        with torch.cuda.stream(stream):
            # the arm's builder layout (hk_autotune_build, untimed setup)
            ctx.transform(frame_mats(sc, 0))
            if args.layout:
                ctx.set_build_layout(*args.layout)
                layout = dict(zip(("subtree_max", "subtree_depth", "level_streams"), args.layout))
            else:
                layout = ctx.autotune_build(mode, 3)
            for f in range(args.warmup):
                ctx.frame(frame_mats(sc, f), sc.camera, sc.lights, W, H, rgba.data_ptr(), mode, variant, True)
            stream.synchronize()
            t_frame, rays = 0.0, 0
            for f in frames:
                m = frame_mats(sc, f)
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.frame(m, sc.camera, sc.lights, W, H, rgba.data_ptr(), mode, variant, True)
                e1.record(stream)
                stream.synchronize()
                t_frame += e0.elapsed_time(e1)
                p, s_ = ctx.ray_counts()
                rays += p + s_
            # stages apart (no graph): build, then trace + shade
            t_build, t_trace = [], []
            for f in frames[: min(len(frames), 10)]:
                ctx.transform(frame_mats(sc, f))
                flush.zero_()
                e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
                e0.record(stream)
                ctx.L.hk_build(ctx.h, mode, None)
                e1.record(stream)
                ctx.render_device(sc.camera, sc.lights, W, H, rgba.data_ptr(), variant)
                e2.record(stream)
                stream.synchronize()
                t_build.append(e0.elapsed_time(e1))
                t_trace.append(e1.elapsed_time(e2))
            ctx.transform(frame_mats(sc, args.cost_frame))
            st = ctx.build(mode)
            cost = ctx.tree_cost(1.0, 1.5)
            learned_nodes, fallback_nodes = st["learned_nodes"], st["fallback_nodes"]
            # algorithmic bytes of the build: per level, each reference's index
            # (4 B) and clipped box (24 B) read and its next-level slot (8 B)
            # written; the tree's nodes (8 B) and leaf references (4 B) written
            _, lrefs = ctx.level_counts()
            # deferred subtrees: each root's references read once (index and
            # box, 28 B) by the warp that builds the subtree in registers
            sub = ctx.subtree_counts()
            build_bytes = (int(lrefs.astype(np.int64).sum()) * 36 + sub["root_refs"] * 28 + st["nodes"] * 8 +
                           st["refs"] * 4)
        ms = t_frame / len(frames)
        out[name] = {"build": "%s%s" % (mode_s, ", exact SAH on nodes <= %d refs" % exact_max if exact_max else ""),
                     "ms_per_frame": ms, "mrays_s": rays / (t_frame / 1000.0) / 1e6,
                     "build_ms": float(np.median(t_build)), "trace_shade_ms": float(np.median(t_trace)),
                     "sah_cost": cost, "sah_cost_vs_reference": (cost / ref_cost) if ref_cost else None,
                     "build_bytes": build_bytes,
                     "build_gbs": build_bytes / (float(np.median(t_build)) * 1e-3) / 1e9,
                     "layout": None if layout is None else {k: layout[k] for k in ("subtree_max", "subtree_depth",
                                                                                   "level_streams")}}
        if mode == hk.BUILD_LEARNED:
            out[name].update({"learned_nodes": learned_nodes, "fallback_nodes": fallback_nodes})
        ctx.close()
    if "ms_per_frame" in out.get("learned", {}) and "ms_per_frame" in out.get("exact", {}):
        out["learned_speedup_vs_exact"] = out["exact"]["ms_per_frame"] / out["learned"]["ms_per_frame"]
        out["learned_cost_vs_exact"] = out["learned"]["sah_cost"] / out["exact"]["sah_cost"]
        out["learned_speedup_vs_binned"] = out["binned"]["ms_per_frame"] / out["learned"]["ms_per_frame"]
    out["cost_frame"] = args.cost_frame
    out["reference_sah_cost"] = ref_cost
    out["frames"] = [frames[0], frames[-1]]
    return out


def trace_roofline(ctx, sc, stream, variant):
    import torch

    import hulktracer_b200 as hk
    W, H = sc.width, sc.height
    n = W * H
    rays_h = ctx.camera_rays(sc.camera, W, H)
    if W % 8 == 0 and H % 4 == 0:   # the frame traces primary rays in 8x4-pixel tiles
        rays_h = np.ascontiguousarray(rays_h.reshape(H // 4, 4, W // 8, 8, 8).transpose(0, 2, 1, 3, 4).reshape(-1, 8))
    d_rays = torch.from_numpy(rays_h).cuda()
    d_hits = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    ctx.set_counting(True)
    ctx.trace_device(d_rays.data_ptr(), n, d_hits.data_ptr(), variant)
    ctx.synchronize()
    cnt = ctx.counters()
    ctx.set_counting(False)
    n_node, n_ref, n_tri = (float(x) / n for x in cnt)
    b_ray = 32 + 8 + 8 * n_node + 4 * n_ref + 36 * n_tri
    reps = 20
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    with torch.cuda.stream(stream):
        for _ in range(3):
            ctx.trace_device(d_rays.data_ptr(), n, d_hits.data_ptr(), variant)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            ctx.trace_device(d_rays.data_ptr(), n, d_hits.data_ptr(), variant)
            e1.record(stream)
    torch.cuda.synchronize()
    t = sum(e0.elapsed_time(e1) for e0, e1 in ev) / 1000.0 / reps
    del flush
    peak, src = measured_peak()
    achieved = n * b_ray / t / 1e9
    # DRAM and L2 bytes of one launch from the committed ncu summary of the
    # same kernel and workload (dram__bytes_read.sum + dram__bytes_write.sum,
    # lts__t_sectors.sum x 32); the summary names its tree's builder layout
    traffic = l2_bytes = None
    vname = {v: k for k, v in hk.VARIANTS.items()}.get(variant, "")
    prof_rel = os.path.join("profiles", "k_trace_%s_%s_primary.md" % (vname, traffic_tag(sc)))
    prof = os.path.join(ROOT, prof_rel)
    if os.path.exists(prof):
        with open(prof) as f:
            for line in f:
                if line.startswith("| traffic_bytes_per_launch |"):
                    traffic = int(line.split("|")[2])
                if line.startswith("| l2_bytes_per_launch |"):
                    l2_bytes = int(line.split("|")[2])
    out = {"kernel": "k_trace primary rays", "bound": "hbm", "achieved": achieved, "peak": peak,
           "peak_source": src, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
           "traffic_source": (prof_rel + " (dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of "
                              "the same kernel and workload; the file names the tree's layout)")
           if traffic is not None else None,
           "launch_ms": t * 1000.0, "rays_per_launch": n, "bytes_per_ray": b_ray,
           "l2": "flushed (256 MB write) before every timed launch",
           "per_ray": {"nodes": n_node, "refs": n_ref, "tris": n_tri}, "mrays_per_s": n / t / 1e6}
    if l2_bytes is not None:
        # the scene stays in L2: the bytes L2 served the launch, over its time
        out["l2_gbs"] = l2_bytes / t / 1e9
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
