"""Small, self-contained GPU cases for profiler captures (ncu) of single kernels.

    python -m hulktracer_b200.profile_case --case trace --variant shortstack
    python -m hulktracer_b200.profile_case --case build
    python -m hulktracer_b200.profile_case --case frame
    python -m hulktracer_b200.profile_case --case aff --aff scene.aff --frames 60
    python -m hulktracer_b200.profile_case --case stream --pools 1 0.25 0.05 0.01

Each case sets up the animated 64-part scene (~200k triangles, 1280x720), does
its warm-up work first and then launches the kernel of interest a few times, so
an ncu command can select it with -k / -s / -c. The aff case instead renders an
AFF (BART) scene frame by frame on the reference's fixed-tick clock and prints
device times per frame. The stream case traces the frame's primary rays with
leaves paged in from host memory (hk_trace_streamed) for pools of the given
fractions of the tree's leaf records, beside the resident kd-restart traversal.
"""
from __future__ import annotations

import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main():
    import numpy as np
    import torch

    import hulktracer_b200 as hk
    from hulktracer_b200 import scenes

    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="trace", choices=["trace", "build", "frame", "breakdown", "batch", "aff",
                                                         "stream"])
    ap.add_argument("--pools", type=float, nargs="+", default=[1.0, 0.25, 0.05, 0.01],
                    help="stream case: pool sizes as fractions of the leaf records")
    ap.add_argument("--aff", help="aff case: the scene file")
    ap.add_argument("--frames", type=int, default=60, help="aff case: frames timed")
    ap.add_argument("--size", type=int, nargs=2, help="aff case: image size (default: the file's resolution)")
    ap.add_argument("--scenes", type=int, default=64, help="batch case: number of scenes")
    ap.add_argument("--rays", type=int, nargs=2, default=[65_536, 4_194_304], help="batch case: ray batch range")
    ap.add_argument("--tris", type=int, nargs=2, default=[10_000, 2_000_000], help="batch case: triangle range")
    ap.add_argument("--variant", default="shortstack")
    ap.add_argument("--mode", default="binned", choices=["binned", "learned", "resort"],
                    help="resort: the reference's --treeType=SAH builder with its own constants "
                         "(Ct 1, Ci 5, depth 20, leaves below 10, every 5th polygon sampled)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--weights", default=os.path.join(ROOT, "hulktracer_b200", "weights", "proposer.bin"))
    ap.add_argument("--exact-max", type=int, default=0, help="exact SAH on nodes of at most this many refs")
    ap.add_argument("--layout", type=int, nargs=3, metavar=("SUBTREE_MAX", "SUBTREE_DEPTH", "LEVEL_STREAMS"),
                    help="builder layout (hk_set_build_layout) instead of the library default")
    a = ap.parse_args()
    if a.case == "batch":
        batch_case(a)
        return
    if a.case == "aff":
        aff_case(a)
        return
    sc = scenes.animated_parts()
    W, H = sc.width, sc.height
    resort = dict(traverse_cost=1.0, intersect_cost=5.0, max_depth=20, leaf_size=9, sah_sample=5)
    ctx = hk.Context(exact_max=a.exact_max, **(resort if a.mode == "resort" else {}))
    if a.mode == "learned":
        ctx.mlp_load(a.weights)
    if a.layout:
        ctx.set_build_layout(*a.layout)
    ctx.upload(sc.verts, sc.tris)
    ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    ctx.transform(scenes.part_matrices(sc, 1))
    mode = {"learned": hk.BUILD_LEARNED, "resort": hk.BUILD_SAH_RESORT}.get(a.mode, hk.BUILD_BINNED)
    st = ctx.build(mode)
    if a.case == "trace":
        # primary rays in the frame's 8x4-pixel tile order
        rays_h = ctx.camera_rays(sc.camera, W, H)
        rays_h = np.ascontiguousarray(rays_h.reshape(H // 4, 4, W // 8, 8, 8).transpose(0, 2, 1, 3, 4).reshape(-1, 8))
        rays = torch.from_numpy(rays_h).cuda()
        hits = torch.zeros(2 * W * H, dtype=torch.int32, device="cuda")
        for _ in range(a.reps):
            ctx.trace_device(rays.data_ptr(), W * H, hits.data_ptr(), hk.VARIANTS[a.variant])
        ctx.synchronize()
    elif a.case == "build":
        ms = []
        for _ in range(a.reps):
            st = ctx.build(mode)
            ms.append(st["build_ms"])
        print("build_ms per build: %s" % ", ".join("%.3f" % m for m in ms))
    elif a.case == "breakdown":
        # device time per stage (CUDA events, no graph), median of reps
        import json
        out = torch.zeros(W * H, dtype=torch.int32, device="cuda")
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        rays = torch.from_numpy(ctx.camera_rays(sc.camera, W, H)).cuda()
        rays = rays.reshape(H // 4, 4, W // 8, 8, 8).permute(0, 2, 1, 3, 4).reshape(-1, 8).contiguous()
        hits = torch.zeros(2 * W * H, dtype=torch.int32, device="cuda")
        v = hk.VARIANTS[a.variant]
        res = {}

        def timed(name, fn, reps=10):
            ts = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                stream.synchronize()
                ts.append(e0.elapsed_time(e1))
            res[name] = sorted(ts)[len(ts) // 2]

        mats = scenes.part_matrices(sc, 2)
        with torch.cuda.stream(stream):
            timed("transform+precompute", lambda: ctx.transform(mats))
            timed("build", lambda: ctx.L.hk_build(ctx.h, mode, None))
            timed("trace_primary", lambda: ctx.trace_device(rays.data_ptr(), W * H, hits.data_ptr(), v))
            timed("render(primary+shadow+shade)", lambda: ctx.render_device(sc.camera, sc.lights, W, H, out.data_ptr(), v))
            timed("frame_graph", lambda: ctx.frame(mats, sc.camera, sc.lights, W, H, out.data_ptr(), mode, v, True))
            timed("frame_nograph", lambda: ctx.frame(mats, sc.camera, sc.lights, W, H, out.data_ptr(), mode, v, False))
        p_, s_ = ctx.ray_counts()
        res["rays"] = {"primary": p_, "shadow": s_}
        res["tree"] = ctx.stats()
        print(json.dumps(res))
    elif a.case == "stream":
        import json
        rays_h = ctx.camera_rays(sc.camera, W, H)
        rays = torch.from_numpy(rays_h).cuda()
        hits = torch.zeros(2 * W * H, dtype=torch.int32, device="cuda")
        res = {"rays": W * H}
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        for name in ("restart", "restart_early"):
            ts = []
            for _ in range(a.reps + 1):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.trace_device(rays.data_ptr(), W * H, hits.data_ptr(), hk.VARIANTS[name])
                e1.record(stream)
                stream.synchronize()
                ts.append(e0.elapsed_time(e1))
            res[name + "_ms"] = sorted(ts[1:])[len(ts[1:]) // 2]
        ctx.set_stream(None)
        cn = ctx.export_compact()[0]
        leaves = cn[(cn[:, 0] & 3) == 3]
        total = int(leaves[:, 1].sum())
        res["leaf_records"] = total
        ref = ctx.trace(rays_h, hk.RESTART)
        for frac in a.pools:
            pool = max(int(leaves[:, 1].max()), int(total * frac))
            ctx.stream_setup(pool)
            h1, cold = ctx.trace_streamed(rays_h)
            _, warm = ctx.trace_streamed(rays_h)
            assert np.array_equal(h1["tri"], ref["tri"])
            cold["pool_records"] = pool
            cold["paged_gbs"] = cold["bytes_paged"] / (cold["ms"] * 1e6) if cold["ms"] > 0 else 0.0
            res["pool_%g" % frac] = {"cold": cold, "warm": warm}
        print(json.dumps(res))
    else:
        out = torch.zeros(W * H, dtype=torch.int32, device="cuda")
        for f in range(a.reps):
            ctx.frame(scenes.part_matrices(sc, f), sc.camera, sc.lights, W, H, out.data_ptr(), mode,
                      hk.VARIANTS[a.variant], True)
        ctx.synchronize()
    print("case %s done: tree %s" % (a.case, {k: st[k] for k in ("nodes", "refs", "depth")}))


def aff_case(a):
    """Frames of an AFF scene through hk_frame (transform, build, trace,
    shadows, shading in one CUDA graph), timed with CUDA events."""
    import json

    import numpy as np
    import torch

    import hulktracer_b200 as hk
    from hulktracer_b200.engine import Aff, fixed_tick_time

    aff = Aff(a.aff)
    info = aff.info
    W, H = a.size if a.size else (info["resx"], info["resy"])
    W, H = W // 8 * 8, H // 4 * 4
    lights = aff.lights()
    if lights.shape[0] == 0:
        lights = np.array([[1, 1, 1, 1, 0, 100, 0, 1]], np.float32)
    ctx = hk.Context(exact_max=a.exact_max)
    mode = hk.BUILD_LEARNED if a.mode == "learned" else hk.BUILD_BINNED
    if a.mode == "learned":
        ctx.mlp_load(a.weights)
    ctx.load_aff(aff, 0.0)
    out = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    v = hk.VARIANTS[a.variant]
    times = [fixed_tick_time(f) for f in range(a.frames)]
    with torch.cuda.stream(stream):
        for t in times[:3]:      # warm-up, graph capture
            ctx.frame(aff.part_matrices(t), aff.camera(t), lights, W, H, out.data_ptr(), mode, v, True)
        ms, stats = [], []
        for t in times:
            mats, cam = aff.part_matrices(t), aff.camera(t)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.frame(mats, cam, lights, W, H, out.data_ptr(), mode, v, True)
            e1.record(stream)
            stream.synchronize()
            ms.append(e0.elapsed_time(e1))
    p_, s_ = ctx.ray_counts()
    st = ctx.stats()
    res = {"scene": os.path.basename(a.aff), "tris": info["nt"], "meshes": info["nmeshes"],
           "dynamic_meshes": info["ndynamic"], "size": [W, H], "frames": a.frames, "build": a.mode,
           "ms_per_frame_median": float(np.median(ms)), "ms_per_frame_mean": float(np.mean(ms)),
           "rays_last_frame": {"primary": p_, "shadow": s_},
           "mrays_s": (p_ + s_) / (float(np.median(ms)) * 1e3),
           "tree_last_frame": {k: st[k] for k in ("nodes", "refs", "depth", "build_ms")}}
    print(json.dumps(res))


def batch_case(a):
    """Many scenes, one persistent launch: 64 clustered-soup scenes with
    log-uniform triangle counts in [10k, 2M] and log-uniform ray batches in
    [64k, 4M] (a quarter primary rays, the rest cosine-weighted rays leaving
    random surface points: shadow / diffuse-bounce stand-ins). Prints the
    aggregate Mrays/s of the batched launch, the per-scene completion times
    (p50 / p99) and, for comparison, one launch per scene."""
    import json
    import time

    import numpy as np
    import torch

    import hulktracer_b200 as hk
    from hulktracer_b200 import scenes
    t0 = time.time()
    sets = scenes.batch_scenes(n_scenes=a.scenes, tris=tuple(a.tris), rays=tuple(a.rays))
    rays = [scenes.incoherent_rays(sc, nr, seed=1000 + i) for i, (sc, nr) in enumerate(sets)]
    ctx = hk.Context()
    batch = hk.engine.Batch(ctx)
    offsets = [0]
    for i, (sc, nr) in enumerate(sets):
        batch.add_scene(sc.verts, sc.tris)
        offsets.append(offsets[-1] + nr)
    allr = np.concatenate(rays)
    n = allr.shape[0]
    d_rays = torch.from_numpy(allr).cuda()
    d_hits = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    setup_s = time.time() - t0
    tuned, cfg = None, {}
    if a.variant == "auto":
        # the batch launch itself timed for each candidate (a configuration
        # tuned on one scene does not carry over to the whole batch): variant,
        # block size, short-stack depth; the fastest is kept
        t1 = time.time()
        cands = [(vn, bs, ss) for vn in ("ropes", "shortstack", "fullstack", "restart_early")
                 for bs in (64, 128, 256) for ss in ((4, 6, 8) if vn == "shortstack" else (6,))]
        best = None
        for vn, bs, ss in cands:
            ctx.set_trace_config(bs, ss)
            batch.trace_device(d_rays.data_ptr(), offsets, d_hits.data_ptr(), hk.VARIANTS[vn])
            ts = []
            for _ in range(2):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                batch.trace_device(d_rays.data_ptr(), offsets, d_hits.data_ptr(), hk.VARIANTS[vn])
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            if best is None or min(ts) < best[0]:
                best = (min(ts), vn, bs, ss)
        tuned = {"variant": best[1], "block_size": best[2], "short_stack": best[3], "best_ms": best[0],
                 "tried": len(cands), "tune_s": round(time.time() - t1, 1)}
        cfg = {"block_size": best[2], "short_stack": best[3]}
        ctx.set_trace_config(best[2], best[3])
    v = hk.VARIANTS[tuned["variant"]] if tuned else hk.VARIANTS[a.variant]
    for _ in range(2):
        batch.trace_device(d_rays.data_ptr(), offsets, d_hits.data_ptr(), v)
    torch.cuda.synchronize()
    reps, ms_all, per = 5, [], []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ms = batch.trace_device(d_rays.data_ptr(), offsets, d_hits.data_ptr(), v)
        e1.record()
        torch.cuda.synchronize()
        ms_all.append(e0.elapsed_time(e1))
        per.append(ms)
    t = float(np.median(ms_all))
    per = np.median(np.stack(per), axis=0)
    # one launch per scene, same rays (each scene's own context and tree)
    single = []
    for i, (sc, nr) in enumerate(sets):
        c = hk.Context(**cfg)
        c.upload(sc.verts, sc.tris)
        c.precompute()
        c.build()
        single.append(c)
    def run_single():
        for i, c in enumerate(single):
            c.trace_device(d_rays.data_ptr() + 32 * offsets[i], offsets[i + 1] - offsets[i],
                           d_hits.data_ptr() + 8 * offsets[i], v)
        for c in single:
            c.synchronize()
    run_single()
    ts = []
    for _ in range(3):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        run_single()
        ts.append((time.perf_counter() - t1) * 1000.0)
    out = {"scenes": len(sets), "tris_total": int(sum(sc.ntris for sc, _ in sets)), "rays": int(n),
           "variant": {x: k for k, x in hk.VARIANTS.items()}[v], "autotune": tuned, "batched_ms": t, "batched_mrays_s": n / t / 1e3,
           "scene_done_ms_p50": float(np.percentile(per, 50)), "scene_done_ms_p99": float(np.percentile(per, 99)),
           "per_scene_launches_ms": float(np.median(ts)), "per_scene_mrays_s": n / float(np.median(ts)) / 1e3,
           "setup_s": round(setup_s, 1)}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
