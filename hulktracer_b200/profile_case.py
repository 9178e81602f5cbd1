"""Small, self-contained GPU cases for profiler captures (ncu) of single kernels.

    python -m hulktracer_b200.profile_case --case trace --variant shortstack
    python -m hulktracer_b200.profile_case --case build
    python -m hulktracer_b200.profile_case --case frame

Each case sets up the animated 64-part scene (~200k triangles, 1280x720), does
its warm-up work first and then launches the kernel of interest a few times, so
an ncu command can select it with -k / -s / -c.
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
    ap.add_argument("--case", default="trace", choices=["trace", "build", "frame", "breakdown"])
    ap.add_argument("--variant", default="shortstack")
    ap.add_argument("--mode", default="binned", choices=["binned", "learned"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--weights", default=os.path.join(ROOT, "hulktracer_b200", "weights", "proposer.bin"))
    ap.add_argument("--exact-max", type=int, default=0, help="exact SAH on nodes of at most this many refs")
    a = ap.parse_args()
    sc = scenes.animated_parts()
    W, H = sc.width, sc.height
    ctx = hk.Context(exact_max=a.exact_max)
    if a.mode == "learned":
        ctx.mlp_load(a.weights)
    ctx.upload(sc.verts, sc.tris)
    ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    ctx.transform(scenes.part_matrices(sc, 1))
    mode = hk.BUILD_LEARNED if a.mode == "learned" else hk.BUILD_BINNED
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
        for _ in range(a.reps):
            st = ctx.build(mode)
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
    else:
        out = torch.zeros(W * H, dtype=torch.int32, device="cuda")
        for f in range(a.reps):
            ctx.frame(scenes.part_matrices(sc, f), sc.camera, sc.lights, W, H, out.data_ptr(), mode,
                      hk.VARIANTS[a.variant], True)
        ctx.synchronize()
    print("case %s done: tree %s" % (a.case, {k: st[k] for k in ("nodes", "refs", "depth")}))


if __name__ == "__main__":
    main()
