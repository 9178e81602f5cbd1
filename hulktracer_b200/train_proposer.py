"""Train the learned split proposer on the GPU.

    python -m hulktracer_b200.train_proposer [--scenes 160] [--epochs 24] \
        [--out hulktracer_b200/weights/proposer.bin]

Data: every node of 33..1024 references that the exact SAH splits in
exact-SAH builds (``HK_BUILD_BINNED`` with ``exact_max`` 1024 and recording
on) of seeded scenes from the two generators of the benchmark scenes --
rigid-part animations (``animated_parts`` with other seeds, part counts and
scales, at several frames) and clustered triangle soups (``cluster_soup``, the
large static generator at other sizes). A row's features are the node's
binned-SAH histogram (the features the learned build computes), its label the
(axis, bin) holding the exact plane. The bench's animated scene (seed 3) is
held out and used for validation only.

Training runs entirely in libhulkcuda.so (``hk_mlp_train``: FP32 SGEMM
forward/backward, softmax cross-entropy, Adam); the weights are written with
``hk_mlp_save`` and a JSON log beside them.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FLOP_PER_ROW = 2 * (200 * 256 + 2 * 256 * 256 + 256 * 96)


def record_scenes(ctx, n_scenes, seed, frames_per_scene, log):
    import numpy as np

    from hulktracer_b200 import scenes
    rng = np.random.default_rng(seed)
    builds = 0
    for i in range(n_scenes):
        if i % 4 == 3:
            n = int(np.exp(rng.uniform(np.log(50_000), np.log(1_000_000))))
            sc = scenes.cluster_soup(n, seed=int(rng.integers(1 << 30)),
                                     n_clusters=int(rng.integers(16, 256)), extent=float(rng.uniform(20, 80)))
            ctx.upload(sc.verts, sc.tris)
            ctx.set_box(sc.scene_box())
            ctx.precompute()
            ctx.build()
            builds += 1
        else:
            s = int(rng.integers(1000, 1 << 30))
            sc = scenes.animated_parts(seed=s, n_parts=int(rng.integers(16, 97)), width=64, height=64,
                                       scale=float(rng.uniform(0.6, 1.6)))
            ctx.upload(sc.verts, sc.tris)
            ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
            for f in rng.choice(60, size=frames_per_scene, replace=False):
                ctx.transform(scenes.part_matrices(sc, int(f)))
                ctx.build()
                builds += 1
        if (i + 1) % 20 == 0:
            log("  %d scenes, %d builds, %d rows" % (i + 1, builds, ctx.mlp_dataset(fetch=False)))
    return builds


def validate(ctx, frames=(0, 20, 40, 59)):
    """Top-1 / top-4 agreement with the exact search on the held-out scene."""
    import numpy as np

    from hulktracer_b200 import scenes
    sc = scenes.animated_parts()
    ctx.mlp_record(1 << 20)
    ctx.upload(sc.verts, sc.tris)
    ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    for f in frames:
        ctx.transform(scenes.part_matrices(sc, f))
        ctx.build()
    X, y = ctx.mlp_dataset()
    ctx.mlp_record(0)
    Z = ctx.mlp_forward(X)
    top = np.argsort(-Z, axis=1)
    return {"rows": int(X.shape[0]), "top1": float((top[:, 0] == y).mean()),
            "top4": float((top[:, :4] == y[:, None]).any(1).mean())}


def main():
    import numpy as np

    import hulktracer_b200 as hk

    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=160)
    ap.add_argument("--frames", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--capacity", type=int, default=12_000_000)
    ap.add_argument("--out", default=os.path.join(ROOT, "hulktracer_b200", "weights", "proposer.bin"))
    a = ap.parse_args()

    def log(msg):
        print(msg, flush=True)

    ctx = hk.Context(exact_max=1024)
    ctx.mlp_init(a.seed)
    ctx.mlp_record(a.capacity)
    t0 = time.time()
    builds = record_scenes(ctx, a.scenes, a.seed, a.frames, log)
    rows = ctx.mlp_dataset(fetch=False)
    t_data = time.time() - t0
    log("recorded %d rows from %d builds in %.1f s" % (rows, builds, t_data))
    # held-out agreement of the untrained network (its own context: validation
    # records into the recording buffer, which holds the training set here)
    pre = hk.Context(exact_max=1024)
    pre.mlp_init(a.seed)
    before = validate(pre)
    pre.close()
    # two phases: lr, then lr / 4
    e1 = max(1, (3 * a.epochs) // 4)
    t1 = time.time()
    l1 = ctx.mlp_train(epochs=e1, batch=a.batch, lr=a.lr, seed=a.seed)
    l2 = ctx.mlp_train(epochs=a.epochs - e1, batch=a.batch, lr=a.lr / 4, seed=a.seed + 1) if a.epochs > e1 else []
    ctx.synchronize()
    t_train = time.time() - t1
    losses = [float(x) for x in list(l1) + list(l2)]
    steps = (rows // a.batch) * a.epochs
    log("trained %d epochs (%d steps) in %.1f s; loss %.4f -> %.4f" % (a.epochs, steps, t_train, losses[0],
                                                                       losses[-1]))
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    ctx.mlp_save(a.out)
    after = validate(ctx)
    info = {
        "rows": int(rows), "builds": builds, "scenes": a.scenes, "frames_per_animated_scene": a.frames,
        "epochs": a.epochs, "batch": a.batch, "lr": a.lr, "seed": a.seed, "losses": losses,
        "record_s": round(t_data, 2), "train_s": round(t_train, 2),
        "train_rows_per_s": round(rows * a.epochs / t_train, 1),
        "train_tflops": round(3 * FLOP_PER_ROW * rows * a.epochs / t_train / 1e12, 3),
        "heldout_untrained": before, "heldout_trained": after,
    }
    with open(os.path.splitext(a.out)[0] + "_train.json", "w") as f:
        json.dump(info, f, indent=1)
    log(json.dumps({k: v for k, v in info.items() if k != "losses"}))
    del np


if __name__ == "__main__":
    main()
