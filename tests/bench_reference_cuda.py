"""Time the reference ASTRA Toolbox's own CUDA projectors (built from its
sources into oracle/_ref/ by oracle/ref.mk) on the cone-beam workload, next to
libb2tomo on the same inputs, and report their agreement.

    python tests/bench_reference_cuda.py [--n 512] [--views 720] [--det 832] [--reps 3]

Prints one JSON line: per-call milliseconds and GUPS of the reference ConeFP /
ConeBP and of b2t_fp3d / b2t_bp3d, and the relative L2 difference of the
outputs.  Each reference call allocates its texture array and synchronises, as
it does inside ASTRA; both sides are timed with CUDA events around the call.
"""
import argparse
import importlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--views", type=int, default=720)
    ap.add_argument("--det", type=int, default=832)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--kind", default="cone", choices=["cone", "parallel3d"])
    args = ap.parse_args()
    import torch
    from oracle import ref
    astra = importlib.import_module("astra-toolbox_b200")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    ang = np.linspace(0, 2 * np.pi if args.kind == "cone" else np.pi, args.views, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(args.n, args.n, args.n)
    if args.kind == "cone":
        pg = astra.create_proj_geom('cone', 1.0, 1.0, args.det, args.det, ang, 1000.0, 500.0)
    else:
        pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, args.det, args.det, ang)
    pr = astra.Projector3D(pg, vg)
    kind = pr.geom.kind
    views, vs = ref.geom3d(vg, pg)
    assert np.array_equal(views, pr.geom.views_array())
    dev = torch.device("cuda", 0)
    vol = ph.ellipsoids(pr.vol_shape, 12, seed=0, axes=(0.04 * args.n, 0.4 * args.n), device=dev)
    nv, na, nu = pr.proj_shape

    def timed(fn):
        ts = []
        out = None
        for i in range(args.reps + 1):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.synchronize()
            if i > 0:
                ts.append(e0.elapsed_time(e1))
        return out, float(np.median(ts))

    proj_ref, t_fp_ref = timed(lambda: ref.cuda_fp3d(kind, views, vol, nu, nv, vs))
    proj_b2t = torch.zeros(pr.proj_shape, device=dev)
    _, t_fp_b2t = timed(lambda: pr.fp(vol, proj_b2t))
    back_ref, t_bp_ref = timed(lambda: ref.cuda_bp3d(kind, views, proj_ref, pr.vol_shape, vs))
    back_b2t = torch.zeros(pr.vol_shape, device=dev)
    _, t_bp_b2t = timed(lambda: pr.bp(proj_ref, back_b2t))

    def rl2(a, b):
        return float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))

    upd = float(args.n) ** 3 * args.views
    out = {"workload": "%s %d^3, %d views, %d^2 detector" % (args.kind, args.n, args.views, args.det),
           "ref_fp_ms": t_fp_ref, "ref_bp_ms": t_bp_ref, "b2t_fp_ms": t_fp_b2t, "b2t_bp_ms": t_bp_b2t,
           "ref_fp_gups": upd / t_fp_ref / 1e6, "ref_bp_gups": upd / t_bp_ref / 1e6,
           "b2t_fp_gups": upd / t_fp_b2t / 1e6, "b2t_bp_gups": upd / t_bp_b2t / 1e6,
           "fp_speedup": t_fp_ref / t_fp_b2t, "bp_speedup": t_bp_ref / t_bp_b2t,
           "fp_rel_l2_b2t_vs_ref": rl2(proj_b2t, proj_ref), "bp_rel_l2_b2t_vs_ref": rl2(back_b2t, back_ref)}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
