"""Benchmark: cone-beam FP + BP at 512^3 x 720 views (832^2 detector, SOD 1000,
ODD 500) on seeded synthetic ellipsoid phantoms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one forward projection (b2t_fp3d, SET) plus one backprojection
(b2t_bp3d, SET) of the full workload, inputs resident in HBM.  The metric is
GUPS = voxel-view updates per second, 2 * 512^3 * 720 per step (FP + BP).
With N GPUs (torchrun, one process per GPU) every rank projects its own
independent phantom (weak scaling, no collective on the data path); value is
the total updates of all ranks divided by the slowest rank's time.

--impl reference times the reference's CPU path for this workload on the host
cores: the reference has no CPU 3D projector, so this is the FP64 port of its
model (oracle/), multi-threaded over all host threads, on a bounded sample of
views per step.
"""
import argparse
import ctypes
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_VOX, N_ANG, N_DET, SOD, ODD, N_ELL = 512, 720, 832, 1000.0, 500.0, 12


def workload(n=N_VOX, na=N_ANG, nd=N_DET):
    astra = importlib.import_module("astra-toolbox_b200")
    ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(n, n, n)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, nd, nd, ang, SOD, ODD)
    return astra, vg, pg


def config_dict(n, na, nd, extra=None):
    c = {"workload": "cone FP+BP, %d^3 volume, %d views over 2pi, %dx%d detector, SOD %g, ODD %g, "
                     "%d seeded random ellipsoids" % (n, na, nd, nd, SOD, ODD, N_ELL),
         "global_batch": 1, "volume": [n, n, n], "views": na, "detector": [nd, nd],
         "l2_policy": "inputs larger than L2 (volume %.0f MB, projections %.0f MB > 126 MB)"
                      % (n ** 3 * 4 / 1e6, nd * nd * na * 4 / 1e6),
         "parallelism": "independent problem per GPU"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
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
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(vol_cpu, pr, n_views, nthreads):
    """FP64 oracle FP of n_views views; returns (GUPS, seconds, threads)."""
    from oracle import oracle as orc
    nv, na, nu = pr.proj_shape
    views = pr.geom.views_array()
    sel = np.linspace(0, na - 1, n_views).round().astype(int)
    sub = views[sel]
    t0 = time.perf_counter()
    orc.fp3d(2, sub, vol_cpu, nu, nv, pr.geom.vol_scale, nthreads=nthreads)
    dt = time.perf_counter() - t0
    n = vol_cpu.size
    return n * n_views / dt / 1e9, dt


def run_reference(args):
    """--impl reference: the CPU path (FP64 port of the model) on host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import torch
    astra, vg, pg = workload(args.n, args.views, args.det)
    proj_mod = importlib.import_module("astra-toolbox_b200.projector")
    pr = proj_mod.Projector3D.__new__(proj_mod.Projector3D)
    pr.geom = importlib.import_module("astra-toolbox_b200.geometry").Geometry3D(vg, pg)
    pr.proj_shape = pr.geom.proj_shape
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    vol = ph.ellipsoids((args.n, args.n, args.n), N_ELL, seed=0, device="cpu").numpy()
    threads = os.cpu_count() or 1
    samples = []
    for i in range(args.warmup + args.steps):
        g, dt = cpu_sample(vol, pr, args.ref_views, threads)
        if i >= args.warmup:
            samples.append((g, dt))
    gups = float(np.median([s[0] for s in samples]))
    ms = float(np.median([s[1] for s in samples])) * 1e3
    sample = ("FP64 oracle forward projection of %d of the %d views per step (all %d^2 rays of each view), "
              "GUPS extrapolated per view" % (args.ref_views, args.views, args.det))
    line = {"metric": "cone FP/BP GUPS at 512^3x720", "value": gups, "unit": "GUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": config_dict(args.n, args.views, args.det),
            "cpu_baseline": {"value": gups, "unit": "GUPS", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": gups, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_VOX)
    ap.add_argument("--views", type=int, default=N_ANG)
    ap.add_argument("--det", type=int, default=N_DET)
    ap.add_argument("--dtype", default="float32", choices=["float32", "float16", "bfloat16"])
    ap.add_argument("--ref-views", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    astra, vg, pg = workload(args.n, args.views, args.det)
    lib = importlib.import_module("astra-toolbox_b200._lib").load()
    lib.b2t_kernel_launches.restype = ctypes.c_uint64
    pr = astra.Projector3D(pg, vg)
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    tdt = getattr(torch, args.dtype)
    vol = ph.ellipsoids(pr.vol_shape, N_ELL, seed=rank, device=dev).to(tdt)
    proj = torch.zeros(pr.proj_shape, device=dev, dtype=tdt)
    back = torch.zeros(pr.vol_shape, device=dev, dtype=tdt)
    stream = torch.cuda.current_stream(dev)

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        pr.fp(vol, proj)
        if ev:
            ev[1].record(stream)
        pr.bp(proj, back)
        if ev:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    launches0 = lib.b2t_kernel_launches()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for i in range(args.steps):
        step(evs[i])
    end.record(stream)
    torch.cuda.synchronize(dev)
    launches = lib.b2t_kernel_launches() - launches0
    clocks = sampler.stop()
    barrier()
    total_ms = start.elapsed_time(end)
    fp_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    bp_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
    t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_step = total_ms / args.steps
    updates = float(args.n) ** 3 * args.views
    value = 2 * updates * world / (ms_step * 1e-3) / 1e9

    # end to end through the public API with host buffers: direct_FP3D then
    # direct_BP3D on pinned host arrays (H2D input, kernels, D2H output)
    e2e = None
    if not args.no_e2e:
        P = importlib.import_module("astra-toolbox_b200.projector")
        hvol = vol.cpu().pin_memory()
        hproj = torch.empty(pr.proj_shape, dtype=tdt).pin_memory()
        hback = torch.empty(pr.vol_shape, dtype=tdt).pin_memory()
        dvol = torch.empty_like(vol)
        dproj = torch.empty_like(proj)
        dback = torch.empty_like(back)

        def e2e_step():
            dvol.copy_(hvol, non_blocking=True)
            pr.fp(dvol, dproj)
            hproj.copy_(dproj, non_blocking=True)
            dproj.copy_(hproj, non_blocking=True)
            pr.bp(dproj, dback)
            hback.copy_(dback, non_blocking=True)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize(dev)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ke = max(1, min(args.steps, 3))
        for _ in range(ke):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        et = torch.tensor([e0.elapsed_time(e1) / ke], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        esz = vol.element_size()
        vb = vol.numel() * esz
        pb = proj.numel() * esz
        e2e = {"value": 2 * updates * world / (float(et.item()) * 1e-3) / 1e9, "unit": "GUPS",
               "h2d_bytes_per_step": vb + pb, "d2h_bytes_per_step": pb + vb,
               "ms_per_step": float(et.item()),
               "path": "Projector3D.fp/bp (the direct_FP3D / direct_BP3D path) with pinned host input "
                       "copied in and output copied out each call"}
        del dvol, dproj, dback

    cpu = None
    if rank == 0 and not args.no_cpu:
        vcpu = vol.float().cpu().numpy()
        threads = os.cpu_count() or 1
        g, dt = cpu_sample(vcpu, pr, args.ref_views, threads)
        cpu = {"value": g, "unit": "GUPS", "cores": threads, "kind": "port",
               "sample": "FP64 oracle forward projection of %d views of this workload on %d host threads "
                         "(%.1f s), GUPS per view" % (args.ref_views, threads, dt)}

    # roofline of the dominant kernel (the larger of FP and BP)
    esz = vol.element_size()
    vol_bytes = vol.numel() * esz
    proj_bytes = proj.numel() * esz
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak_hbm = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak_hbm, peak_src = 6650.0, "fallback"
    dom = "fp" if fp_ms >= bp_ms else "bp"
    dom_ms = max(fp_ms, bp_ms)
    # compulsory HBM bytes of one call: read the input once (plus its padded
    # copy: one write and one read) and write the output once
    if dom == "fp":
        alg_bytes = vol_bytes * 3 + proj_bytes
    else:
        alg_bytes = proj_bytes * 3 + vol_bytes
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "b2t_fp3d" if dom == "fp" else "b2t_bp3d",
                "achieved": achieved, "peak": peak_hbm, "unit": "GB/s", "frac": achieved / peak_hbm,
                "traffic": None, "peak_source": peak_src,
                "note": "projectors are bound by on-chip interpolation reads, not HBM; "
                        "fp_gups=%.1f bp_gups=%.1f" % (updates / (fp_ms * 1e-3) / 1e9,
                                                        updates / (bp_ms * 1e-3) / 1e9)}
    if rank == 0:
        line = {"metric": "cone FP/BP GUPS at 512^3x720", "value": value, "unit": "GUPS", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": {"float32": "f32", "float16": "f16 storage, f32 math",
                          "bfloat16": "bf16 storage, f32 math"}[args.dtype],
                "data": "synthetic", "config": config_dict(args.n, args.views, args.det),
                "fp_ms": fp_ms, "bp_ms": bp_ms,
                "fp_gups": updates / (fp_ms * 1e-3) / 1e9, "bp_gups": updates / (bp_ms * 1e-3) / 1e9,
                "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks, "roofline": roofline,
                "cpu_baseline": cpu}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
