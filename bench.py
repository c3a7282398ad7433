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
model (oracle/), multi-threaded over all host threads, on a bounded sample per
step (FP of a few views, BP of a few z-slices over all views); it imports
nothing of the library.

The default arm also reports, after its timed region: `parity` (this run's
FP output on sampled views and BP output on sampled z-slices against the FP64
oracle on the same inputs, which is also the CPU baseline's sample) and
`ref_cuda` (the reference's own CUDA build, oracle/_ref, timed on the same
inputs and GPU, with the agreement of the outputs).
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


def astra_dicts(n, na, nd):
    """The workload's volume and projection geometry as the reference's
    geometry dictionaries (python/astra/creators.py), built without the
    library."""
    ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)
    vg = {'GridRowCount': n, 'GridColCount': n, 'GridSliceCount': n,
          'option': {'WindowMinX': -n / 2., 'WindowMaxX': n / 2., 'WindowMinY': -n / 2., 'WindowMaxY': n / 2.,
                     'WindowMinZ': -n / 2., 'WindowMaxZ': n / 2.}}
    pg = {'type': 'cone', 'DetectorSpacingX': 1.0, 'DetectorSpacingY': 1.0, 'DetectorRowCount': nd,
          'DetectorColCount': nd, 'ProjectionAngles': ang, 'DistanceOriginSource': SOD,
          'DistanceOriginDetector': ODD}
    return ang, vg, pg


def reference_geometry(n, na, nd):
    """Per-view vectors of the workload from the reference's own
    convertAstraGeometry (oracle/_ref, the reference built from its sources),
    else from the oracle's numpy restatement; (views, voxel size, source)."""
    from oracle import oracle as orc
    from oracle import ref
    ang, vg, pg = astra_dicts(n, na, nd)
    if ref.available():
        views, vs = ref.geom3d(vg, pg)
        return views, vs, "reference convertAstraGeometry (oracle/_ref)"
    return orc.cone_views(ang, nd, nd, SOD, ODD), np.ones(3, np.float32), "oracle cone_views (numpy)"


def phantom_module():
    """The seeded ellipsoid generator (pure numpy / torch), loaded from its
    file so that the reference arm imports nothing of the library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_b2t_phantom", os.path.join(ROOT, "astra-toolbox_b200",
                                                                               "phantom.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def sample_views(na, k):
    return [int(v) for v in np.linspace(0, na - 1, k).round().astype(int)]


def sample_slices(nz, k):
    return [int(z) for z in np.linspace(0, nz - 1, k).round().astype(int)]


def oracle_sample(vol_np, proj_np, views, vs, nu, nv, fp_sel, bp_slices, nthreads):
    """The FP64 oracle (the CPU restatement of the reference's ray / voxel
    model) on a bounded sample of the workload: the forward projection of the
    views fp_sel (all rays of each) and the backprojection of the z-slices
    bp_slices over all views.  Returns the outputs, the seconds of each and
    the voxel-view updates they stand for (n^3 per FP view, n^2 x views per
    BP slice, the GUPS unit of the GPU arm)."""
    from oracle import oracle as orc
    nz, ny, nx = vol_np.shape
    na = views.shape[0]
    t0 = time.perf_counter()
    fp = orc.fp3d(orc.CONE, views[fp_sel], vol_np, nu, nv, vs, nthreads=nthreads)
    t1 = time.perf_counter()
    bp = orc.bp3d_slices(orc.CONE, views, proj_np, (nz, ny, nx), bp_slices, vs, nthreads=nthreads)
    t2 = time.perf_counter()
    units = float(nx * ny * nz) * len(fp_sel) + float(nx * ny) * len(bp_slices) * na
    return {"fp": fp, "bp": bp, "fp_s": t1 - t0, "bp_s": t2 - t1, "units": units}


def run_reference(args):
    """--impl reference: the reference's CPU path for this workload on the
    host cores.  The reference has no CPU 3D projector (its cone FP/BP exist
    only as CUDA kernels), so this is the FP64 port of its model (oracle/),
    over all host threads, on a bounded sample per step: the FP of
    --ref-views views and the BP of --ref-slices z-slices over all views.
    Imports nothing of the library (geometry from the reference build or the
    oracle, phantom from its file)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    views, vs, geom_src = reference_geometry(args.n, args.views, args.det)
    ph = phantom_module()
    vol = ph.ellipsoids((args.n, args.n, args.n), N_ELL, seed=0, device="cpu").numpy()
    # BP input: the oracle's time does not depend on the values, and the
    # full projections of the phantom cannot be computed on the host in a
    # bench step; a constant array of the full projection shape stands in
    proj = np.ones((args.det, args.views, args.det), dtype=np.float32)
    threads = os.cpu_count() or 1
    fp_sel = sample_views(args.views, args.ref_views)
    bp_sl = sample_slices(args.n, args.ref_slices)
    samples = []
    for i in range(args.warmup + args.steps):
        r = oracle_sample(vol, proj, views, vs, args.det, args.det, fp_sel, bp_sl, threads)
        if i >= args.warmup:
            samples.append((r["units"] / (r["fp_s"] + r["bp_s"]) / 1e9, r["fp_s"] + r["bp_s"]))
    gups = float(np.median([s[0] for s in samples]))
    ms = float(np.median([s[1] for s in samples])) * 1e3
    sample = ("FP64 oracle (CPU port of the reference's cone model) per step: forward projection of views %s "
              "(all %d^2 rays) and backprojection of z-slices %s over all %d views; GUPS = their voxel-view "
              "updates / time; geometry from %s" % (fp_sel, args.det, bp_sl, args.views, geom_src))
    line = {"metric": "cone FP/BP GUPS at 512^3x720", "value": gups, "unit": "GUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": config_dict(args.n, args.views, args.det),
            "cpu_baseline": {"value": gups, "unit": "GUPS", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": gups, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def ref_cuda_block(torch, dev, vol, proj_ours, back_ours, args, reps=3):
    """The reference's own CUDA build (oracle/_ref: astraCUDA3d::ConeFP /
    ConeBP, cuda/3d/cone_fp.cu:444-504, cone_bp.cu:380-401, unchanged) on the
    same inputs and GPU: CUDA-event time per call (median of reps after one
    warm-up call; every reference call allocates its texture array and
    synchronises, as inside ASTRA), clocks during those calls, speed-ups of
    this library's calls, and the relative L2 difference of the outputs."""
    from oracle import ref
    if not ref.available():
        return {"unavailable": "oracle/_ref/libastra_ref.so is not built"}
    if vol.dtype != torch.float32:
        return {"unavailable": "the reference projects float32 data only"}
    views, vs, _ = reference_geometry(args.n, args.views, args.det)
    views = np.ascontiguousarray(views)
    vsc = np.ascontiguousarray(vs, dtype=np.float32)
    n, na, nd = args.n, args.views, args.det
    L = ref.lib()
    out_p = torch.zeros_like(proj_ours)
    out_v = torch.zeros_like(back_ours)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, out):
        ts = []
        for i in range(reps + 1):
            out.zero_()
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            assert rc == 0, "reference call failed"
            if i > 0:
                ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    sampler = ClockSampler(dev.index or 0)
    sampler.start()
    time.sleep(0.3)
    t_fp = timed(lambda: L.ref_cuda_fp3d(2, views.ctypes.data, n, n, n, na, nd, nd, vsc.ctypes.data, 1.0, 1,
                                         vol.data_ptr(), out_p.data_ptr()), out_p)
    # both BPs read the same projections: this library's FP output
    t_bp = timed(lambda: L.ref_cuda_bp3d(2, 0, views.ctypes.data, n, n, n, na, nd, nd, vsc.ctypes.data, 1.0, 1,
                                         proj_ours.data_ptr(), out_v.data_ptr()), out_v)
    clocks = sampler.stop()

    def rl2(a, b):
        return float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))

    upd = float(n) ** 3 * na
    res = {"what": "reference ConeFP / ConeBP built from its sources (oracle/ref.mk), same inputs, same GPU",
           "fp_ms": t_fp, "bp_ms": t_bp, "fp_gups": upd / t_fp / 1e6, "bp_gups": upd / t_bp / 1e6,
           "fpbp_gups": 2 * upd / (t_fp + t_bp) / 1e6,
           "fp_rel_l2_ours_vs_ref": rl2(proj_ours, out_p), "bp_rel_l2_ours_vs_ref": rl2(back_ours, out_v),
           "clocks": clocks}
    del out_p, out_v
    return res


def _timed_region(torch, stream, fn, steps):
    """Time `steps` calls of fn with CUDA events on `stream`; returns ms per call."""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def batch2d_problems(astra, n_prob=64, seed=0):
    """The batched fan-beam workload: n_prob problems, W uniform in
    {128, 256, 512, 1024}, 90-1440 angles over 2pi, 1.5 W detectors of width
    1, source-origin 2 W, origin-detector W (seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    probs = []
    for _ in range(n_prob):
        W = int(rng.choice([128, 256, 512, 1024]))
        na = int(rng.integers(90, 1441))
        ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(W, W)
        pg = astra.create_proj_geom('fanflat', 1.0, int(1.5 * W), ang, 2.0 * W, 1.0 * W)
        probs.append((pg, vg))
    return probs


def run_batch2d(args):
    """--workload batch2d: 64 fan-beam problems of uneven size.  One step =
    FP + BP of every problem: batched (b2t_batch2d_fp / _bp, one persistent
    launch each) against the plain per-problem loop (Projector2D.fp / .bp, the
    reference's call pattern).  Then SIRT 50 iterations of every problem,
    batched (CUDA graph of the batched iteration) against per-problem
    SIRT_CUDA runs.  Metric: GUPS = sum over problems of W^2 x angles x 2 per
    step."""
    import torch
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    astra = importlib.import_module("astra-toolbox_b200")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D2 = importlib.import_module("astra-toolbox_b200.data2d")
    lib = importlib.import_module("astra-toolbox_b200._lib").load()
    lib.b2t_kernel_launches.restype = ctypes.c_uint64
    probs = batch2d_problems(astra)
    B = astra.Batch2D(probs, device=dev)
    imgs = [ph.ellipses(sh, 10, seed=i, axes=(0.04 * sh[1], 0.3 * sh[1]), device=dev)
            for i, sh in enumerate(B.vol_shapes)]
    vols = B.pack_vols(imgs)
    sinos = B.empty_sinos()
    back = B.empty_vols()
    prs = [astra.Projector2D(pg, vg) for pg, vg in probs]
    pv = [v.contiguous() for v in B.vol_views(vols)]
    ps = [torch.zeros(pr.proj_shape, device=dev) for pr in prs]
    pb = [torch.zeros(pr.vol_shape, device=dev) for pr in prs]
    stream = torch.cuda.current_stream(dev)
    updates = float(sum(pr.vol_shape[0] * pr.vol_shape[1] * pr.proj_shape[0] for pr in prs))

    def batched():
        B.fp(vols, sinos)
        B.bp(sinos, back)

    def plain():
        for pr, v, s_, b_ in zip(prs, pv, ps, pb):
            pr.fp(v, s_)
            pr.bp(s_, b_)

    for _ in range(args.warmup):
        batched()
        plain()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    l0 = lib.b2t_kernel_launches()
    ms_b = _timed_region(torch, stream, batched, args.steps)
    launches = lib.b2t_kernel_launches() - l0
    ms_p = _timed_region(torch, stream, plain, args.steps)
    clocks = sampler.stop()
    # SIRT 50: batched vs per problem
    truth_sino = B.fp(vols)
    rec = B.empty_vols()
    ms_sirt_b = _timed_region(torch, stream, lambda: B.sirt(truth_sino, rec.zero_(), 50), 1)
    res_b = B.sirt(truth_sino, rec.zero_(), 50)
    sviews = [s_.contiguous() for s_ in B.sino_views(truth_sino)]

    def plain_loop(kind, iters):
        for (pg, vg), sv in zip(probs, sviews):
            sid = D2.link('-sino', pg, sv)
            vid = D2.create('-vol', vg, 0)
            cfg = A.astra_dict(kind)
            cfg['ProjectionDataId'] = sid
            cfg['ReconstructionDataId'] = vid
            cfg['option'] = {'UseGraph': True}
            aid = A.create(cfg)
            A.run(aid, iters)
            A.delete(aid)
            D2.delete([sid, vid])

    ms_sirt_p = _timed_region(torch, stream, lambda: plain_loop('SIRT_CUDA', 50), 1)
    ms_cgls_b = _timed_region(torch, stream, lambda: B.cgls(truth_sino, rec.zero_(), 30), 1)
    ms_cgls_p = _timed_region(torch, stream, lambda: plain_loop('CGLS_CUDA', 30), 1)
    value = 2 * updates / (ms_b * 1e-3) / 1e9
    line = {"metric": "batched 2D fan FP+BP GUPS (64 problems)", "value": value, "unit": "GUPS", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "64 fan-beam problems, W in {128,256,512,1024}, 90-1440 views over 2pi, "
                                   "1.5 W detectors, SOD 2 W, ODD W, 10 seeded ellipses each",
                       "problems": len(probs), "updates_per_fp": updates},
            "plain_ms_per_step": ms_p, "plain_gups": 2 * updates / (ms_p * 1e-3) / 1e9,
            "batched_over_plain": ms_p / ms_b,
            "sirt50_batched_s": ms_sirt_b * 1e-3, "sirt50_plain_s": ms_sirt_p * 1e-3,
            "sirt50_batched_residual": res_b,
            "cgls30_batched_s": ms_cgls_b * 1e-3, "cgls30_plain_s": ms_cgls_p * 1e-3,
            "timing_note": "SIRT/CGLS times include creating the algorithm objects (weights, buffers) as a user "
                           "would, per problem for the plain loop and once for the batch",
            "e2e": None, "gpu_launches": int(launches), "clocks": clocks, "roofline": None, "cpu_baseline": None}
    print(json.dumps(line))
    B.close()
    return 0


def c1_phantom(n=256, seed=0):
    """The C1 phantom: 10 seeded random ellipses (centres in the inner 80 %,
    semi-axes 10-80 px, random rotation, additive intensities in [0, 1])."""
    rng = np.random.Generator(np.random.PCG64(seed))
    y, x = np.mgrid[0:n, 0:n] + 0.5 - n / 2
    img = np.zeros((n, n), dtype=np.float64)
    for _ in range(10):
        cx, cy = rng.uniform(-0.4, 0.4, 2) * n
        a, b = rng.uniform(10 * n / 256, 80 * n / 256, 2)
        t = rng.uniform(0, np.pi)
        xr = (x - cx) * np.cos(t) + (y - cy) * np.sin(t)
        yr = -(x - cx) * np.sin(t) + (y - cy) * np.cos(t)
        img[(xr / a) ** 2 + (yr / b) ** 2 <= 1] += rng.uniform(0, 1)
    return img.astype(np.float32)


def _c1_cpu_worker(core, kernel, iterations, sino, angles):
    """One host process of the C1 CPU baseline: the reference's CPU SIRT
    (its CPU-only build) pinned to one core; returns seconds."""
    import os as _os
    import time as _time
    try:
        _os.sched_setaffinity(0, {core})
    except (AttributeError, OSError):
        pass
    from oracle import ref as _ref
    t0 = _time.perf_counter()
    _ref.cpu_sirt2d('parallel', kernel, sino, (256, 256), angles, iterations)
    return _time.perf_counter() - t0


def run_c1(args):
    """--workload c1: 2D parallel beam, 256^2 volume of 10 seeded ellipses,
    180 views over pi, 384 detectors of width 1.  GPU: one step = FP + BP
    through Projector2D (metric GUPS = 2 x 256^2 x 180 / step time); SIRT_CUDA
    100 iterations from zero on the exact sinogram (CUDA-graph iterations).
    Beside it the reference's own CPU path (its CPU-only build,
    oracle/_ref/libastra_ref_cpu.so): line and linear FP and BP, SIRT with the
    line projector on one pinned core, and the aggregate over all host cores as
    independent processes, one per core."""
    import torch
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from oracle import ref
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    astra = importlib.import_module("astra-toolbox_b200")
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D2 = importlib.import_module("astra-toolbox_b200.data2d")
    lib = importlib.import_module("astra-toolbox_b200._lib").load()
    lib.b2t_kernel_launches.restype = ctypes.c_uint64
    n, na, nd = 256, 180, 384
    ang = np.linspace(0, np.pi, na, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(n, n)
    pg = astra.create_proj_geom('parallel', 1.0, nd, ang)
    pr = astra.Projector2D(pg, vg)
    img = c1_phantom(n)
    x = torch.from_numpy(img).to(dev)
    sino = torch.zeros(pr.proj_shape, device=dev)
    back = torch.zeros(pr.vol_shape, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        pr.fp(x, sino)
        pr.bp(sino, back)

    for _ in range(args.warmup):
        step()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    l0 = lib.b2t_kernel_launches()
    ms = _timed_region(torch, stream, step, max(args.steps, 50))
    launches = (lib.b2t_kernel_launches() - l0) / max(args.steps, 50) * args.steps
    # SIRT 100 on the exact (CUDA) sinogram
    sid = D2.link('-sino', pg, sino.clone())
    rid = D2.create('-vol', vg, 0)
    cfg = A.astra_dict('SIRT_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    cfg['option'] = {'UseGraph': True}
    aid = A.create(cfg)
    A.run(aid, 100)
    D2.store(rid, 0)
    sirt_ms = _timed_region(torch, stream, lambda: (D2.store(rid, 0), A.run(aid, 100)), 3)
    rec_gpu = D2.get(rid)
    A.delete(aid)
    D2.delete([sid, rid])
    clocks = sampler.stop()
    ups = 2.0 * n * n * na
    extra = {"fp_bp_ms": ms, "sirt100_s": sirt_ms * 1e-3}
    cpu = None
    parity = None
    if ref.cpu_available() and not args.no_cpu:
        t0 = time.perf_counter()
        s_line = ref.cpu_fp2d('parallel', 'line', img, ang, nd)
        t_fp_line = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.cpu_bp2d('parallel', 'line', s_line, (n, n), ang)
        t_bp_line = time.perf_counter() - t0
        t0 = time.perf_counter()
        s_lin = ref.cpu_fp2d('parallel', 'linear', img, ang, nd)
        t_fp_lin = time.perf_counter() - t0
        sino_np = sino.cpu().numpy()
        # SIRT: a bounded number of iterations per process, pinned
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        k1, kn = 20, 10
        with ctx.Pool(1) as pool:
            t_one = pool.apply(_c1_cpu_worker, (0, 'line', k1, sino_np, ang))
        cores = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else list(range(os.cpu_count() or 1))
        with ctx.Pool(len(cores)) as pool:
            ts = pool.starmap(_c1_cpu_worker, [(c, 'line', kn, sino_np, ang) for c in cores])
        it_per_s_all = sum(kn / t for t in ts)
        cpu = {"value": ups / (t_fp_line + t_bp_line) / 1e9, "unit": "GUPS", "cores": 1, "kind": "reference",
               "sample": "the reference's CPU 'line' projector (its CPU-only build), one FP + one BP of this "
                         "workload on one core",
               "fp_line_ms": t_fp_line * 1e3, "bp_line_ms": t_bp_line * 1e3, "fp_linear_ms": t_fp_lin * 1e3,
               "sirt100_line_s_one_core": t_one * 100 / k1,
               "sirt100_per_s_all_cores": it_per_s_all / 100, "all_cores": len(cores),
               "sirt_sample": "SIRT (line projector) of %d iterations on core 0 (taskset-style affinity), "
                              "extrapolated to 100; %d iterations in each of %d independent processes, one per "
                              "core, aggregate" % (k1, kn, len(cores))}
        rec_cpu = ref.cpu_sirt2d('parallel', 'linear', s_lin, (n, n), ang, 100)

        def rl2(a, b):
            return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

        parity = {"fp_vs_reference_cpu_linear": rl2(sino_np, s_lin),
                  "fp_vs_reference_cpu_line": rl2(sino_np, s_line),
                  "sirt100_vs_reference_cpu_linear_sirt100": rl2(rec_gpu, rec_cpu),
                  "tolerances": {"linear": 1e-4, "line": 3e-2, "sirt100": 2e-2}}
    line = {"metric": "2D parallel FP+BP GUPS at 256^2x180 (C1)", "value": ups / (ms * 1e-3) / 1e9,
            "unit": "GUPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "2D parallel beam, 256^2 volume of 10 seeded ellipses, 180 views over pi, 384 "
                                   "detectors; FP+BP per step, SIRT_CUDA 100 iterations", "workload_kind": "c1"},
            "e2e": None, "gpu_launches": int(launches), "clocks": clocks, "roofline": None, "cpu_baseline": cpu,
            "parity": parity}
    line.update(extra)
    print(json.dumps(line))
    return 0


def ref_algo_fdk(torch, args, proj, rec):
    """The reference's FDK_CUDA object (oracle/_ref) on a copy of the same
    projections: seconds for one run (host clock, the call synchronises) and
    the relative L2 difference from this library's reconstruction."""
    from oracle import ref
    if not ref.available():
        return {"unavailable": "oracle/_ref/libastra_ref.so is not built"}
    ang = np.linspace(0, 2 * np.pi, args.views, endpoint=False).astype(np.float32)
    out = torch.zeros_like(rec)
    ts = []
    for _ in range(2):
        p = proj.clone()
        out.zero_()
        torch.cuda.synchronize()
        alg = ref.Algo3D('FDK_CUDA', ang, SOD, ODD, p, out)
        t0 = time.perf_counter()
        alg.run(1)
        ts.append(time.perf_counter() - t0)
        alg.close()
    d = float(torch.linalg.vector_norm((rec - out).double()) / torch.linalg.vector_norm(out.double()))
    return {"what": "reference FDK_CUDA object (src/CudaFDKAlgorithm3D.cpp), same projections, same GPU",
            "s": ts[-1], "volumes_per_s": 1.0 / ts[-1], "rel_l2_ours_vs_ref": d}


def ref_algo_iterative(torch, args, kind, proj, our_run):
    """Time to a fixed residual.  The reference's SIRT3D_CUDA / CGLS3D_CUDA
    object runs --ref-iters iterations from zero on the same projections; its
    relative residual |b - A x| / |b| is the target (the residual the
    reference reaches at the configuration's iteration count).  our_run(k)
    runs this library's algorithm k iterations from zero and returns (seconds,
    relative residual); the smallest k reaching the target is searched and
    timed.  Both sides host-clocked around synchronising calls."""
    from oracle import ref
    if not ref.available():
        return {"unavailable": "oracle/_ref/libastra_ref.so is not built"}
    K = args.ref_iters
    ang = np.linspace(0, 2 * np.pi, args.views, endpoint=False).astype(np.float32)
    nv, na, nu = proj.shape
    bnorm = float(torch.linalg.vector_norm(proj.double()))

    def ref_run(k):
        vol = torch.zeros((args.n, args.n, args.n), device=proj.device)
        torch.cuda.synchronize()
        alg = ref.Algo3D(kind, ang, SOD, ODD, proj, vol)
        t0 = time.perf_counter()
        alg.run(k)
        dt = time.perf_counter() - t0
        res = alg.residual() / bnorm
        alg.close()
        return dt, res

    t1, _ = ref_run(1)
    tK, target = ref_run(K)
    ref_per_iter = (tK - t1) / (K - 1)
    # ours: the iteration count at which the residual reaches the target
    lo, hi = 1, K
    t_hi, r_hi = our_run(hi)
    while r_hi > target and hi < 2 * K:
        lo, hi = hi + 1, min(2 * K, hi + max(1, K // 4))
        t_hi, r_hi = our_run(hi)
    while lo < hi:
        mid = (lo + hi) // 2
        _, r = our_run(mid)
        if r <= target:
            hi = mid
        else:
            lo = mid + 1
    t_ours, r_ours = our_run(hi)
    return {"what": "reference %s object (src/Cuda%sAlgorithm3D.cpp), same projections, same GPU; it takes "
                    "host-memory data only, so each run copies the projections in and the volume out"
                    % (kind, "Sirt" if kind.startswith("SIRT") else "Cgls"),
            "ref_iterations": K, "ref_s": tK, "ref_s_per_iter": ref_per_iter,
            "target_relative_residual": target, "ours_iterations_to_target": hi,
            "ours_relative_residual": r_ours, "ours_s_to_target": t_ours,
            "time_to_residual_speedup": tK / t_ours if r_ours <= target else None}


def c5_vectors(na=1500, cols=1280, rows=1024, sod=1500.0, odd=600.0, seed=0):
    """The C5 cone_vec geometry: the circular orbit (source-origin 1500,
    origin-detector 600, 1280 x 1024 pixels of size 1, na views over 2 pi)
    with every view's detector jittered (seeded): its centre shifted by
    N(0, 0.5 px) along u and v, and u / v tilted by N(0, 0.1 deg) about the
    other detector axes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.zeros((na, 12))
    for i in range(na):
        t = 2 * np.pi * i / na
        src = np.array([np.sin(t) * sod, -np.cos(t) * sod, 0.0])
        det = np.array([-np.sin(t) * odd, np.cos(t) * odd, 0.0])
        u = np.array([np.cos(t), np.sin(t), 0.0])
        v = np.array([0.0, 0.0, 1.0])
        n = np.cross(u, v)
        a, b = np.deg2rad(rng.normal(0.0, 0.1, 2))
        u2 = u * np.cos(a) + n * np.sin(a)        # tilt u about v
        v2 = v * np.cos(b) + n * np.sin(b)        # tilt v about u
        det = det + rng.normal(0.0, 0.5) * u + rng.normal(0.0, 0.5) * v
        out[i] = np.concatenate([src, det, u2, v2])
    return out


def run_c5(args):
    """--workload c5: 1024^3 volume of 20 seeded ellipsoids, cone_vec geometry
    of 1500 jittered views (c5_vectors), 1280 x 1024 detector.  For FP32,
    FP16 and BF16 storage: FP and BP times (GUPS), the FP's error against the
    FP64 oracle on sampled views (on the stored, rounded volume), and 30 CGLS
    iterations from zero with FP64 inner products -- CGLS3D_CUDA for FP32; for
    FP16 / BF16 the same recurrences with the iterates stored in the half
    type, the library's half-storage projectors and b2t_dot_f64 -- with each
    half-storage result's difference from the FP32 one.  Metric: FP + BP
    GUPS with FP32 storage."""
    import torch
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from oracle import oracle as orc
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    astra = importlib.import_module("astra-toolbox_b200")
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D3 = importlib.import_module("astra-toolbox_b200.data3d")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    L = importlib.import_module("astra-toolbox_b200._lib")
    lib = L.load()
    lib.b2t_kernel_launches.restype = ctypes.c_uint64
    n, na, cols, rows = args.n if args.n != N_VOX else 1024, args.c5_views, 1280, 1024
    vecs = c5_vectors(na, cols, rows)
    vg = astra.create_vol_geom(n, n, n)
    pg = astra.create_proj_geom('cone_vec', rows, cols, vecs)
    pr = astra.Projector3D(pg, vg)
    stream = torch.cuda.current_stream(dev)
    x32 = ph.ellipsoids(pr.vol_shape, 20, seed=0, axes=(0.04 * n, 0.4 * n), device=dev)
    ups = float(n) ** 3 * na
    sel = sample_views(na, 2)
    out = {}
    b32 = None
    rec32 = None
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    for name, dt in (("f32", torch.float32), ("f16", torch.float16), ("bf16", torch.bfloat16)):
        if name not in args.c5_types:
            continue
        code = {torch.float32: L.F32, torch.float16: L.F16, torch.bfloat16: L.BF16}[dt]
        x = x32.to(dt)
        b = torch.zeros(pr.proj_shape, device=dev, dtype=dt)
        pr.fp(x, b)
        ms_fp = _timed_region(torch, stream, lambda: pr.fp(x, b), 2)
        back = torch.zeros(pr.vol_shape, device=dev, dtype=dt)
        ms_bp = _timed_region(torch, stream, lambda: pr.bp(b, back), 2)
        del back
        ref = orc.fp3d(orc.CONE, pr.geom.views_array()[sel], x.float().cpu().numpy(), cols, rows, pr.geom.vol_scale)
        got = b[:, sel, :].double().cpu().numpy()
        err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        if dt == torch.float32:
            b32 = b
            pid = D3.link('-proj3d', pg, b)
            rid = D3.create('-vol', vg, 0)
            cfg = A.astra_dict('CGLS3D_CUDA')
            cfg['ProjectionDataId'] = pid
            cfg['ReconstructionDataId'] = rid
            cfg['option'] = {'UseGraph': True}
            aid = A.create(cfg)
            t0 = time.perf_counter()
            A.run(aid, args.c5_iters)
            torch.cuda.synchronize()
            t_cgls = time.perf_counter() - t0
            res = A.get_res_norm(aid) / float(b.double().norm())
            rec32 = D3.get_shared(rid).clone()
            A.delete(aid)
            D3.delete([pid, rid])
            diff = None
        else:
            # CGLS with the iterates in the storage type (FP32 arithmetic per
            # element), FP64 inner products
            bh = b32.to(dt) if b32 is not None else b

            def dot(a_, b_):
                r_ = torch.zeros(1, dtype=torch.float64, device=dev)
                L.check(lib.b2t_dot_f64(a_.data_ptr(), b_.data_ptr(), a_.numel(), code, r_.data_ptr(),
                                        stream.cuda_stream))
                return r_

            # the operator scaled by 1 / c (c = sqrt(views x n), the projectors'
            # output scale) keeps A^T r and A p inside the FP16 range; the
            # iterate is then c x
            c = float(np.sqrt(na * n))
            sc = 1.0 / c
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            xr = torch.zeros(pr.vol_shape, device=dev, dtype=dt)
            r = bh.clone()
            p = torch.zeros(pr.vol_shape, device=dev, dtype=dt)
            pr.bp(r, p, output_scale=sc)
            q = torch.zeros(pr.proj_shape, device=dev, dtype=dt)
            z = torch.zeros(pr.vol_shape, device=dev, dtype=dt)
            gamma = dot(p, p)
            for _ in range(args.c5_iters):
                pr.fp(p, q, output_scale=sc)
                alpha = (gamma / dot(q, q)).float()
                xr.add_((p.float() * alpha).to(dt))
                r.sub_((q.float() * alpha).to(dt))
                pr.bp(r, z, output_scale=sc)
                g2 = dot(z, z)
                beta = (g2 / gamma).float()
                p.copy_((z.float() + p.float() * beta).to(dt))
                gamma = g2
            torch.cuda.synchronize()
            t_cgls = time.perf_counter() - t0
            pr.fp(xr, q, output_scale=sc)
            res = float((bh.double() - q.double()).norm() / bh.double().norm())
            diff = (float(torch.linalg.vector_norm((xr.float() * sc - rec32).double()) /
                          torch.linalg.vector_norm(rec32.double())) if rec32 is not None else None)
            del xr, r, p, q, z
        out[name] = {"fp_ms": ms_fp, "bp_ms": ms_bp, "fp_gups": ups / ms_fp / 1e6, "bp_gups": ups / ms_bp / 1e6,
                     "fp_rel_l2_vs_oracle": err, "oracle_views": sel,
                     "cgls_iterations": args.c5_iters, "cgls_s": t_cgls, "cgls_s_per_iter": t_cgls / args.c5_iters,
                     "cgls_relative_residual": res, "cgls_rel_l2_vs_f32": diff}
        if dt != torch.float32:
            del b
        torch.cuda.empty_cache()
    clocks = sampler.stop()
    f32 = out.get("f32", next(iter(out.values())))
    value = 2 * ups / (f32["fp_ms"] + f32["bp_ms"]) / 1e6
    line = {"metric": "cone_vec FP+BP GUPS at 1024^3x1500 (C5), f32 storage", "value": value, "unit": "GUPS",
            "n_gpus": 1, "steps": 2, "warmup": 1, "ms_per_step": f32["fp_ms"] + f32["bp_ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f16/bf16 storage beside)",
            "data": "synthetic",
            "config": {"workload": "cone_vec %d^3 volume of 20 seeded ellipsoids, %d jittered views (0.5 px shift, "
                                   "0.1 deg tilt), 1280x1024 detector, SOD 1500, ODD 600; CGLS %d iterations"
                                   % (n, na, args.c5_iters), "workload_kind": "c5"},
            "storage": out, "e2e": None, "clocks": clocks, "roofline": None, "cpu_baseline": None}
    print(json.dumps(line))
    return 0


def run_workload(args):
    """--workload fdk | sirt3d | cgls3d on the same 512^3 x 720 cone geometry.

    fdk: one step = b2t_fdk (pre-weighting, Ram-Lak filter on the tensor
    cores, FDK backprojection) of the phantom's projections; metric volumes/s.
    sirt3d / cgls3d: SIRT3D_CUDA / CGLS3D_CUDA through astra.algorithm on the
    phantom's exact projections (CUDA-graph iterations), one step = one
    iteration; metric seconds per iteration, with the relative residual
    |b - Ax| / |b| reached after warm-up + timed iterations."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    astra, vg, pg = workload(args.n, args.views, args.det)
    lib = importlib.import_module("astra-toolbox_b200._lib").load()
    lib.b2t_kernel_launches.restype = ctypes.c_uint64
    P = importlib.import_module("astra-toolbox_b200.projector")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    pr = astra.Projector3D(pg, vg)
    vol = ph.ellipsoids(pr.vol_shape, N_ELL, seed=0, device=dev)
    proj = torch.zeros(pr.proj_shape, device=dev)
    pr.fp(vol, proj)
    stream = torch.cuda.current_stream(dev)
    sampler = ClockSampler(0)
    extra = {}
    if args.workload == "fdk":
        rec = torch.zeros(pr.vol_shape, device=dev)
        for _ in range(args.warmup):
            P.fdk(pr, proj, rec)
        sampler.start()
        time.sleep(0.3)
        l0 = lib.b2t_kernel_launches()
        ms = _timed_region(torch, stream, lambda: P.fdk(pr, proj, rec), args.steps)
        launches = lib.b2t_kernel_launches() - l0
        clocks = sampler.stop()
        # the filter alone (in place on a copy): split, taps, tcgen05 GEMM
        work = proj.clone()
        ms_filter = _timed_region(torch, stream, lambda: P.fdk_weight_filter(pr, work), 3)
        nv, na, nu = pr.proj_shape
        flops_alg = 2.0 * nv * na * nu * nu
        kh = (nu + 1) // 2
        flops_tc = 6 * 2 * (2.0 * nv * na * kh * kh)
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"bf16_tflops": 1590.0}
        tpeak = peaks.get("bf16_tflops", 1590.0)
        roof = {"bound": "tensor", "kernel": "ramp filter (b2t_fdk_weight_filter: split + tcgen05 Toeplitz GEMM)",
                "achieved": flops_alg / (ms_filter * 1e-3) / 1e12, "peak": tpeak, "unit": "TFLOP/s",
                "frac": flops_alg / (ms_filter * 1e-3) / 1e12 / tpeak, "traffic": None,
                "algorithmic_flops": flops_alg, "tensor_flops_executed": flops_tc,
                "tensor_achieved_tflops": flops_tc / (ms_filter * 1e-3) / 1e12,
                "note": "algorithmic = 2 M nu^2 (the dense Toeplitz product, M = det rows x views); executed = "
                        "6 split-BF16 products x 2 parities x 2 M (nu/2)^2; duration includes the split kernel"}
        value, unit, hib = 1e3 / ms, "volumes/s", True
        metric = "FDK volumes/s at 512^3x720"
        extra = {"filter_ms": ms_filter, "fdk_ms": ms}
        # end to end: host projections in, host volume out
        hproj = proj.cpu().pin_memory()
        hrec = torch.empty(pr.vol_shape).pin_memory()
        dproj = torch.empty_like(proj)

        def serial_step():
            dproj.copy_(hproj, non_blocking=True)
            P.fdk(pr, dproj, rec)
            hrec.copy_(rec, non_blocking=True)

        serial_step()
        sms = _timed_region(torch, stream, serial_step, max(1, min(args.steps, 3)))
        # the library's host-data entry point (b2t_fdk_host): angle blocks
        # uploaded while earlier ones are filtered and backprojected, the last
        # block's volume downloaded in z-chunks as they are final; blocking,
        # timed on the host clock
        ke = max(1, min(args.steps, 3))
        for _ in range(2):
            P.fdk_host(pr, hproj, hrec)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(ke):
            P.fdk_host(pr, hproj, hrec)
        ems = (time.perf_counter() - t0) * 1e3 / ke
        e2e = {"value": 1e3 / ems, "unit": unit, "h2d_bytes_per_step": proj.numel() * 4,
               "d2h_bytes_per_step": rec.numel() * 4, "ms_per_step": ems,
               "path": "projector.fdk_host on pinned host projections and volume (b2t_fdk_host: transfers "
                       "pipelined with the filter and backprojection in angle blocks); host clock around the "
                       "blocking calls",
               "serial_path": {"value": 1e3 / sms, "ms_per_step": sms,
                               "path": "copy in, fdk(), copy out on one stream (CUDA events)"}}
        if not args.no_ref_cuda:
            P.fdk(pr, proj, rec)
            extra["ref_cuda"] = ref_algo_fdk(torch, args, proj, rec)
            if "s" in extra["ref_cuda"]:
                extra["ref_cuda"]["speedup"] = extra["ref_cuda"]["s"] / (ms * 1e-3)
    else:
        D3 = importlib.import_module("astra-toolbox_b200.data3d")
        A = importlib.import_module("astra-toolbox_b200.algorithm")
        pid = D3.link('-proj3d', pg, proj)
        rid = D3.create('-vol', vg, 0)
        cfg = A.astra_dict('SIRT3D_CUDA' if args.workload == "sirt3d" else 'CGLS3D_CUDA')
        cfg['ProjectionDataId'] = pid
        cfg['ReconstructionDataId'] = rid
        cfg['option'] = {'UseGraph': True}
        aid = A.create(cfg)
        A.run(aid, args.warmup)
        sampler.start()
        time.sleep(0.3)
        l0 = lib.b2t_kernel_launches()
        ms = _timed_region(torch, stream, lambda: A.run(aid, args.steps), 1) / args.steps
        launches = lib.b2t_kernel_launches() - l0
        restart = None
        if args.workload == "cgls3d" and args.steps > 1:
            # CGLS restarts (r = b - A x, p = A^T r) on every run call, as the
            # reference's CGLS3D_CUDA does: time a one-iteration run too and
            # report the iteration and the restart apart
            ms1 = _timed_region(torch, stream, lambda: A.run(aid, 1), 1)
            total = ms * args.steps
            ms = (total - ms1) / (args.steps - 1)
            restart = ms1 - ms
        clocks = sampler.stop()
        res = A.get_res_norm(aid)
        bnorm = float(proj.double().norm())
        A.delete(aid)
        D3.delete([pid, rid])
        ref_block = None
        if not args.no_ref_cuda:
            kind = 'SIRT3D_CUDA' if args.workload == "sirt3d" else 'CGLS3D_CUDA'

            def our_run(k):
                rid2 = D3.create('-vol', vg, 0)
                pid2 = D3.link('-proj3d', pg, proj)
                c2 = A.astra_dict(kind)
                c2['ProjectionDataId'] = pid2
                c2['ReconstructionDataId'] = rid2
                c2['option'] = {'UseGraph': True}
                a2 = A.create(c2)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                A.run(a2, k)
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                r = A.get_res_norm(a2) / bnorm
                A.delete(a2)
                D3.delete([pid2, rid2])
                return dt, r

            ref_block = ref_algo_iterative(torch, args, kind, proj, our_run)
        value, unit, hib = ms * 1e-3, "s/iter", False
        metric = ("SIRT3D" if args.workload == "sirt3d" else "CGLS3D") + " s/iter at 512^3x720"
        extra = {"iterations_before_residual": args.warmup + args.steps + (1 if restart is not None else 0),
                 "relative_residual": res / bnorm if bnorm > 0 else None}
        if restart is not None:
            extra["restart_ms_per_run"] = restart
            extra["timing"] = ("run(steps) and run(1) timed; s/iter = (T_steps - T_1) / (steps - 1), the "
                               "restart every run call does is reported apart")
        if ref_block is not None:
            extra["ref_cuda"] = ref_block
        roof = None
        e2e = None
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(args.n, args.views, args.det, {"workload_kind": args.workload}),
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks, "roofline": roof, "cpu_baseline": None}
    line.update(extra)
    print(json.dumps(line))
    return 0


def run_extra(args):
    """--workload stream | sart2d | cyl | matched.

    stream: FP + BP of the cone workload from pinned host memory through a
    device budget (--budget-gb, default 4) that forces z-slabs and angle
    blocks (b2t_fp3d_host / b2t_bp3d_host); one step = one FP + one BP,
    host to host; metric GUPS of the pair (2 x Nx Ny Nz Nangles / time),
    timed on the host clock around the blocking calls; the device-resident
    FP + BP time is reported beside it.
    sart2d: SART_CUDA on a 256^2 parallel-beam problem (180 views over pi,
    384 detectors), sequential order, CUDA-graph steps; one step = one sweep
    (180 single-view updates); metric sweeps/s.
    cyl: cyl_cone_vec FP + BP, 256^3 volume, 360 views, 256 x 384 detector on
    a cylinder centred at the source; metric GUPS of the pair.
    matched: the exact transpose of the FP (projection kernel matched_bp, the
    autograd backward) on the cone workload; one step = one matched BP of the
    phantom's projections; metric GUPS (Nx Ny Nz Nangles / time), with the
    dot-product test <A x, y> = <x, A^T y> (FP64 sums) of this run's output
    and the path statistics (B2T_MATCHED_PATH=slab selects the slab
    transpose)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    astra = importlib.import_module("astra-toolbox_b200")
    lib = importlib.import_module("astra-toolbox_b200._lib").load()
    lib.b2t_kernel_launches.restype = ctypes.c_uint64
    P = importlib.import_module("astra-toolbox_b200.projector")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    stream = torch.cuda.current_stream(dev)
    sampler = ClockSampler(0)
    extra, roof, e2e = {}, None, None
    if args.workload == "stream":
        astra, vg, pg = workload(args.n, args.views, args.det)
        pr = astra.Projector3D(pg, vg)
        vol = ph.ellipsoids(pr.vol_shape, N_ELL, seed=0, device=dev)
        dproj = torch.zeros(pr.proj_shape, device=dev)
        drec = torch.zeros(pr.vol_shape, device=dev)
        hvol = vol.cpu().pin_memory()
        hproj = torch.zeros(pr.proj_shape).pin_memory()
        hrec = torch.zeros(pr.vol_shape).pin_memory()
        budget = int(args.budget_gb * 1e9)
        astra.set_gpu_index(0, memory=budget)
        plan = {op: P.stream_plan(pr, op) for op in ("fp", "bp")}

        def step():
            P.fp3d_host(pr, hvol, hproj)
            P.bp3d_host(pr, hproj, hrec)

        for _ in range(args.warmup):
            step()
        sampler.start()
        time.sleep(0.3)
        l0 = lib.b2t_kernel_launches()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        ms = (time.perf_counter() - t0) * 1e3 / args.steps
        launches = lib.b2t_kernel_launches() - l0
        clocks = sampler.stop()
        astra.set_gpu_index(0, memory=0)
        ms_dev = _timed_region(torch, stream, lambda: (pr.fp(vol, dproj), pr.bp(dproj, drec)), max(1, args.steps))
        ups = 2.0 * np.prod(pr.vol_shape) * pr.proj_shape[1]
        value, unit, hib = ups / (ms * 1e-3) / 1e9, "GUPS", True
        metric = "streamed FP+BP GUPS at %d^3x%d from host memory, %.1f GB device budget" % (
            args.n, args.views, args.budget_gb)
        extra = {"device_resident_ms": ms_dev, "device_resident_gups": ups / (ms_dev * 1e-3) / 1e9,
                 "plan": {"fp_slab_z": plan["fp"][0], "fp_block_views": plan["fp"][1],
                          "bp_slab_z": plan["bp"][0], "bp_block_views": plan["bp"][1]},
                 "host_bytes_per_step": int(2 * (hvol.numel() + hproj.numel()) * 4),
                 "timing": "host clock around the blocking host-to-host calls"}
        e2e = {"value": value, "unit": unit, "h2d_bytes_per_step": int((hvol.numel() + hproj.numel()) * 4),
               "d2h_bytes_per_step": int((hproj.numel() + hrec.numel()) * 4), "ms_per_step": ms,
               "path": "b2t_fp3d_host + b2t_bp3d_host (every byte in and out of host memory)"}
        cfgd = config_dict(args.n, args.views, args.det, {"workload_kind": "stream", "budget_gb": args.budget_gb})
    elif args.workload == "sart2d":
        ang = np.linspace(0, np.pi, 180, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(256, 256)
        pg = astra.create_proj_geom('parallel', 1.0, 384, ang)
        pr = astra.Projector2D(pg, vg)
        x = ph.ellipsoids((1, 256, 256), 10, seed=0, axes=(10.0, 80.0), device=dev)[0].contiguous()
        b = torch.zeros(pr.proj_shape, device=dev)
        pr.fp(x, b)
        D2 = importlib.import_module("astra-toolbox_b200.data2d")
        A = importlib.import_module("astra-toolbox_b200.algorithm")
        sid = D2.link('-sino', pg, b)
        rid = D2.create('-vol', vg, 0)
        cfg = A.astra_dict('SART_CUDA')
        cfg['ProjectionDataId'] = sid
        cfg['ReconstructionDataId'] = rid
        cfg['option'] = {'UseGraph': True, 'ProjectionOrder': 'sequential'}
        aid = A.create(cfg)
        A.run(aid, 180 * args.warmup)
        sampler.start()
        time.sleep(0.3)
        l0 = lib.b2t_kernel_launches()
        ms = _timed_region(torch, stream, lambda: A.run(aid, 180), args.steps)
        launches = lib.b2t_kernel_launches() - l0
        clocks = sampler.stop()
        res = A.get_res_norm(aid)
        A.delete(aid)
        D2.delete([sid, rid])
        value, unit, hib = 1e3 / ms, "sweeps/s", True
        metric = "SART_CUDA sweeps/s at 256^2, 180 views, 384 detectors"
        extra = {"us_per_view_step": ms * 1e3 / 180, "relative_residual": res / float(b.double().norm()),
                 "sweeps_before_residual": args.warmup + args.steps}
        cfgd = {"workload": "SART_CUDA, 256^2 parallel beam, 180 views over pi, 384 detectors, 10 seeded ellipses, "
                            "sequential order", "workload_kind": "sart2d"}
    elif args.workload == "matched":
        astra, vg, pg = workload(args.n, args.views, args.det)
        pr = astra.Projector3D(pg, vg, {'ProjectionKernel': 'matched_bp'})
        vol = ph.ellipsoids(pr.vol_shape, N_ELL, seed=0, device=dev)
        proj = torch.zeros(pr.proj_shape, device=dev)
        pr.fp(vol, proj)
        rec = torch.zeros(pr.vol_shape, device=dev)
        for _ in range(args.warmup):
            pr.bp(proj, rec)
        st = (ctypes.c_uint64 * 4)()
        lib.b2t_matched_path_stats(st)
        sampler.start()
        time.sleep(0.3)
        l0 = lib.b2t_kernel_launches()
        ms = _timed_region(torch, stream, lambda: pr.bp(proj, rec), args.steps)
        launches = lib.b2t_kernel_launches() - l0
        clocks = sampler.stop()
        lib.b2t_matched_path_stats(st)
        x = ph.ellipsoids(pr.vol_shape, N_ELL, seed=1, device=dev)
        ax = torch.zeros(pr.proj_shape, device=dev)
        pr.fp(x, ax)
        lhs = float(torch.sum(ax.double() * proj.double()))
        rhs = float(torch.sum(x.double() * rec.double()))
        ups = float(np.prod(pr.vol_shape)) * pr.proj_shape[1]
        value, unit, hib = ups / (ms * 1e-3) / 1e9, "GUPS", True
        metric = "matched BP (exact FP transpose) GUPS at %d^3x%d" % (args.n, args.views)
        path = "slab" if os.environ.get("B2T_MATCHED_PATH") == "slab" else "scatter"
        extra = {"path": path, "dot_test_rel": abs(lhs - rhs) / abs(lhs),
                 "path_stats": {"slices_in_smem": int(st[0]), "slices_global": int(st[1]),
                                "slab_launches": int(st[2]), "scatter_launches": int(st[3])}}
        cfgd = config_dict(args.n, args.views, args.det, {"workload_kind": "matched"})
    else:
        n, na, rows, cols = 256, 360, 256, 384
        sod, odd = 600.0, 300.0
        vecs = []
        for i in range(na):
            t = 2 * np.pi * i / na
            src = [np.sin(t) * sod, -np.cos(t) * sod, 0.0]
            det = [-np.sin(t) * odd, np.cos(t) * odd, 0.0]
            u = [np.cos(t) * 1.4, np.sin(t) * 1.4, 0.0]
            vecs.append(src + det + u + [0.0, 0.0, 1.4, sod + odd])
        vg = astra.create_vol_geom(n, n, n)
        pg = astra.create_proj_geom('cyl_cone_vec', rows, cols, np.array(vecs))
        pr = astra.Projector3D(pg, vg)
        vol = ph.ellipsoids(pr.vol_shape, N_ELL, seed=0, axes=(10.0, 100.0), device=dev)
        proj = torch.zeros(pr.proj_shape, device=dev)
        rec = torch.zeros(pr.vol_shape, device=dev)

        def step():
            pr.fp(vol, proj)
            pr.bp(proj, rec)

        for _ in range(args.warmup):
            step()
        sampler.start()
        time.sleep(0.3)
        l0 = lib.b2t_kernel_launches()
        ms = _timed_region(torch, stream, step, args.steps)
        launches = lib.b2t_kernel_launches() - l0
        clocks = sampler.stop()
        ms_fp = _timed_region(torch, stream, lambda: pr.fp(vol, proj), max(1, args.steps))
        ups = 2.0 * n ** 3 * na
        value, unit, hib = ups / (ms * 1e-3) / 1e9, "GUPS", True
        metric = "cyl_cone_vec FP+BP GUPS at 256^3x360"
        extra = {"fp_ms": ms_fp, "bp_ms": ms - ms_fp}
        cfgd = {"workload": "cyl_cone_vec FP+BP, 256^3 volume, 360 views over 2pi, 256x384 detector on a cylinder "
                            "of radius SOD+ODD=900 centred at the source, SOD 600", "workload_kind": "cyl"}
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfgd, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clocks, "roofline": roof, "cpu_baseline": None}
    line.update(extra)
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
    ap.add_argument("--ref-views", type=int, default=2, help="FP views per step of --impl reference")
    ap.add_argument("--ref-slices", type=int, default=1, help="BP z-slices per step of --impl reference")
    ap.add_argument("--parity-views", type=int, default=4, help="FP views of the CPU baseline / parity sample")
    ap.add_argument("--parity-slices", type=int, default=3, help="BP z-slices of the CPU baseline / parity sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip timing the reference's CUDA build")
    ap.add_argument("--ref-iters", type=int, default=30,
                    help="iterations of the reference's SIRT3D / CGLS3D whose residual is the target")
    ap.add_argument("--workload", default="fpbp",
                    choices=["fpbp", "fdk", "sirt3d", "cgls3d", "batch2d", "stream", "sart2d", "cyl", "c1", "c5",
                             "matched"])
    ap.add_argument("--c5-views", type=int, default=1500)
    ap.add_argument("--c5-iters", type=int, default=30)
    ap.add_argument("--c5-types", default="f32,f16,bf16")
    ap.add_argument("--budget-gb", type=float, default=4.0, help="device budget of --workload stream")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch2d":
        return run_batch2d(args)
    if args.workload == "c1":
        return run_c1(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.workload in ("stream", "sart2d", "cyl", "matched"):
        return run_extra(args)
    if args.workload != "fpbp":
        return run_workload(args)

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

    # end to end through the public API with host buffers.  Headline: the
    # host-data entry points (projector.fp3d_host / bp3d_host, i.e.
    # b2t_fp3d_host / b2t_bp3d_host), which pipeline the transfers with the
    # kernels in angle blocks; beside it the device-data path with the
    # copies around it (copy in, direct_FP3D / direct_BP3D, copy out).
    e2e = None
    if not args.no_e2e:
        P = importlib.import_module("astra-toolbox_b200.projector")
        hvol = vol.cpu().pin_memory()
        hproj = torch.empty(pr.proj_shape, dtype=tdt).pin_memory()
        hback = torch.empty(pr.vol_shape, dtype=tdt).pin_memory()
        esz = vol.element_size()
        vb = vol.numel() * esz
        pb = proj.numel() * esz
        ke = max(1, min(args.steps, 3))

        def host_step():
            P.fp3d_host(pr, hvol, hproj)
            P.bp3d_host(pr, hproj, hback)

        host_path = args.dtype == "float32"  # the host-data entry points take FP32
        if host_path:
            for _ in range(2):
                host_step()
            torch.cuda.synchronize(dev)
            barrier()
            t0 = time.perf_counter()
            for _ in range(ke):
                host_step()  # blocking: returns with the results in host memory
            torch.cuda.synchronize(dev)
            et = torch.tensor([(time.perf_counter() - t0) * 1e3 / ke], device=dev, dtype=torch.float64)
            if world > 1:
                dist.all_reduce(et, op=dist.ReduceOp.MAX)

        dvol = torch.empty_like(vol)
        dproj = torch.empty_like(proj)
        dback = torch.empty_like(back)

        def device_step():
            dvol.copy_(hvol, non_blocking=True)
            pr.fp(dvol, dproj)
            hproj.copy_(dproj, non_blocking=True)
            dproj.copy_(hproj, non_blocking=True)
            pr.bp(dproj, dback)
            hback.copy_(dback, non_blocking=True)

        for _ in range(2):
            device_step()
        torch.cuda.synchronize(dev)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ke):
            device_step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        dt = torch.tensor([e0.elapsed_time(e1) / ke], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(dt, op=dist.ReduceOp.MAX)
        dpath = {"value": 2 * updates * world / (float(dt.item()) * 1e-3) / 1e9, "ms_per_step": float(dt.item()),
                 "path": "copy in, Projector3D.fp, copy out, copy in, Projector3D.bp, copy out on one stream "
                         "(CUDA events)"}
        if not host_path:
            e2e = {"value": dpath["value"], "unit": "GUPS", "h2d_bytes_per_step": vb + pb,
                   "d2h_bytes_per_step": pb + vb, "ms_per_step": dpath["ms_per_step"], "path": dpath["path"]}
        else:
            e2e = {"value": 2 * updates * world / (float(et.item()) * 1e-3) / 1e9, "unit": "GUPS",
                   "h2d_bytes_per_step": vb + pb, "d2h_bytes_per_step": pb + vb,
                   "ms_per_step": float(et.item()),
                   "path": "projector.fp3d_host then projector.bp3d_host on pinned host arrays (b2t_fp3d_host / "
                           "b2t_bp3d_host: volume copied in, projections copied out and in again, volume "
                           "copied out, transfers pipelined with the kernels in angle blocks); host clock "
                           "around the blocking calls",
                   "device_data_path": dpath}
        del dvol, dproj, dback

    # CPU baseline and parity: the FP64 oracle on a sample of this workload
    # (views of the FP, z-slices of the BP), run once after the timed region
    # on the same inputs; its outputs are compared with this run's GPU
    # outputs on the same views and slices (the full-size accuracy of the
    # timed configuration)
    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu:
        vcpu = vol.float().cpu().numpy()
        pcpu = proj.float().cpu().numpy()
        threads = os.cpu_count() or 1
        fp_sel = sample_views(args.views, args.parity_views)
        bp_sl = sample_slices(args.n, args.parity_slices)
        nv_, na_, nu_ = pr.proj_shape
        r = oracle_sample(vcpu, pcpu, pr.geom.views_array(), pr.geom.vol_scale, nu_, nv_, fp_sel, bp_sl, threads)
        dt = r["fp_s"] + r["bp_s"]
        cpu = {"value": r["units"] / dt / 1e9, "unit": "GUPS", "cores": threads, "kind": "port",
               "sample": "FP64 oracle (CPU port of the reference's cone model) on %d host threads: forward "
                         "projection of views %s (all %d^2 rays, %.1f s) and backprojection of z-slices %s over "
                         "all %d views (%.1f s); GUPS = their voxel-view updates / time"
                         % (threads, fp_sel, args.det, r["fp_s"], bp_sl, args.views, r["bp_s"])}
        del pcpu

        def rl2(a, b):
            return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

        got_fp = proj[:, fp_sel, :].double().cpu().numpy()
        got_bp = back[bp_sl].double().cpu().numpy()
        parity = {"fp_rel_l2_vs_oracle": rl2(got_fp, r["fp"]), "fp_views": fp_sel,
                  "bp_rel_l2_vs_oracle": rl2(got_bp, r["bp"]), "bp_slices": bp_sl,
                  "fp_rel_l2_worst_view": max(rl2(got_fp[:, i], r["fp"][:, i]) for i in range(len(fp_sel))),
                  "bp_rel_l2_worst_slice": max(rl2(got_bp[i], r["bp"][i]) for i in range(len(bp_sl))),
                  "tolerance": 1e-5 if args.dtype == "float32" else None,
                  "oracle": "FP64 restatement of cone_fp.cu:154-231 / cone_bp.cu:55-133 (oracle/b2t_oracle.c) on "
                            "this run's inputs: FP of the phantom, BP of this run's FP output"}
    ref_cuda = None
    if rank == 0 and not args.no_ref_cuda:
        ref_cuda = ref_cuda_block(torch, dev, vol, proj, back, args)
        if "fp_ms" in ref_cuda:
            ref_cuda["fp_speedup"] = ref_cuda["fp_ms"] / fp_ms
            ref_cuda["bp_speedup"] = ref_cuda["bp_ms"] / bp_ms
            ref_cuda["fpbp_speedup"] = (ref_cuda["fp_ms"] + ref_cuda["bp_ms"]) / ms_step

    # roofline of the dominant call (the larger of FP and BP).  The projectors
    # are bound by on-chip interpolation reads, not by HBM: the forward
    # projector reads a 4-texel bilinear footprint per ray sample (through L1),
    # the backprojector a 4-texel footprint per voxel-view update (from
    # TMA-staged shared memory).  Algorithmic on-chip bytes = units x 4 texels
    # x element size; units = det_u * det_v * views * N (the reference's loop
    # trip count along the dominant axis) for FP, N^3 * views for BP.  The roof
    # is the measured streaming load bandwidth of L1 (FP) or shared memory (BP)
    # on this GPU.  The compulsory HBM bytes are reported beside it.
    esz = vol.element_size()
    vol_bytes = vol.numel() * esz
    proj_bytes = proj.numel() * esz
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak_hbm = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak_hbm, peak_src = 6650.0, "fallback"
    onchip = {}
    for which, name in ((0, "smem"), (1, "l1")):
        g = ctypes.c_double(0.0)
        st = lib.b2t_onchip_peak(which, ctypes.byref(g))
        onchip[name] = g.value if st == 0 else None
    dom = "fp" if fp_ms >= bp_ms else "bp"
    dom_ms = max(fp_ms, bp_ms)
    if dom == "fp":
        units = float(args.det) * args.det * args.views * args.n
        hbm_bytes = vol_bytes + proj_bytes  # compulsory: volume read once, projections written once
        peak_on = onchip["l1"]
    else:
        units = updates
        hbm_bytes = proj_bytes + vol_bytes  # compulsory: projections read once, volume written once
        peak_on = onchip["smem"]
    alg_bytes = units * 4 * esz
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    # DRAM bytes (read + write) of the dominant call's launches, per call.
    # FP: the bytes per sample of one ncu capture of the FP kernel at 384^3 x
    # 360 views, 624^2 (21.43 GB for 744.6 M warp-samples of 32 rays; profiles/
    # cone_fp_slab_384cube_360views.md) times this call's samples; BP: one
    # capture of this exact workload (profiles/dram_traffic_cone_fpbp_512cube_
    # 720views.md).  Null for other workloads and storage types.
    traffic, traffic_src = None, None
    if (args.n, args.views, args.det, args.dtype) == (N_VOX, N_ANG, N_DET, "float32"):
        if dom == "fp":
            traffic = (20.96 + 0.47) * 1e9 / (744633280.0 * 32) * units
            traffic_src = "scaled by samples from an ncu capture of the FP at 384^3 x 360 views, 624^2"
        else:
            traffic = (15.87 + 0.53 + 0.95 + 0.50) * 1e9
            traffic_src = "ncu capture of this workload"
    hbm_achieved = hbm_bytes / (dom_ms * 1e-3) / 1e9
    roofline = {"bound": "l1" if dom == "fp" else "smem",
                "kernel": "b2t_fp3d" if dom == "fp" else "b2t_bp3d",
                "achieved": achieved, "peak": peak_on, "unit": "GB/s",
                "frac": (achieved / peak_on) if peak_on else None,
                "traffic": traffic, "units_per_launch": units, "bytes_per_unit": 4 * esz,
                "traffic_note": "DRAM bytes of one whole call (the FP's x- and y-major launches, or the BP's "
                                "launch), %s; the slice boxes / tiles are re-read on chip, DRAM moves about "
                                "1/18 of the algorithmic bytes" % traffic_src,
                "peak_source": "measured on this GPU by b2t_onchip_peak (16-byte streaming loads); the FP "
                               "reads its samples from TMA-staged shared memory, whose measured roof is "
                               "within 1 % of the L1 one",
                "onchip_peaks_gbs": onchip,
                "hbm": {"achieved": hbm_achieved, "peak": peak_hbm, "frac": hbm_achieved / peak_hbm,
                        "compulsory_bytes": hbm_bytes, "peak_source": peak_src},
                "note": "duration = the whole b2t call (CUDA events), including its layout kernel; "
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
                "cpu_baseline": cpu, "parity": parity, "ref_cuda": ref_cuda}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
