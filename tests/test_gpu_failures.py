"""Failure handling on the GPU, without faulting, trapping or hanging it.

- Bounded waits: b2t_selftest_bounded_wait runs the pipelined kernels' wait
  helper against an mbarrier phase and a device flag that nothing completes;
  the wait must give up within its limit, set the device error word and come
  back as B2T_ERR_TIMEOUT, and the context must stay usable.
- Allocation failures: b2t_debug_fail_alloc makes the n-th device allocation
  of a call fail (host-side injection, as a real out-of-memory would); every
  call must return B2T_ERR_NO_MEMORY cleanly, hold no allocation afterwards,
  and the next call must succeed with the right result.
- Abort: b2t_algo_abort from a second host thread stops a running SIRT3D
  between iterations (the reference's shouldAbort hook,
  src/CudaSirtAlgorithm3D.cpp:348, src/Globals.cpp:47-58).
"""
import ctypes
import importlib
import threading
import time

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _lib():
    L = importlib.import_module("astra-toolbox_b200._lib")
    return L, L.load()


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_gives_up_and_reports(astra, orc, which):
    L, lib = _lib()
    flags = ctypes.c_uint32(0)
    assert lib.b2t_device_errors(ctypes.byref(flags)) == L.B2T_OK  # start clean
    t0 = time.perf_counter()
    st = lib.b2t_selftest_bounded_wait(which, 20_000_000, None)  # ~10 ms at 2 GHz
    dt = time.perf_counter() - t0
    assert st == 6, (st, lib.b2t_last_error())  # B2T_ERR_TIMEOUT
    assert b"gave up" in lib.b2t_last_error()
    assert dt < 5.0
    # the error word was read and cleared by the call
    assert lib.b2t_device_errors(ctypes.byref(flags)) == L.B2T_OK and flags.value == 0
    # the context is still usable: a projection after the timeout is right
    ang = np.linspace(0, 2 * np.pi, 12, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(20, 24, 16)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 20, 28, ang, 100.0, 50.0)
    pr = astra.Projector3D(pg, vg)
    vol = np.random.default_rng(1).random(pr.vol_shape, dtype=np.float32)
    tp = torch.zeros(pr.proj_shape, device="cuda")
    pr.fp(torch.from_numpy(vol).cuda(), tp)
    nv, na, nu = pr.proj_shape
    ref = orc.fp3d(2, pr.geom.views_array(), vol, nu, nv, pr.geom.vol_scale)
    assert rel_l2(tp.cpu().numpy(), ref) < 1e-5


def test_bounded_wait_rejects_bad_arguments():
    L, lib = _lib()
    assert lib.b2t_selftest_bounded_wait(2, 1000, None) == 1
    assert lib.b2t_selftest_bounded_wait(0, 0, None) == 1
    assert lib.b2t_selftest_bounded_wait(0, 5_000_000_000, None) == 1


def _cases(astra):
    """Calls that allocate device memory, each returning its result."""
    P = importlib.import_module("astra-toolbox_b200.projector")
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D3 = importlib.import_module("astra-toolbox_b200.data3d")
    ang = np.linspace(0, 2 * np.pi, 24, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(24, 28, 20)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 26, 34, ang, 120.0, 60.0)
    pr = astra.Projector3D(pg, vg)
    g = torch.Generator().manual_seed(3)
    vol = torch.rand(pr.vol_shape, generator=g).cuda()
    proj = torch.rand(pr.proj_shape, generator=g).cuda()

    def fp():
        out = torch.zeros(pr.proj_shape, device="cuda")
        pr.fp(vol, out)
        return out

    def bp():
        out = torch.zeros(pr.vol_shape, device="cuda")
        pr.bp(proj, out)
        return out

    def fdk():
        out = torch.zeros(pr.vol_shape, device="cuda")
        P.fdk(pr, proj.clone(), out)
        return out

    def streamed_fp():
        out = torch.zeros(pr.proj_shape).pin_memory()
        P.fp3d_host(pr, vol.cpu().pin_memory(), out)
        return out.cuda()

    def algo(kind):
        def run():
            pid = D3.link('-proj3d', pg, proj.clone())
            rid = D3.create('-vol', vg, 0)
            cfg = A.astra_dict(kind)
            cfg['ProjectionDataId'] = pid
            cfg['ReconstructionDataId'] = rid
            try:
                aid = A.create(cfg)
                try:
                    A.run(aid, 3)
                finally:
                    A.delete(aid)
                return D3.get_shared(rid).clone()
            finally:
                D3.delete([pid, rid])
        return run

    return {"fp": fp, "bp": bp, "fdk": fdk, "streamed_fp": streamed_fp, "sirt3d": algo('SIRT3D_CUDA'),
            "cgls3d": algo('CGLS3D_CUDA')}


@pytest.mark.parametrize("case", ["fp", "bp", "fdk", "streamed_fp", "sirt3d", "cgls3d"])
def test_injected_allocation_failures_are_clean(astra, case):
    """Fail each allocation of the call in turn.  The call either returns
    B2T_ERR_NO_MEMORY holding nothing, or recovers (the FP falls back from the
    cell layout to the padded copy, which needs a quarter of the memory) with
    the same result to rounding; the next call runs normally."""
    L, lib = _lib()
    fn = _cases(astra)[case]
    want = fn().cpu().numpy()
    torch.cuda.synchronize()
    base = lib.b2t_debug_live_allocations()
    pending = ctypes.c_int64(0)
    outcomes = []
    try:
        for n in range(1, 40):
            assert lib.b2t_debug_fail_alloc(n, None) == L.B2T_OK
            try:
                got = fn()
                ok = True
            except L.AstraError as e:
                assert e.status == 4, str(e)  # B2T_ERR_NO_MEMORY
                assert "injected allocation failure" in str(e)
                ok = False
            torch.cuda.synchronize()
            assert lib.b2t_debug_fail_alloc(0, ctypes.byref(pending)) == L.B2T_OK
            assert lib.b2t_debug_live_allocations() == base, (case, n)
            if pending.value > 0:
                # the call made fewer than n allocations: every one was tried
                assert ok
                break
            outcomes.append(ok)
            if ok:
                assert rel_l2(got.cpu().numpy(), want) < 1e-5, (case, n)
        else:
            pytest.fail("the call made more than 39 allocations")
    finally:
        lib.b2t_debug_fail_alloc(0, None)
    assert len(outcomes) >= 1, outcomes
    if case == "fp":
        assert all(outcomes), outcomes  # every single failure is absorbed by the fallback
    else:
        assert not all(outcomes), outcomes
    got = fn()
    torch.cuda.synchronize()
    assert lib.b2t_debug_live_allocations() == base
    assert np.array_equal(got.cpu().numpy(), want)


def test_abort_from_another_thread(astra):
    L, lib = _lib()
    D3 = importlib.import_module("astra-toolbox_b200.data3d")
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    ang = np.linspace(0, 2 * np.pi, 24, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(24, 28, 20)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 26, 34, ang, 120.0, 60.0)
    proj = torch.rand((26, 24, 34), generator=torch.Generator().manual_seed(0)).cuda()
    pid = D3.link('-proj3d', pg, proj)
    rid = D3.create('-vol', vg, 0)
    cfg = A.astra_dict('SIRT3D_CUDA')
    cfg['ProjectionDataId'] = pid
    cfg['ReconstructionDataId'] = rid
    aid = A.create(cfg)
    outcome = {}

    def runner():
        t0 = time.perf_counter()
        try:
            A.run(aid, 10_000_000)
            outcome["status"] = 0
        except L.AstraError as e:
            outcome["status"] = e.status
            outcome["msg"] = str(e)
        torch.cuda.synchronize()
        outcome["s"] = time.perf_counter() - t0

    th = threading.Thread(target=runner)
    th.start()
    time.sleep(0.5)
    A.abort(aid)
    th.join(timeout=60)
    assert not th.is_alive()
    assert outcome["status"] == 5, outcome  # B2T_ERR_ABORTED
    assert "aborted after" in outcome["msg"]
    assert outcome["s"] < 30
    # the algorithm object stays usable: a later run of a few iterations works
    A.run(aid, 2)
    torch.cuda.synchronize()
    assert torch.isfinite(D3.get_shared(rid)).all()
    A.delete(aid)
    D3.delete([pid, rid])
