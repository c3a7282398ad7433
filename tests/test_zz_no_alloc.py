"""b2t_dot_f64_noalloc through the C ABI: the allocation-free FP64 inner
product, for callers that cannot allocate device memory at the point of the
call (a real-time loop that must not wait on the allocator, a host that hands
out all device memory from its own pool).  It launches with the same shape as
b2t_dot_f64, so on two calls in a row, the second smaller than the first (so
that partial sums left by the first call cannot leak into it), it must return
exactly the same bits.  Collected last on purpose."""
import ctypes
import importlib
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _lib():
    L = importlib.import_module("astra-toolbox_b200._lib")
    return L, L.load()


def _dot(name, a, b):
    L, lib = _lib()
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=a.device)
    st = getattr(lib, name)(a.data_ptr(), b.data_ptr(), a.numel(), L.F32, out.data_ptr(),
                            torch.cuda.current_stream(a.device).cuda_stream)
    assert st == L.B2T_OK, lib.b2t_last_error()
    torch.cuda.synchronize(a.device)
    return float(out.item())


@pytest.mark.gpu
def test_noalloc_dot_matches_allocating_dot_twice_in_a_row():
    g = torch.Generator(device="cuda").manual_seed(0)
    for n in (3_100_000, 1_500_001):
        a = torch.randn(n, device="cuda", generator=g)
        b = torch.randn(n, device="cuda", generator=g)
        want = _dot("b2t_dot_f64", a, b)
        got = _dot("b2t_dot_f64_noalloc", a, b)
        assert got == want, (n, got, want)
        # squared norm (b aliases a), as the CGLS steps use it
        want2 = _dot("b2t_dot_f64", a, a)
        got2 = _dot("b2t_dot_f64_noalloc", a, a)
        assert got2 == want2, (n, got2, want2)
        ref = float(np.dot(a.double().cpu().numpy(), b.double().cpu().numpy()))
        assert abs(got - ref) <= 1e-9 * max(1.0, abs(ref))


@pytest.mark.gpu
def test_noalloc_dot_speed_matches_allocating_dot():
    """Same launch shape, so the same time up to the allocator's share."""
    n = 64 << 20
    a = torch.randn(n, device="cuda")
    s = torch.cuda.current_stream()

    def timed(name):
        for _ in range(3):
            _dot(name, a, a)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        L, lib = _lib()
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        fn = getattr(lib, name)
        e0.record(s)
        for _ in range(20):
            fn(a.data_ptr(), a.data_ptr(), n, L.F32, out.data_ptr(), s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 20

    t_alloc = timed("b2t_dot_f64")
    t_noalloc = timed("b2t_dot_f64_noalloc")
    print("dot of %d floats: b2t_dot_f64 %.3f ms, b2t_dot_f64_noalloc %.3f ms" % (n, t_alloc, t_noalloc))
    assert t_noalloc <= 1.5 * t_alloc + 0.02


@pytest.mark.gpu
def test_noalloc_dot_rejects_sizes_beyond_its_scratch():
    L, lib = _lib()
    a = torch.zeros(16, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    n = 4096 * (1 << 20) + 1  # one element more than the fixed scratch covers
    st = lib.b2t_dot_f64_noalloc(a.data_ptr(), a.data_ptr(), n, L.F32, out.data_ptr(), None)
    assert st == L.B2T_OK + 1  # B2T_ERR_INVALID_ARG, raised before any device work
    assert b"exceed the maximum" in lib.b2t_last_error()
