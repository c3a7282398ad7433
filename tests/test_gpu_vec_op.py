"""b2t_vec_op (the processVol3D<op> / processData<op> replacement) through the
C ABI: every op against numpy on the 16-byte vector path (aligned, n a
multiple of 4) and the scalar path (an odd n, an offset pointer), including
opInvert's threshold (cuda/3d/arith3d.cu:87-94: values not above 1e-6 become
0).  The reference's ops compute out += a * b and similar as one contracted
FMA per element (nvcc's default), which numpy's float64 evaluation rounded
to float32 matches to one rounding."""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _lib():
    L = importlib.import_module("astra-toolbox_b200._lib")
    return L, L.load()


def _ref(op, o, a, b, s, L):
    o, a, b = o.astype(np.float64), a.astype(np.float64), b.astype(np.float64)
    s = float(np.float32(s))
    if op == L.OP_SET:
        r = np.full_like(o, s)
    elif op == L.OP_MUL_SCALAR:
        r = o * s
    elif op == L.OP_MUL:
        r = o * a
    elif op == L.OP_ADD_MUL:
        r = o + a * b
    elif op == L.OP_ADD_SCALED:
        r = o + a * s
    elif op == L.OP_SCALE_AND_ADD:
        r = a + o * s
    elif op == L.OP_INVERT:
        o32 = o.astype(np.float32)
        with np.errstate(divide="ignore"):
            r = np.where(o32 > np.float32(1e-6), np.float32(1.0) / o32, np.float32(0.0))  # IEEE float32 division
    elif op == L.OP_CLAMP_MIN:
        r = np.maximum(o, s)
    elif op == L.OP_CLAMP_MAX:
        r = np.minimum(o, s)
    elif op == L.OP_ADD:
        r = o + a
    return r.astype(np.float32)


OPS = ["OP_SET", "OP_MUL_SCALAR", "OP_MUL", "OP_ADD_MUL", "OP_ADD_SCALED", "OP_SCALE_AND_ADD", "OP_INVERT",
       "OP_CLAMP_MIN", "OP_CLAMP_MAX", "OP_ADD"]


@pytest.mark.parametrize("name", OPS)
@pytest.mark.parametrize("vector_path", [True, False])
def test_vec_op_vs_numpy(name, vector_path):
    L, lib = _lib()
    op = getattr(L, name)
    n = 1 << 20 if vector_path else (1 << 20) + 3
    off = 0 if vector_path else 1  # a 4-byte offset breaks the 16-byte alignment
    rng = np.random.default_rng(op)
    o = rng.standard_normal(n + off).astype(np.float32)
    if op == L.OP_INVERT:
        o = np.abs(o) * 1e-5  # straddles the 1e-6 threshold
        o[off:off + 4] = [1e-6, np.nextafter(np.float32(1e-6), np.float32(1)), 0.0, -1.0]
    a = rng.standard_normal(n + off).astype(np.float32)
    b = rng.standard_normal(n + off).astype(np.float32)
    s = 0.37
    to, ta, tb = (torch.from_numpy(v).cuda() for v in (o, a, b))
    st = lib.b2t_vec_op(op, to.data_ptr() + 4 * off, ta.data_ptr() + 4 * off, tb.data_ptr() + 4 * off, s, n,
                        torch.cuda.current_stream().cuda_stream)
    assert st == L.B2T_OK, lib.b2t_last_error()
    torch.cuda.synchronize()
    got = to.cpu().numpy()
    want = _ref(op, o[off:], a[off:], b[off:], s, L)
    assert got[:off].tobytes() == o[:off].tobytes()  # nothing written before the range
    if op in (L.OP_SET, L.OP_CLAMP_MIN, L.OP_CLAMP_MAX, L.OP_INVERT, L.OP_MUL, L.OP_MUL_SCALAR, L.OP_ADD):
        # one rounding of an exact result: bit-exact
        assert np.array_equal(got[off:], want)
    else:
        np.testing.assert_allclose(got[off:], want, rtol=2e-7, atol=1e-7)
    if op == L.OP_INVERT:
        assert got[off:off + 4].tolist() == [0.0, np.float32(1.0) / np.nextafter(np.float32(1e-6), np.float32(1)),
                                             0.0, 0.0]


def test_vec_op_rejects_bad_arguments():
    L, lib = _lib()
    t = torch.zeros(8, device='cuda')
    assert lib.b2t_vec_op(42, t.data_ptr(), None, None, 0.0, 8, None) == 1
    assert lib.b2t_vec_op(L.OP_ADD_MUL, t.data_ptr(), t.data_ptr(), None, 0.0, 8, None) == 1  # b missing
    assert lib.b2t_vec_op(L.OP_SET, None, None, None, 0.0, 8, None) == 1
    assert lib.b2t_vec_op(L.OP_SET, None, None, None, 0.0, 0, None) == L.B2T_OK  # empty: no work
