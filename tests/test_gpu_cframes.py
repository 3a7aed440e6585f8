"""GPU tests of iarray_b200_opt_gemm_cframes (host frames in, host frame out, pipelined
per chunk row of C).  Its frame must be byte-identical to the one the reference's call
sequence produces through this library: iarray_from_cframe(a), iarray_from_cframe(b),
iarray_opt_gemm, iarray_to_cframe."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _frames(ia, ctx, A, B, ca, ba, cb, bb):
    fa = ia.Container.from_numpy(ctx, A, ca, ba).to_cframe()
    fb = ia.Container.from_numpy(ctx, B, cb, bb).to_cframe()
    return fa, fb


def _sequential(ia, ctx, fa, fb, cc, bc):
    a = ia.Container.from_cframe(ctx, fa)
    b = ia.Container.from_cframe(ctx, fb)
    return ia.opt_gemm(ctx, a, b, cc, bc).to_cframe()


@pytest.mark.parametrize("form", ["native", "split"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("M,K,N,c0,c1,c2,b", [
    (300, 257, 200, 64, 128, 96, 32),      # ragged last band, ragged chunks in every dimension
    (512, 512, 512, 128, 128, 128, 64),    # four full bands
    (70, 33, 50, 70, 33, 50, 11),          # one band
    (200, 100, 150, 50, 100, 75, 25),      # column chunks off 16-byte boundaries
])
def test_cframes_matches_sequential_calls(ia, form, dtype, M, K, N, c0, c1, c2, b):
    ctx = ia.Context(form=ia.FORM_SPLIT if form == "split" else ia.FORM_NATIVE, encoder=ia.ENCODER_PARALLEL)
    rng = np.random.default_rng(M + K + N)
    A = (rng.uniform(-1, 1, (M, K)) * np.exp2(rng.integers(-8, 9, (M, K)))).astype(dtype)
    B = (rng.uniform(-1, 1, (K, N)) * np.exp2(rng.integers(-8, 9, (K, N)))).astype(dtype)
    fa, fb = _frames(ia, ctx, A, B, (c0, c1), (b, b), (c1, c2), (b, b))
    want = _sequential(ia, ctx, fa, fb, (c0, c2), (b, b))
    out, n = ia.opt_gemm_cframes(ctx, fa, fb, (c0, c2), (b, b))
    assert n == len(want)
    assert out[:n].tobytes() == want
    c = ia.Container.from_cframe(ctx, out[:n].tobytes()).to_numpy()
    ref = A.astype(np.float64) @ B.astype(np.float64)
    tol = 1e-13 if dtype == np.float64 else 1e-4
    assert np.linalg.norm(c - ref) <= tol * np.linalg.norm(ref)


def test_cframes_pinned_buffers_and_repeat(ia):
    import torch
    ctx = ia.Context(form=ia.FORM_SPLIT, encoder=ia.ENCODER_PARALLEL)
    rng = np.random.default_rng(9)
    A, B = rng.standard_normal((640, 384)), rng.standard_normal((384, 320))
    fa, fb = _frames(ia, ctx, A, B, (128, 128), (32, 32), (128, 64), (32, 32))

    def pinned(x):
        t = torch.empty(len(x), dtype=torch.uint8, pin_memory=True).numpy()
        t[:] = np.frombuffer(x, np.uint8)
        return t
    pa, pb = pinned(fa), pinned(fb)
    out = torch.empty(640 * 320 * 8 * 2 + (1 << 20), dtype=torch.uint8, pin_memory=True).numpy()
    want = _sequential(ia, ctx, fa, fb, (128, 64), (32, 32))
    for _ in range(3):
        out[:] = 0xAB
        _, n = ia.opt_gemm_cframes(ctx, pa, pb, (128, 64), (32, 32), out=out)
        assert out[:n].tobytes() == want


def test_cframes_too_small_buffer_reports_length(ia):
    ctx = ia.Context()
    rng = np.random.default_rng(10)
    A, B = rng.standard_normal((200, 100)), rng.standard_normal((100, 150))
    fa, fb = _frames(ia, ctx, A, B, (50, 100), (25, 50), (100, 75), (50, 25))
    want = _sequential(ia, ctx, fa, fb, (50, 75), (25, 25))
    small = np.zeros(100, np.uint8)
    with pytest.raises(ia.IArrayError) as e:
        ia.opt_gemm_cframes(ctx, fa, fb, (50, 75), (25, 25), out=small)
    assert "TOO_SMALL" in str(e.value) or "small" in str(e.value).lower()
    out = np.zeros(len(want), np.uint8)
    _, n = ia.opt_gemm_cframes(ctx, fa, fb, (50, 75), (25, 25), out=out)
    assert n == len(want) and out.tobytes() == want


def test_cframes_partition_errors(ia):
    ctx = ia.Context()
    A, B = np.ones((64, 32)), np.ones((32, 48))
    fa, fb = _frames(ia, ctx, A, B, (32, 32), (16, 16), (32, 48), (16, 16))
    with pytest.raises(ia.IArrayError):
        ia.opt_gemm_cframes(ctx, fa, fb, (16, 48), (16, 16))      # C chunk rows differ from A's
    with pytest.raises(ia.IArrayError):
        ia.opt_gemm_cframes(ctx, fa, fa, (32, 32), (16, 16))      # inner shapes differ
