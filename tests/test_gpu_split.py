"""GPU tests of the split-precision forms through the C ABI.

float64 (Ozaki scheme II on INT8 tensor cores): integer-valued products are exact; for
wide-range random data the normwise error against the double-double oracle must stay
within 4x the native FP64 path's error (the project's acceptance bar), and below 1e-14.
"""
import numpy as np
import pytest

import oracle as O
from ref_fixtures import GEMM

pytestmark = pytest.mark.gpu


def _split_ctx(ia):
    c = ia.Context()
    c.set_form(ia.FORM_SPLIT)
    return c


def _scaled(rng, shape):
    return rng.uniform(-1, 1, shape) * np.exp2(rng.integers(-8, 9, shape))


@pytest.mark.parametrize("M,K,N,cs,bs", [
    (300, 257, 200, 128, 32),        # ragged: M, N not tile multiples, K not a multiple of 128
    (256, 1024, 512, 256, 64),
    (129, 130, 257, 64, 16),
    (1000, 1000, 1000, 500, 100),
])
def test_split_f64_error_within_bar(ia, M, K, N, cs, bs):
    rng = np.random.default_rng(M + K + N)
    A, B = _scaled(rng, (M, K)), _scaled(rng, (K, N))
    sctx, nctx = _split_ctx(ia), ia.Context()
    Ac = ia.Container.from_numpy(nctx, A, (cs, cs), (bs, bs))
    Bc = ia.Container.from_numpy(nctx, B, (cs, cs), (bs, bs))
    cn = ia.opt_gemm(nctx, Ac, Bc, (cs, cs), (bs, bs)).to_numpy()
    cs_ = ia.opt_gemm(sctx, Ac, Bc, (cs, cs), (bs, bs)).to_numpy()
    rows = np.arange(M)
    hi, lo = O.dd_rows(A, B, rows)
    en = O.normwise_error(cn, hi, lo, rows)
    es = O.normwise_error(cs_, hi, lo, rows)
    assert es <= 1e-14, es
    assert es <= 4 * max(en, 1e-17), (es, en)


@pytest.mark.parametrize("fx", [f for f in GEMM if f[1] == "f8"], ids=lambda f: f[0])
def test_split_f64_exact_on_integer_fixtures(ia, fx):
    """The reference's arange fixtures: every product is an integer below 2^53, so the
    split form must reproduce it exactly."""
    name, dt, (xs, xc, xb), (ys, yc, yb), (zs, zc, zb) = fx
    ctx = _split_ctx(ia)
    X = ia.Container.arange(ctx, xs, np.float64, 0, 1, xc, xb)
    Y = ia.Container.arange(ctx, ys, np.float64, 0, 1, yc, yb)
    z = ia.matmul(ctx, X, Y, zc, zb).to_numpy()
    x, y = X.to_numpy(), Y.to_numpy()
    assert np.array_equal(z, O.dense_gemm(x, y))


def test_split_f64_zero_rows_and_signs(ia):
    rng = np.random.default_rng(3)
    A = _scaled(rng, (200, 300))
    A[5] = 0.0
    A[:, 7] = 0.0
    B = -_scaled(rng, (300, 150))
    B[:, 3] = 0.0
    ctx = _split_ctx(ia)
    C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (128, 128), (32, 32)),
                  ia.Container.from_numpy(ctx, B, (128, 128), (32, 32)), (128, 128), (32, 32)).to_numpy()
    hi, lo = O.dd_rows(A, B, np.arange(200))
    assert not C[5].any() and not C[:, 3].any()
    assert O.normwise_error(C, hi, lo, np.arange(200)) <= 1e-14


@pytest.mark.parametrize("nterms", [14, 15, 16])
def test_split_f64_more_moduli_is_at_least_as_accurate(ia, nterms):
    rng = np.random.default_rng(nterms)
    A, B = _scaled(rng, (256, 512)), _scaled(rng, (512, 256))
    ctx = ia.Context(form=ia.FORM_SPLIT, split_terms=nterms)
    C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (256, 256), (64, 64)),
                  ia.Container.from_numpy(ctx, B, (256, 256), (64, 64)), (256, 256), (64, 64)).to_numpy()
    hi, lo = O.dd_rows(A, B, np.arange(256))
    assert O.normwise_error(C, hi, lo, np.arange(256)) <= 2e-15


def _f32_inputs(rng, M, K, N):
    i, j = np.meshgrid(np.arange(M), np.arange(K), indexing="ij")
    A = rng.standard_normal((M, K)) + 0.1 * np.sin(0.003 * (i + j))
    i, j = np.meshgrid(np.arange(K), np.arange(N), indexing="ij")
    B = rng.standard_normal((K, N)) + 0.1 * np.sin(0.003 * (i + j))
    return A.astype(np.float32), B.astype(np.float32)


@pytest.mark.parametrize("M,K,N,cs,bs", [
    (300, 257, 200, 128, 32),        # ragged tiles and a K that is not a multiple of 64
    (256, 1024, 512, 256, 64),
    (1000, 1000, 1000, 500, 100),
    (64, 4096, 96, 64, 32),
])
def test_split_f32_bf16_error(ia, M, K, N, cs, bs):
    """float32 split forms on tcgen05 with FP32 accumulation in segments, against the
    float64 product of the same float32 operands.  Six products (three bf16 words per
    operand, the default): float32 accuracy, within 2x the FFMA path's error.  Three
    products (two words, 3xBF16): the split holds each operand to about 2^-17 relative,
    so the error sits near 4e-6 whatever the accumulation."""
    rng = np.random.default_rng(4 + M + K + N)
    A, B = _f32_inputs(rng, M, K, N)
    sctx, nctx = _split_ctx(ia), ia.Context()
    Ac = ia.Container.from_numpy(nctx, A, (cs, cs), (bs, bs))
    Bc = ia.Container.from_numpy(nctx, B, (cs, cs), (bs, bs))
    cn = ia.opt_gemm(nctx, Ac, Bc, (cs, cs), (bs, bs)).to_numpy()
    cs6 = ia.opt_gemm(sctx, Ac, Bc, (cs, cs), (bs, bs)).to_numpy()
    sctx.set_split_products_f32(3)
    cs3 = ia.opt_gemm(sctx, Ac, Bc, (cs, cs), (bs, bs)).to_numpy()
    exact = A.astype(np.float64) @ B.astype(np.float64)
    nrm = np.linalg.norm(exact)
    en = np.linalg.norm(cn - exact) / nrm
    e6 = np.linalg.norm(cs6 - exact) / nrm
    e3 = np.linalg.norm(cs3 - exact) / nrm
    assert e6 <= max(2 * en, 5e-7), (e6, en)
    assert e3 <= 8e-6, (e3, en)
    assert np.abs(cs6 - exact).max() <= 1e-5 * np.abs(exact).max()


def test_split_f32_zero_and_single_tile(ia):
    ctx = _split_ctx(ia)
    A = np.zeros((5, 7), np.float32)
    B = np.ones((7, 3), np.float32)
    Ac = ia.Container.from_numpy(ctx, A, (5, 7), (5, 7))
    Bc = ia.Container.from_numpy(ctx, B, (7, 3), (7, 3))
    assert not ia.opt_gemm(ctx, Ac, Bc, (5, 3), (5, 3)).to_numpy().any()
    A = np.full((5, 7), 0.5, np.float32)
    Ac = ia.Container.from_numpy(ctx, A, (5, 7), (5, 7))
    assert np.array_equal(ia.opt_gemm(ctx, Ac, Bc, (5, 3), (5, 3)).to_numpy(), np.full((5, 3), 3.5, np.float32))


def _classes(c):
    return np.isnan(c), np.isposinf(c), np.isneginf(c)


def _nonfinite_inputs(rng, dtype):
    A = _scaled(rng, (150, 230)).astype(dtype)
    B = _scaled(rng, (230, 170)).astype(dtype)
    A[3, 10] = np.nan
    A[7, 2] = np.inf
    A[9, 100] = -np.inf
    B[4, 5] = -np.inf
    B[50, 60] = np.nan
    return A, B


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_split_nonfinite_propagates_like_native(ia, dtype):
    """A NaN or an infinity in a row of A (column of B) reaches that row (column) of C with
    the same IEEE classes as the native product; every other output stays accurate."""
    rng = np.random.default_rng(11)
    A, B = _nonfinite_inputs(rng, dtype)
    ctx = _split_ctx(ia)
    C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (64, 64), (32, 32)),
                  ia.Container.from_numpy(ctx, B, (64, 64), (32, 32)), (64, 64), (32, 32)).to_numpy()
    with np.errstate(invalid="ignore", over="ignore"):
        ref = A @ B
    for got, want in zip(_classes(C), _classes(ref)):
        assert np.array_equal(got, want)
    rows = np.setdiff1d(np.arange(A.shape[0]), [3, 7, 9])
    cols = np.setdiff1d(np.arange(B.shape[1]), [5, 60])
    a, b = A[rows].astype(np.float64), B[:, cols].astype(np.float64)
    exact = a @ b
    err = np.linalg.norm(C[np.ix_(rows, cols)] - exact) / np.linalg.norm(exact)
    assert err <= (1e-14 if dtype == np.float64 else 5e-5), err


def test_split_f64_extreme_magnitudes(ia):
    """Rows and columns near the ends of the float64 range: the scaling takes their norms
    without overflow or underflow, so every block of C keeps the split form's accuracy."""
    rng = np.random.default_rng(12)
    A, B = _scaled(rng, (120, 300)), _scaled(rng, (300, 110))
    A[:20] *= 2.0 ** -600
    A[20:40] *= 2.0 ** 600
    B[:, :20] *= 2.0 ** -300
    B[:, 20:40] *= 2.0 ** 300
    ctx = _split_ctx(ia)
    C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (64, 64), (32, 32)),
                  ia.Container.from_numpy(ctx, B, (64, 64), (32, 32)), (64, 64), (32, 32)).to_numpy()
    rows = np.arange(A.shape[0])
    hi, lo = O.dd_rows(A, B, rows)
    for rs in (slice(0, 20), slice(20, 40), slice(40, 120)):
        for cs in (slice(0, 20), slice(20, 40), slice(40, 110)):
            h, l, c = hi[rs, cs], lo[rs, cs], C[rs, cs]
            scale = np.abs(h).max()
            d = ((c - h) - l) / scale
            assert np.all(np.isfinite(c))
            assert np.linalg.norm(d) <= 1e-14 * np.linalg.norm(h / scale), (rs, cs)


def test_split_f64_fewer_moduli(ia):
    """8 and 10 moduli (two 40-bit reconstruction chunks) stay exact on small integers and
    lose accuracy only as the smaller product of moduli dictates."""
    rng = np.random.default_rng(13)
    A, B = _scaled(rng, (96, 512)), _scaled(rng, (512, 80))
    hi, lo = O.dd_rows(A, B, np.arange(96))
    errs = []
    for nterms in (8, 10, 12, 14):
        ctx = ia.Context(form=ia.FORM_SPLIT, split_terms=nterms)
        C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (64, 64), (32, 32)),
                      ia.Container.from_numpy(ctx, B, (64, 64), (32, 32)), (64, 64), (32, 32)).to_numpy()
        errs.append(O.normwise_error(C, hi, lo, np.arange(96)))
    assert errs[0] <= 1e-6 and errs[-1] <= 1e-14, errs
    assert all(errs[i + 1] <= errs[i] for i in range(len(errs) - 1)), errs
    X = np.arange(48 * 64, dtype=np.float64).reshape(48, 64) % 17
    Y = np.arange(64 * 40, dtype=np.float64).reshape(64, 40) % 13
    ctx = ia.Context(form=ia.FORM_SPLIT, split_terms=8)
    Z = ia.matmul(ctx, ia.Container.from_numpy(ctx, X, (32, 32), (16, 16)),
                  ia.Container.from_numpy(ctx, Y, (32, 32), (16, 16)), (32, 32), (16, 16)).to_numpy()
    assert np.array_equal(Z, X @ Y)


@pytest.mark.parametrize("M,K,N", [(3000, 900, 700), (5000, 520, 1100), (8192, 256, 384)])
def test_split_f64_row_slices_equal_whole(ia, M, K, N):
    """Each row of C depends only on its row of A and on B: the row scaling, the residues, the
    INT8 sums and the reconstruction do not see the other rows.  So the product computed in
    slices of at most 1000 rows (as the pipelined call computes its bands of C) is bitwise the
    whole product, NaN and infinity rows included."""
    import ctypes
    import torch
    rng = np.random.default_rng(M + K)
    a, b = _scaled(rng, (M, K)), _scaled(rng, (K, N))
    a[M // 3, 5] = np.nan
    a[M - 1, K - 1] = np.inf
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    C1 = torch.empty((M, N), dtype=torch.float64, device="cuda")
    C2 = torch.empty((M, N), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx = _split_ctx(ia)

    def gemm(m, r0, C):
        ia.check(ia.lib().iarray_b200_dense_gemm(
            ctx.ptr, ia.DTYPE_DOUBLE, m, N, K, ctypes.c_void_p(A.data_ptr() + r0 * K * 8), K,
            ctypes.c_void_p(B.data_ptr()), N, ctypes.c_void_p(C.data_ptr() + r0 * N * 8), N), "dense_gemm")

    gemm(M, 0, C1)
    for r0 in range(0, M, 1000):
        gemm(min(1000, M - r0), r0, C2)
    ctx.synchronize()
    c1, c2 = C1.cpu().numpy(), C2.cpu().numpy()
    assert c1.tobytes() == c2.tobytes()
    assert np.isnan(c1[M // 3]).all() and not np.isfinite(c1[M - 1]).any()
    rows = np.array([0, 1, M // 2, M - 2])
    hi, lo = O.dd_rows(a, b, rows)
    d = (c1[rows] - hi) - lo
    assert np.linalg.norm(d) <= 1e-14 * np.linalg.norm(hi)


@pytest.mark.parametrize("M,K,N,ch,bl", [
    (300, 200, 260, (100, 120), (40, 40)),     # array and chunk padding (chunk 120 = 3 blocks of 40)
    (512, 300, 512, (256, 256), (64, 64)),     # no padding
    (130, 70, 100, (64, 52), (32, 20)),        # blocks wider than the chunk's last columns
    (100, 50, 90, (50, 30), (25, 10)),         # chunk columns not a multiple of 4: dense C, then gather
])
@pytest.mark.parametrize("encoder", ["parallel", "liblz4"])
def test_split_f64_output_written_into_encoder_image(ia, M, K, N, ch, bl, encoder):
    """The split form writes C's reconstruction straight into the encoder's shuffled block image
    (no dense C, no gather).  C's chunks must be byte for byte those of the same values encoded
    from a dense array, its values those of the dense split product; rows and columns with NaN or
    infinity go through the non-finite fix into the same image."""
    import ctypes
    import torch
    rng = np.random.default_rng(M * N + K)
    a, b = _scaled(rng, (M, K)), _scaled(rng, (K, N))
    a[M // 2, 3] = np.nan
    b[K - 1, N // 3] = np.inf
    enc = ia.ENCODER_LIBLZ4 if encoder == "liblz4" else ia.ENCODER_PARALLEL
    ctx = ia.Context(form=ia.FORM_SPLIT, encoder=enc)
    Ac = ia.Container.from_numpy(ctx, a, ch, bl)
    Bc = ia.Container.from_numpy(ctx, b, (ch[1], ch[1]), (bl[1], bl[1]))
    C = ia.matmul(ctx, Ac, Bc, ch, bl)
    got = C.to_numpy()
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    D = torch.empty((M, N), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ia.check(ia.lib().iarray_b200_dense_gemm(ctx.ptr, ia.DTYPE_DOUBLE, M, N, K, ctypes.c_void_p(A.data_ptr()), K,
                                              ctypes.c_void_p(B.data_ptr()), N, ctypes.c_void_p(D.data_ptr()), N),
             "dense_gemm")
    ctx.synchronize()
    dense = D.cpu().numpy()
    assert got.tobytes() == dense.tobytes()
    assert np.isnan(got[M // 2]).all() and not np.isfinite(got[:, N // 3]).any()
    ref = ia.Container.from_numpy(ctx, dense, ch, bl)
    assert C.chunks() == ref.chunks()
    ctx.close()


@pytest.mark.parametrize("M,K,N,ch,bl", [
    (512, 300, 768, (256, 256), (64, 128)),
    (1024, 200, 512, (512, 512), (128, 256)),
    (300, 200, 260, (100, 120), (40, 40)),     # chunk and array padding
])
def test_split_f32_output_chunks_equal_dense_encode(ia, M, K, N, ch, bl):
    """float32 split form through iarray_linalg_matmul: C's values are bitwise those of the dense
    split product on device operands and its chunks byte for byte those of that product encoded
    from an array, NaN and infinity rows and columns included."""
    import ctypes
    import torch
    rng = np.random.default_rng(M + N + K)
    a = rng.standard_normal((M, K)).astype(np.float32)
    b = rng.standard_normal((K, N)).astype(np.float32)
    a[M // 2, 3] = np.nan
    b[K - 1, N // 3] = np.inf
    ctx = ia.Context(form=ia.FORM_SPLIT, encoder=ia.ENCODER_PARALLEL)
    Ac = ia.Container.from_numpy(ctx, a, ch, bl)
    Bc = ia.Container.from_numpy(ctx, b, (100, ch[1]), (50, bl[1]))
    C = ia.matmul(ctx, Ac, Bc, ch, bl)
    got = C.to_numpy()
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    D = torch.empty((M, N), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ia.check(ia.lib().iarray_b200_dense_gemm(ctx.ptr, ia.DTYPE_FLOAT, M, N, K, ctypes.c_void_p(A.data_ptr()), K,
                                              ctypes.c_void_p(B.data_ptr()), N, ctypes.c_void_p(D.data_ptr()), N),
             "dense_gemm")
    ctx.synchronize()
    dense = D.cpu().numpy()
    assert got.tobytes() == dense.tobytes()
    assert np.isnan(got[M // 2]).all() and not np.isfinite(got[:, N // 3]).any()
    ref = ia.Container.from_numpy(ctx, dense, ch, bl)
    assert C.chunks() == ref.chunks()
    ctx.close()
