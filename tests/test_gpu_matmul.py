"""GPU parity of the matmul entry points (through the C ABI) against the oracle, on the
reference's own test fixtures and on random data.

Tolerances: the reference tests compare elementwise |z - o| / z against MKL with
1e-14 (float64) / 1e-5 (float32) (tests/test_linalg_gemm.c:128-147).  Here `o` is the
oracle's k-ascending product of the same decoded operands.  For random float64 data,
where block order legitimately changes the last bits, the bar is normwise:
||C - C_oracle||_F / ||C_oracle||_F <= 1e-14.
"""
import numpy as np
import pytest

import oracle as O
from ref_fixtures import GEMM, GEMM_T, GEMV, GEMV_T, OPT_GEMV, TOL

pytestmark = pytest.mark.gpu


def _exact(x, y):
    """The product of the decoded operands in float64 (exact for the integer fixtures);
    float32 results are judged against it, as the reference judges iarray against MKL."""
    return O.dense_gemm(x.astype(np.float64), y.astype(np.float64))


def _rel_ok(z, o, tol):
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs((z.astype(np.float64) - o.astype(np.float64)) / z.astype(np.float64))
    r[(z == 0) & (o == 0)] = 0
    return float(np.nanmax(r)) <= tol, float(np.nanmax(r))


def _arange(shape, dtype):
    return np.arange(int(np.prod(shape)), dtype=np.float64).astype(dtype).reshape(shape)


def _linspace(shape, dtype):
    n = int(np.prod(shape))
    return (np.arange(n, dtype=np.float64) * (10.0 / (n - 1))).astype(dtype).reshape(shape)


@pytest.mark.parametrize("fx", GEMM, ids=[f[0] for f in GEMM])
def test_linalg_matmul_reference_fixtures(ctx, ia, fx):
    name, dt, (xs, xc, xb), (ys, yc, yb), (zs, zc, zb) = fx
    dtype = np.dtype(dt)
    X = ia.Container.arange(ctx, xs, dtype, 0, 1, xc, xb)
    Y = ia.Container.arange(ctx, ys, dtype, 0, 1, yc, yb)
    x, y = X.to_numpy(), Y.to_numpy()
    assert np.array_equal(x, _arange(xs, dtype)) and np.array_equal(y, _arange(ys, dtype))
    Z = ia.matmul(ctx, X, Y, zc, zb)
    z = Z.to_numpy()
    o = _exact(x, y)
    ok, worst = _rel_ok(z, o, TOL[dt])
    assert ok, worst
    if dt == "f8":                        # integer products below 2^53: exact in any order
        assert np.array_equal(z, o)


@pytest.mark.parametrize("fx", GEMM_T, ids=[f[0] for f in GEMM_T])
def test_linalg_matmul_transposed_fixtures(ctx, ia, fx):
    name, dt, (xs, xc, xb), (ys, yc, yb), (zs, zc, zb) = fx
    dtype = np.dtype(dt)
    X = ia.Container.arange(ctx, xs, dtype, 0, 1, xc, xb)
    Y = ia.Container.arange(ctx, ys, dtype, 0, 1, yc, yb)
    Xt, Yt = X.transpose(), Y.transpose()
    assert Xt.shape == (xs[1], xs[0])
    x, y = Xt.to_numpy(), Yt.to_numpy()
    assert np.array_equal(x, _arange(xs, dtype).T)
    z = ia.matmul(ctx, Xt, Yt, zc, zb).to_numpy()
    ok, worst = _rel_ok(z, _exact(x, y), TOL[dt])
    assert ok, worst


@pytest.mark.parametrize("fx", GEMV + GEMV_T, ids=[f[0] + ("_T" if f in GEMV_T else "") for f in GEMV + GEMV_T])
def test_linalg_matmul_gemv_reference_fixtures(ctx, ia, fx):
    name, dt, (xs, xc, xb), (ys, yc, yb), (zs, zc, zb) = fx
    dtype = np.dtype(dt)
    X = ia.Container.linspace(ctx, xs, dtype, 0, 10, xc, xb)
    if fx in GEMV_T:
        X = X.transpose()
    Y = ia.Container.linspace(ctx, ys, dtype, 0, 10, yc, yb)
    x, y = X.to_numpy(), Y.to_numpy()
    np.testing.assert_allclose(y, _linspace(ys, dtype), rtol=1e-6)
    z = ia.matmul(ctx, X, Y, zc, zb).to_numpy()
    assert z.shape == (x.shape[0],)
    ok, worst = _rel_ok(z, _exact(x, y), TOL[dt])
    assert ok, worst


@pytest.mark.parametrize("fx", OPT_GEMV, ids=[f[0] for f in OPT_GEMV])
def test_opt_gemv_reference_fixtures(ctx, ia, fx):
    name, dt, (xs, xc, xb), (ys, yc, yb), (zs, zc, zb) = fx
    dtype = np.dtype(dt)
    X = ia.Container.linspace(ctx, xs, dtype, 0, 10, xc, xb)
    Y = ia.Container.linspace(ctx, ys, dtype, 0, 10, yc, yb)
    z = ia.opt_gemv(ctx, X, Y, zc, zb).to_numpy()
    x, y = X.to_numpy(), Y.to_numpy()
    ok, worst = _rel_ok(z, _exact(x, y), TOL[dt])
    assert ok, worst


def _rand(rng, shape, dtype, scaled=False):
    a = rng.uniform(-1, 1, shape)
    if scaled:
        a = a * 2.0 ** rng.integers(-8, 9, shape)
    return a.astype(dtype)


@pytest.mark.parametrize("M,K,N,cs,bs", [
    (1000, 1000, 1000, 500, 100),           # the plain drop-in configuration's partition
    (333, 257, 129, 128, 32),
    (64, 2048, 96, 64, 32),
])
def test_opt_gemm_matches_oracle_blockpair(ctx, ia, M, K, N, cs, bs):
    rng = np.random.default_rng(7)
    A, B = _rand(rng, (M, K), np.float64, True), _rand(rng, (K, N), np.float64, True)
    Ac = ia.Container.from_numpy(ctx, A, (cs, cs), (bs, bs))
    Bc = ia.Container.from_numpy(ctx, B, (cs, cs), (bs, bs))
    C = ia.opt_gemm(ctx, Ac, Bc, (cs, cs), (bs, bs)).to_numpy()
    ga, ach = O.encode_array(A, (cs, cs), (bs, bs))
    gb, bch = O.encode_array(B, (cs, cs), (bs, bs))
    ref = O.opt_gemm(ga, ach, gb, bch, O.Geom((M, N), (cs, cs), (bs, bs), 8), O.DTYPE_DOUBLE)
    err = np.linalg.norm(C - ref) / np.linalg.norm(ref)
    assert err <= 1e-14, err


def test_matmul_float32_random_matches_oracle(ctx, ia):
    rng = np.random.default_rng(8)
    A, B = _rand(rng, (700, 513), np.float32), _rand(rng, (513, 301), np.float32)
    Ac = ia.Container.from_numpy(ctx, A, (256, 256), (64, 64))
    Bc = ia.Container.from_numpy(ctx, B, (256, 128), (64, 32))
    C = ia.matmul(ctx, Ac, Bc, (256, 128), (64, 32)).to_numpy()
    ref = A.astype(np.float64) @ B.astype(np.float64)
    err = np.linalg.norm(C - ref) / np.linalg.norm(ref)
    assert err <= 1e-6, err


def test_matmul_output_chunks_are_valid_blosc2(ctx, ia):
    """The result's chunks decode with the oracle (the reference's decoder restated)
    to exactly what the library returns, and re-encode byte-identically."""
    rng = np.random.default_rng(9)
    A, B = _rand(rng, (300, 400), np.float64), _rand(rng, (400, 200), np.float64)
    C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (128, 128), (32, 32)),
                  ia.Container.from_numpy(ctx, B, (128, 128), (32, 32)), (100, 64), (25, 32))
    c = C.to_numpy()
    g = O.Geom((300, 200), (100, 64), (25, 32), 8)
    chunks = C.chunks()
    assert np.array_equal(O.decode_array(g, chunks, np.float64), c)
    _, ref = O.encode_array(c, (100, 64), (25, 32))
    assert chunks == ref


def test_opt_gemm_a_and_b_partitions(ctx, ia):
    rng = np.random.default_rng(10)
    M, K, N = 256, 200, 96
    A, B = _rand(rng, (M, K), np.float64), _rand(rng, (K, N), np.float64)
    # iarray_opt_gemm_a: A chunk = one block row x all K; B chunk = all K x one block col
    Aa = ia.Container.from_numpy(ctx, A, (64, 200), (64, 50))
    Ba = ia.Container.from_numpy(ctx, B, (200, 32), (50, 32))
    Ca = ia.opt_gemm_a(ctx, Aa, Ba, (64, 96), (64, 32)).to_numpy()
    ref = O.dense_gemm(A, B)
    assert np.linalg.norm(Ca - ref) / np.linalg.norm(ref) <= 1e-14
    Cb = ia.opt_gemm_b(ctx, Aa, Ba, (256, 32), (64, 32)).to_numpy()
    assert np.linalg.norm(Cb - ref) / np.linalg.norm(ref) <= 1e-14


def test_partition_and_shape_errors(ctx, ia):
    rng = np.random.default_rng(11)
    A = ia.Container.from_numpy(ctx, _rand(rng, (64, 64), np.float64), (32, 32), (16, 16))
    B = ia.Container.from_numpy(ctx, _rand(rng, (64, 64), np.float64), (32, 16), (16, 16))
    B32 = ia.Container.from_numpy(ctx, _rand(rng, (64, 64), np.float32), (32, 32), (16, 16))
    Bs = ia.Container.from_numpy(ctx, _rand(rng, (48, 64), np.float64), (32, 32), (16, 16))
    cases = [
        (lambda: ia.opt_gemm(ctx, A, B, (32, 32), (16, 16)), "INVALID_CHUNKSHAPE"),
        (lambda: ia.opt_gemm(ctx, A, A, (32, 32), (8, 16)), "INVALID_BLOCKSHAPE"),
        (lambda: ia.matmul(ctx, A, B32, (32, 32), (16, 16)), "INVALID_DTYPE"),
        (lambda: ia.matmul(ctx, A, Bs, (32, 32), (16, 16)), "INVALID_SHAPE"),
        (lambda: ia.matmul(ctx, A, A, (128, 32), (16, 16)), "INVALID_CHUNKSHAPE"),
    ]
    for fn, name in cases:
        with pytest.raises(ia.IArrayError) as e:
            fn()
        assert e.value.name == name


def test_matmul_persists_output_when_urlpath_given(ctx, ia, tmp_path):
    rng = np.random.default_rng(12)
    A, B = _rand(rng, (100, 80), np.float64), _rand(rng, (80, 60), np.float64)
    p = str(tmp_path / "c.iarray")
    C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (50, 40), (25, 20)),
                  ia.Container.from_numpy(ctx, B, (40, 30), (20, 15)), (50, 30), (25, 15), urlpath=p)
    assert np.array_equal(ia.Container.open(ctx, p).to_numpy(), C.to_numpy())


@pytest.mark.parametrize("form", ["native", "split"])
@pytest.mark.parametrize("K", [33, 1, 129])
def test_dense_f64_reads_nothing_past_k(ctx, ia, K, form):
    """Dense operands have rows padded past K (leading dimension a multiple of 32) and
    nothing writes the padding.  NaN planted there must not reach C: every product reads
    only the K columns of A (and the K rows of B)."""
    import ctypes
    import torch
    M, N = 100, 50
    lda, ldb, ldc = (K + 31) // 32 * 32, 64, 64
    rng = np.random.default_rng(K)
    a = rng.integers(-8, 9, (M, K)).astype(np.float64)
    b = rng.integers(-8, 9, (K, N)).astype(np.float64)
    A = torch.full((M, lda), float("nan"), dtype=torch.float64, device="cuda")
    B = torch.full((K + 3, ldb), float("nan"), dtype=torch.float64, device="cuda")
    A[:, :K] = torch.from_numpy(a).cuda()
    B[:K, :N] = torch.from_numpy(b).cuda()
    C = torch.zeros((M, ldc), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()          # the library's stream does not wait for torch's
    c = ia.Context(form=ia.FORM_SPLIT if form == "split" else ia.FORM_NATIVE)
    ia.check(ia.lib().iarray_b200_dense_gemm(c.ptr, ia.DTYPE_DOUBLE, M, N, K, ctypes.c_void_p(A.data_ptr()), lda,
                                              ctypes.c_void_p(B.data_ptr()), ldb, ctypes.c_void_p(C.data_ptr()), ldc),
             "dense_gemm")
    c.synchronize()
    assert np.array_equal(C[:, :N].cpu().numpy(), a @ b)
