"""The benchmark configurations asserted at their stated sizes, through the C ABI.

- precision float64: A, B 8192 x 8192, entries uniform(-1, 1) x 2^U{-8..8} (default_rng(3),
  A then B), chunk 2048^2, block 256^2.  The split form's normwise error against the
  double-double oracle on 256 sampled rows (default_rng(99)) is at most 4x the native FP64
  form's, and both stay below 1e-14.
- plain GEMV: float32 A 20000 x 20000 with A[i, j] = sin(0.001 i) + cos(0.002 j), x
  uniform(-1, 1) (default_rng(2)), chunk 4000^2, block 500^2: iarray_opt_gemv against the
  float64 product of the same float32 operands.
- precision float32: A 16384 x 4096, B 4096 x 16384, normal(0, 1) (default_rng(4)) plus
  0.1 sin(0.003 (i + j)), chunk 4096^2, block 512^2: both split forms (3 and 6 BF16
  products) and the native FFMA form against the float64 product on 256 sampled rows.
- batching: the first 64 problems of the 512-problem batch (m, n, k uniform in [64, 2048],
  default_rng(5), chunk 512^2, block 128^2), both forms, byte-identical to single products.

Inputs are seeded synthetic matrices with the configurations' shapes and distributions.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def test_precision_f64_8192(ia):
    n, ch, bl = 8192, (2048, 2048), (256, 256)
    rng = np.random.default_rng(3)
    A = rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n)))
    B = rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n)))
    rows = np.sort(np.random.default_rng(99).choice(n, 256, replace=False))
    hi, lo = O.dd_rows(A, B, rows)
    ctx = ia.Context(encoder=ia.ENCODER_PARALLEL)
    Ac = ia.Container.from_numpy(ctx, A, ch, bl)
    Bc = ia.Container.from_numpy(ctx, B, ch, bl)
    errs = {}
    for name, form in (("native", ia.FORM_NATIVE), ("split", ia.FORM_SPLIT)):
        ctx.set_form(form)
        C = ia.opt_gemm(ctx, Ac, Bc, ch, bl)
        errs[name] = O.normwise_error(C.to_numpy(), hi, lo, rows)
        C.free()
    assert errs["native"] <= 1e-14, errs
    assert errs["split"] <= 1e-14, errs
    assert errs["split"] <= 4 * errs["native"], errs
    Ac.free()
    Bc.free()
    ctx.close()


def test_plain_gemv_f32_20000(ia):
    n, ch, bl = 20000, 4000, 500
    A = np.empty((n, n), np.float32)
    cj = np.cos(0.002 * np.arange(n))
    for r0 in range(0, n, 2000):
        A[r0:r0 + 2000] = (np.sin(0.001 * np.arange(r0, r0 + 2000))[:, None] + cj[None, :]).astype(np.float32)
    x = np.random.default_rng(2).uniform(-1, 1, n).astype(np.float32)
    ref = np.empty(n)
    x64 = x.astype(np.float64)
    for r0 in range(0, n, 2000):
        ref[r0:r0 + 2000] = A[r0:r0 + 2000].astype(np.float64) @ x64
    ctx = ia.Context()
    Ac = ia.Container.from_numpy(ctx, A, (ch, ch), (bl, bl))
    xc = ia.Container.from_numpy(ctx, x, (ch,), (bl,))
    del A
    y = ia.opt_gemv(ctx, Ac, xc, (ch,), (bl,))
    got = y.to_numpy().astype(np.float64)
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    # float32 accumulation over K = 20000: the reference's own bar is 1e-5 relative
    assert err <= 1e-5, err
    # the matmul entry point (panel GEMV) agrees with the block-pair one
    y2 = ia.matmul(ctx, Ac, xc, (ch,), (bl,)).to_numpy().astype(np.float64)
    assert float(np.linalg.norm(y2 - ref) / np.linalg.norm(ref)) <= 1e-5
    for c in (y, Ac, xc):
        c.free()
    ctx.close()


def _f32_config4():
    M, K, N = 16384, 4096, 16384
    rng = np.random.default_rng(4)
    A = rng.standard_normal((M, K))
    A += 0.1 * np.sin(0.003 * (np.arange(M)[:, None] + np.arange(K)[None, :]))
    A = A.astype(np.float32)
    B = rng.standard_normal((K, N))
    B += 0.1 * np.sin(0.003 * (np.arange(K)[:, None] + np.arange(N)[None, :]))
    return A, B.astype(np.float32)


def test_precision_f32_16384x4096x16384(ia):
    A, B = _f32_config4()
    ch, bl = (4096, 4096), (512, 512)
    rows = np.sort(np.random.default_rng(99).choice(A.shape[0], 256, replace=False))
    exact = A[rows].astype(np.float64) @ B.astype(np.float64)
    nrm = np.linalg.norm(exact)
    ctx = ia.Context(encoder=ia.ENCODER_PARALLEL)
    Ac = ia.Container.from_numpy(ctx, A, ch, bl)
    Bc = ia.Container.from_numpy(ctx, B, ch, bl)
    del A, B
    errs = {}
    for name, form, terms in (("native", ia.FORM_NATIVE, 0), ("split6", ia.FORM_SPLIT, 6),
                              ("split3", ia.FORM_SPLIT, 3)):
        ctx.set_form(form)
        if terms:
            ctx.set_split_products_f32(terms)
        C = ia.opt_gemm(ctx, Ac, Bc, ch, bl)
        c = C.to_numpy()[rows].astype(np.float64)
        C.free()
        errs[name] = float(np.linalg.norm(c - exact) / nrm)
    # native FFMA: float32 rounding of the sums
    assert errs["native"] <= 3e-6, errs
    # three-word split, six products, FP32 accumulation in segments: float32 accuracy
    assert errs["split6"] <= 2.5e-6 and errs["split6"] <= 2 * errs["native"], errs
    # two-word split, three products: the split itself holds each operand to about 2^-17,
    # which bounds the error near 4.3e-6 at these sizes even with exact sums
    assert errs["split3"] <= 8e-6, errs
    for c in (Ac, Bc):
        c.free()
    ctx.close()


def _batch_config5(ia, ctx, count):
    rng = np.random.default_rng(5)
    dims = rng.integers(64, 2049, (512, 3))
    As, Bs = [], []
    for m, n, k in dims[:count]:
        As.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (int(m), int(k))), (512, 512), (128, 128)))
        Bs.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (int(k), int(n))), (512, 512), (128, 128)))
    return As, Bs


@pytest.mark.parametrize("form", ["native", "split"])
def test_batching_config_slice_matches_single_products(ia, form):
    ctx = ia.Context(encoder=ia.ENCODER_PARALLEL)
    if form == "split":
        ctx.set_form(ia.FORM_SPLIT, 14)      # the single products' moduli count: byte-identical results
    As, Bs = _batch_config5(ia, ctx, 64)
    cs, bs = [(512, 512)] * len(As), [(128, 128)] * len(As)
    batch = ia.Batch(ctx, As, Bs, cs, bs)
    for rep in range(2):
        outs = batch.run()
        for i, c in enumerate(outs):
            # partitions follow iarray_opt_gemm's rules (chunks may exceed a small shape)
            ref = ia.opt_gemm(ctx, As[i], Bs[i], cs[i], bs[i])
            assert c.chunks() == ref.chunks(), (rep, i)
            ref.free()
            c.free()
    batch.free()
    for c in As + Bs:
        c.free()
    ctx.close()
