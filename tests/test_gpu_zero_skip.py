"""Zero-block skipping of the block-pair products, through the C ABI.

The reference skips a K-block pair when either block is a zero block (every stream of the
block has csize 0) or, depending on the entry point, either chunk is a special-zero chunk
(src/linalg/iarray_gemm.c:17-77, :146-168, :206-211; iarray_gemm_a.c / iarray_gemm_b.c,
iarray_gemv.c).  A skipped pair contributes nothing, so a NaN or an infinity facing a zero
block does not reach C.  Integer-valued operands make every sum exact, so the GPU result
must equal the oracle's restatement of the loop bit for bit (NaN positions included).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _ints(rng, shape, dtype):
    return rng.integers(-8, 9, shape).astype(dtype)


def _zero_blocks(x, block, frac, rng):
    """Zero a fraction of the block grid of x (blocks aligned to `block` from the origin,
    which matches the Caterva blocks when the chunk shape is a multiple of the block)."""
    rb, cb = -(-x.shape[0] // block[0]), -(-x.shape[1] // block[1])
    mask = rng.random((rb, cb)) < frac
    for i, j in zip(*np.nonzero(mask)):
        x[i * block[0]:(i + 1) * block[0], j * block[1]:(j + 1) * block[1]] = 0
    return mask


def _special_zero_chunk(nbytes, blocksize, typesize):
    z = bytearray(32)
    z[0], z[1], z[2], z[3] = 5, 1, 0x25, typesize
    z[4:8] = nbytes.to_bytes(4, "little")
    z[8:12] = blocksize.to_bytes(4, "little")
    z[12:16] = (32).to_bytes(4, "little")
    z[31] = 1 << 4
    return bytes(z)


def _assert_same(got, ref):
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("form", ["native", "split"])
def test_zero_blocks_keep_nan_out(ia, dtype, form):
    rng = np.random.default_rng(21)
    M, K, N, ch, bl = 150, 130, 110, (64, 64), (16, 16)
    A, B = _ints(rng, (M, K), dtype), _ints(rng, (K, N), dtype)
    _zero_blocks(A, bl, 0.3, rng)
    _zero_blocks(B, bl, 0.3, rng)
    # NaN and infinities: some facing zero blocks of the other operand (kept out of C by the
    # skip), some facing non-zero blocks (they propagate)
    for _ in range(12):
        i, k = rng.integers(0, M), rng.integers(0, K)
        A[i, k] = [np.nan, np.inf, -np.inf][rng.integers(0, 3)]
        k2, j = rng.integers(0, K), rng.integers(0, N)
        B[k2, j] = [np.nan, np.inf, -np.inf][rng.integers(0, 3)]
    ctx = ia.Context()
    if form == "split":
        ctx.set_form(ia.FORM_SPLIT)
    Ac = ia.Container.from_numpy(ctx, A, ch, bl)
    Bc = ia.Container.from_numpy(ctx, B, ch, bl)
    got = ia.opt_gemm(ctx, Ac, Bc, ch, bl).to_numpy()
    ga, ach = O.encode_array(A, ch, bl)
    gb, bch = O.encode_array(B, ch, bl)
    dt = O.DTYPE_DOUBLE if dtype == np.float64 else O.DTYPE_FLOAT
    ref = O.opt_gemm(ga, ach, gb, bch, O.Geom((M, N), ch, bl, A.itemsize), dt)
    _assert_same(got, ref)
    # the dense product would have put NaN where the reference skipped
    with np.errstate(invalid="ignore"):
        dense = A.astype(np.float64) @ B.astype(np.float64)
    assert np.isnan(dense).sum() > np.isnan(ref).sum()


@pytest.mark.parametrize("entry,rule", [("opt_gemm", 3), ("opt_gemm_a", 2), ("opt_gemm_b", 1)])
def test_special_zero_chunks_per_entry_point(ia, entry, rule):
    """A special-zero chunk is skipped by iarray_opt_gemm for both operands, by
    iarray_opt_gemm_a only for B and by iarray_opt_gemm_b only for A."""
    rng = np.random.default_rng(22)
    M, K, N = 96, 80, 72
    if entry == "opt_gemm":
        ca, ba, cb, bb, cc, bc = (32, 40), (16, 20), (40, 24), (20, 12), (32, 24), (16, 12)
    elif entry == "opt_gemm_a":                      # A chunks span K; A block rows = its chunk rows
        ca, ba, cb, bb, cc, bc = (32, 80), (32, 20), (80, 24), (20, 24), (32, 72), (32, 24)
    else:                                            # mirrored for iarray_opt_gemm_b
        ca, ba, cb, bb, cc, bc = (32, 80), (32, 20), (80, 24), (20, 24), (96, 24), (32, 24)
    A, B = _ints(rng, (M, K), np.float64), _ints(rng, (K, N), np.float64)
    ga = O.Geom((M, K), ca, ba, 8)
    gb = O.Geom((K, N), cb, bb, 8)
    # chunk 1 of A and chunk 0 of B will be special-zero chunks: put NaN in B's rows facing
    # A's chunk 1 and infinities in A's columns facing B's chunk 0
    kc = 1 % ga.cgrid[1]
    k0, k1 = kc * ca[1], min((kc + 1) * ca[1], K)
    B[k0:k1] = np.where(rng.random((k1 - k0, N)) < 0.05, np.nan, B[k0:k1])
    A[:, :cb[0]] = np.where(rng.random((M, min(cb[0], K))) < 0.05, np.inf, A[:, :cb[0]])
    ga, ach = O.encode_array(A, ca, ba)
    gb, bch = O.encode_array(B, cb, bb)
    ach[1] = _special_zero_chunk(ga.chunk_nbytes, ba[0] * ba[1] * 8, 8)
    bch[0] = _special_zero_chunk(gb.chunk_nbytes, bb[0] * bb[1] * 8, 8)
    ctx = ia.Context()
    Ac = ia.Container.from_chunks(ctx, (M, K), np.float64, ca, ba, ach)
    Bc = ia.Container.from_chunks(ctx, (K, N), np.float64, cb, bb, bch)
    got = getattr(ia, entry)(ctx, Ac, Bc, cc, bc).to_numpy()
    # the oracle's loop writes C partitioned like the operands' pairs; the logical result
    # does not depend on C's partition
    ref = O.opt_gemm(ga, ach, gb, bch, O.Geom((M, N), (ca[0], cb[1]), (ba[0], bb[1]), 8), O.DTYPE_DOUBLE,
                     chunk_rule=rule)
    _assert_same(got, ref)
    assert np.isnan(ref).any()


def test_opt_gemv_zero_blocks(ia):
    rng = np.random.default_rng(23)
    M, K, ch, bl = 300, 260, (100, 80), (25, 20)
    A = _ints(rng, (M, K), np.float64)
    _zero_blocks(A, bl, 0.4, rng)
    x = _ints(rng, (K,), np.float64)
    x[:20] = 0                                       # the first x block is a zero block
    A[5, 3] = np.nan                                 # faces x's zero block: skipped
    A[7, 100] = np.inf
    x[45] = np.nan                                   # propagates unless A's block is zero
    ctx = ia.Context()
    Ac = ia.Container.from_numpy(ctx, A, ch, bl)
    xc = ia.Container.from_numpy(ctx, x, (ch[1],), (bl[1],))
    got = ia.opt_gemv(ctx, Ac, xc, (ch[0],), (bl[0],)).to_numpy()
    ga, ach = O.encode_array(A, ch, bl)
    gx, xch = O.encode_array(x, (ch[1],), (bl[1],))
    ref = O.opt_gemv(ga, ach, gx, xch, O.Geom((M,), (ch[0],), (bl[0],), 8), O.DTYPE_DOUBLE)
    _assert_same(got, ref)


@pytest.mark.parametrize("form", ["native", "split"])
def test_sparse_blocks_product_matches_dense(ia, form):
    """90% of the blocks of A and half of B's are zero: most tiles skip most of their
    k-tiles and some skip all of them; the result still equals the dense product."""
    rng = np.random.default_rng(24)
    n, ch, bl = 1024, (512, 512), (128, 128)
    A = rng.uniform(-1, 1, (n, n))
    B = rng.uniform(-1, 1, (n, n))
    _zero_blocks(A, bl, 0.9, rng)
    _zero_blocks(B, bl, 0.5, rng)
    ctx = ia.Context()
    if form == "split":
        ctx.set_form(ia.FORM_SPLIT)
    Ac = ia.Container.from_numpy(ctx, A, ch, bl)
    Bc = ia.Container.from_numpy(ctx, B, ch, bl)
    got = ia.opt_gemm(ctx, Ac, Bc, ch, bl).to_numpy()
    ref = A @ B
    nrm = np.linalg.norm(ref)
    assert np.linalg.norm(got - ref) <= 1e-14 * nrm
    # row bands whose A blocks are all zero come out exactly zero
    zero_rows = [i for i in range(0, n, bl[0]) if not A[i:i + bl[0]].any()]
    for i in zero_rows:
        assert not got[i:i + bl[0]].any()
