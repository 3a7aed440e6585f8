"""The decode-fused GEMV (y = A x with A's items taken from its chunks straight into the row
sums, the dense A never written), through the C ABI.

Integer-valued operands make every sum exact, so the result must equal the oracle's restatement
of the reference's loops (src/linalg/iarray_gemv.c:88-246 for iarray_opt_gemv,
src/linalg/matmul/gemv.c:71-190 for the panel GEMV) bit for bit, whatever the partition: edge
blocks, chunk padding, unshuffled and memcpyed chunks, special-value chunks.  The sums run in a
fixed order, so repeated calls give the same bytes on any inputs.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _ints(rng, shape, dtype):
    return rng.integers(-8, 9, shape).astype(dtype)


def _special_chunk(nbytes, blocksize, typesize, kind, value=None):
    """A Blosc2 chunk whose special-value bits (byte 31, bits 4-6) say zeros (1), NaN (2) or
    one repeated value (3, the value follows the header)."""
    z = bytearray(32)
    z[0], z[1], z[2], z[3] = 5, 1, 0x25, typesize
    z[4:8] = nbytes.to_bytes(4, "little")
    z[8:12] = blocksize.to_bytes(4, "little")
    z[31] = kind << 4
    if kind == 3:
        z += np.array([value], dtype=np.float64 if typesize == 8 else np.float32).tobytes()
    z[12:16] = len(z).to_bytes(4, "little")
    return bytes(z)


PARTITIONS = [
    # M, K, chunkshape, blockshape
    (300, 260, (100, 80), (25, 20)),
    (517, 333, (128, 96), (32, 24)),        # edge blocks and chunk padding in both dimensions
    (64, 1000, (64, 500), (16, 100)),
    (257, 4096, (128, 4096), (8, 4096)),    # one slice per block row: the longest rows taken
    (1000, 1000, (500, 500), (100, 100)),
]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("part", PARTITIONS, ids=lambda p: f"{p[0]}x{p[1]}_c{p[2][0]}x{p[2][1]}_b{p[3][0]}x{p[3][1]}")
def test_fused_gemv_integer_exact(ia, dtype, part):
    M, K, ch, bl = part
    rng = np.random.default_rng(61)
    A, x = _ints(rng, (M, K), dtype), _ints(rng, (K,), dtype)
    ref = A.astype(np.float64) @ x.astype(np.float64)
    ctx = ia.Context()
    Ac = ia.Container.from_numpy(ctx, A, ch, bl)
    xc = ia.Container.from_numpy(ctx, x, (ch[1],), (bl[1],))
    for entry in (ia.opt_gemv, ia.matmul):
        y = entry(ctx, Ac, xc, (ch[0],), (bl[0],))
        got = y.to_numpy()
        y.free()
        assert got.dtype == dtype
        np.testing.assert_array_equal(got.astype(np.float64), ref)
    ctx.close()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_fused_gemv_chunk_kinds(ia, dtype):
    """Special zero, NaN and value chunks, memcpyed chunks (compression level 0) and unshuffled
    chunks take the item-by-item path of the fused kernel; the result is the oracle's."""
    M, K, ch, bl = 200, 160, (50, 80), (25, 20)
    rng = np.random.default_rng(62)
    A, x = _ints(rng, (M, K), dtype), _ints(rng, (K,), dtype)
    isz = np.dtype(dtype).itemsize
    ga, ach = O.encode_array(A, ch, bl)
    nbytes, bsz = ga.chunk_nbytes, bl[0] * bl[1] * isz
    ach[1] = _special_chunk(nbytes, bsz, isz, 1)
    ach[2] = _special_chunk(nbytes, bsz, isz, 3, 2.0)
    ach[5] = _special_chunk(nbytes, bsz, isz, 2)
    ctx = ia.Context()
    Ac = ia.Container.from_chunks(ctx, (M, K), dtype, ch, bl, ach)
    gx, xch = O.encode_array(x, (ch[1],), (bl[1],))
    xc = ia.Container.from_chunks(ctx, (K,), dtype, (ch[1],), (bl[1],), xch)
    dt = O.DTYPE_DOUBLE if isz == 8 else O.DTYPE_FLOAT
    dense = O.decode_array(ga, ach, dtype)
    # the plain decode of the same chunks (the value chunk's item sits at an odd offset)
    np.testing.assert_array_equal(Ac.to_numpy(), dense)
    got = ia.matmul(ctx, Ac, xc, (ch[0],), (bl[0],)).to_numpy()
    ref = dense.astype(np.float64) @ x.astype(np.float64)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_array_equal(got[~np.isnan(got)].astype(np.float64), ref[~np.isnan(ref)])
    # iarray_opt_gemv skips the special-zero chunk and its NaN chunk faces no zero block of x
    got2 = ia.opt_gemv(ctx, Ac, xc, (ch[0],), (bl[0],)).to_numpy()
    ref2 = O.opt_gemv(ga, ach, gx, xch, O.Geom((M,), (ch[0],), (bl[0],), isz), dt)
    np.testing.assert_array_equal(np.isnan(got2), np.isnan(ref2))
    np.testing.assert_array_equal(got2[~np.isnan(got2)], ref2[~np.isnan(ref2)])
    ctx.close()
    # memcpyed (level 0) and unshuffled chunks
    for level, flags in ((0, 1), (5, 0)):
        cfg = ia.Config.defaults()
        cfg.compression_level, cfg.filter_flags = level, flags
        ctx = ia.Context(cfg=cfg)
        Ac = ia.Container.from_numpy(ctx, A, ch, bl)
        xc = ia.Container.from_numpy(ctx, x, (ch[1],), (bl[1],))
        got = ia.matmul(ctx, Ac, xc, (ch[0],), (bl[0],)).to_numpy()
        np.testing.assert_array_equal(got.astype(np.float64), A.astype(np.float64) @ x.astype(np.float64))
        ctx.close()


def test_fused_gemv_repeats_bitwise(ia):
    """Non-integer data: two calls give the same bytes, and the result is within float32
    rounding of the float64 product."""
    M, K, ch, bl = 3000, 2000, (1000, 1000), (100, 100)
    rng = np.random.default_rng(63)
    A = rng.standard_normal((M, K)).astype(np.float32)
    x = rng.standard_normal(K).astype(np.float32)
    ctx = ia.Context()
    Ac = ia.Container.from_numpy(ctx, A, ch, bl)
    xc = ia.Container.from_numpy(ctx, x, (ch[1],), (bl[1],))
    y1 = ia.opt_gemv(ctx, Ac, xc, (ch[0],), (bl[0],)).to_numpy()
    y2 = ia.opt_gemv(ctx, Ac, xc, (ch[0],), (bl[0],)).to_numpy()
    assert y1.tobytes() == y2.tobytes()
    ref = A.astype(np.float64) @ x.astype(np.float64)
    assert np.linalg.norm(y1 - ref) / np.linalg.norm(ref) < 1e-6
    ctx.close()
