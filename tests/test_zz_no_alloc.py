"""iarray_b200_decode_noalloc, the decode entry point that allocates nothing (its work
buffers live in a fixed device array of the library), checked through the C ABI against
iarray_b200_decode_to_device on the same chunks.  Decoding is byte work: bit-exact."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_BYTES = 8 << 20
MAX_BLOCKS = 4096


def _arr(vals):
    return (ctypes.c_int64 * len(vals))(*vals)


def _device_chunks(torch, c):
    """The container's chunks back to back in caller-allocated device memory."""
    blob = b"".join(c.chunks())
    return torch.frombuffer(bytearray(blob), dtype=torch.uint8).cuda(), len(blob)


def _noalloc(ia, torch, shape, chunk, block, itemsize, dchunks, nbytes, out, ld):
    stream = torch.cuda.current_stream().cuda_stream
    return ia.lib().iarray_b200_decode_noalloc(len(shape), _arr(shape), _arr(chunk), _arr(block), itemsize,
                                               dchunks.data_ptr(), nbytes, out.data_ptr(), ld, stream)


def _existing(ia, ctx, c, out, ld):
    ia.check(ia.lib().iarray_b200_decode_to_device(ctx.ptr, c.ptr, out.data_ptr(), ld), "decode_to_device")


@pytest.mark.parametrize("dtype,shape,chunk,block", [
    (np.float64, (300, 670), (128, 256), (32, 64)),     # ragged edge chunks and interior blocks
    (np.float32, (5000,), (1200,), (256,)),
])
def test_noalloc_decode_matches_decode_to_device_twice(ctx, ia, dtype, shape, chunk, block):
    import torch
    rng = np.random.default_rng(11)
    itemsize = np.dtype(dtype).itemsize
    ld = shape[-1]
    rows = shape[0] if len(shape) == 2 else 1
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    datas = [(np.round(rng.standard_normal(shape), 3)).astype(dtype),      # compressible
             rng.uniform(-1, 1, shape).astype(dtype)]                     # mostly raw streams
    for a in datas:                                                       # two calls in a row
        c = ia.Container.from_numpy(ctx, a, chunk, block)
        dchunks, nbytes = _device_chunks(torch, c)
        mine = torch.full((rows, ld), float("nan"), dtype=tdt, device="cuda")
        ref = torch.full((rows, ld), float("nan"), dtype=tdt, device="cuda")
        ia.check(_noalloc(ia, torch, shape, chunk, block, itemsize, dchunks, nbytes, mine, ld), "decode_noalloc")
        _existing(ia, ctx, c, ref, ld)
        torch.cuda.synchronize()
        m, r = mine.cpu().numpy(), ref.cpu().numpy()
        assert m.tobytes() == r.tobytes()
        assert m.reshape(a.shape).tobytes() == a.tobytes()


def test_noalloc_rejects_oversized_and_corrupt_input(ctx, ia):
    import torch
    dummy = torch.zeros(64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # 1100 x 1000 float64 is 8.8 MB decoded, above the 8 MiB limit: rejected before any launch
    rc = _noalloc(ia, torch, (1100, 1000), (1100, 1000), (100, 100), 8, dummy, 64, out, 1000)
    assert rc & ia.RC_ERROR_BIT and ia.ERR_NAME[rc & 0xFFFFFF] == "NOALLOC_TOO_LARGE"
    # 8192 blocks of 8 items exceed the block limit
    rc = _noalloc(ia, torch, (65536,), (65536,), (8,), 8, dummy, 64, out, 65536)
    assert rc & ia.RC_ERROR_BIT and ia.ERR_NAME[rc & 0xFFFFFF] == "NOALLOC_TOO_LARGE"
    # a truncated chunk buffer is reported as a Blosc failure, and the next call still works
    a = np.arange(64 * 64, dtype=np.float64).reshape(64, 64)
    c = ia.Container.from_numpy(ctx, a, (64, 64), (16, 16))
    dchunks, nbytes = _device_chunks(torch, c)
    dense = torch.zeros((64, 64), dtype=torch.float64, device="cuda")
    rc = _noalloc(ia, torch, (64, 64), (64, 64), (16, 16), 8, dchunks, nbytes // 2, dense, 64)
    assert rc & ia.RC_ERROR_BIT and ia.ERR_NAME[rc & 0xFFFFFF] == "BLOSC_FAILED"
    ia.check(_noalloc(ia, torch, (64, 64), (64, 64), (16, 16), 8, dchunks, nbytes, dense, 64), "decode_noalloc")
    assert np.array_equal(dense.cpu().numpy(), a)


@pytest.mark.parametrize("dtype,shape,chunk,block", [
    (np.int16, (257, 300), (100, 128), (20, 32)),       # 2-byte items: the general scatter path
    (np.uint8, (1000,), (384,), (96,)),                 # 1-byte items, never shuffled
])
def test_noalloc_small_items(ctx, ia, dtype, shape, chunk, block):
    import torch
    rng = np.random.default_rng(12)
    a = (rng.integers(0, 40, shape) * 3).astype(dtype)
    c = ia.Container.from_numpy(ctx, a, chunk, block)
    dchunks, nbytes = _device_chunks(torch, c)
    rows, ld = (shape[0] if len(shape) == 2 else 1), shape[-1]
    tdt = torch.int16 if dtype == np.int16 else torch.uint8
    for _ in range(2):
        mine = torch.full((rows, ld), 7, dtype=tdt, device="cuda")
        ref = torch.full((rows, ld), 7, dtype=tdt, device="cuda")
        ia.check(_noalloc(ia, torch, shape, chunk, block, a.itemsize, dchunks, nbytes, mine, ld), "decode_noalloc")
        _existing(ia, ctx, c, ref, ld)
        torch.cuda.synchronize()
        assert mine.cpu().numpy().tobytes() == ref.cpu().numpy().tobytes() == a.tobytes()


def test_noalloc_at_the_limits_allocates_nothing(ctx, ia):
    """1024 x 1024 float64 in one chunk of 16 x 16 blocks: exactly 8 MiB decoded and 4096
    blocks, both limits reached.  After a first call, further calls leave the device's free
    memory unchanged: the call itself allocates nothing."""
    import torch
    rng = np.random.default_rng(13)
    n = 1024
    a = np.round(rng.standard_normal((n, n)), 2)
    c = ia.Container.from_numpy(ctx, a, (n, n), (16, 16))
    dchunks, nbytes = _device_chunks(torch, c)
    mine = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    ref = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    ia.check(_noalloc(ia, torch, (n, n), (n, n), (16, 16), 8, dchunks, nbytes, mine, n), "decode_noalloc")
    _existing(ia, ctx, c, ref, n)
    torch.cuda.synchronize()
    assert mine.cpu().numpy().tobytes() == ref.cpu().numpy().tobytes() == a.tobytes()
    free0, _ = torch.cuda.mem_get_info()
    mine.zero_()
    torch.cuda.synchronize()
    for _ in range(3):
        ia.check(_noalloc(ia, torch, (n, n), (n, n), (16, 16), 8, dchunks, nbytes, mine, n), "decode_noalloc")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert mine.cpu().numpy().tobytes() == a.tobytes()
    # one more row than the limit is rejected before any launch
    rc = _noalloc(ia, torch, (n + 16, n), (n + 16, n), (16, 16), 8, dchunks, nbytes, mine, n)
    assert rc & ia.RC_ERROR_BIT and ia.ERR_NAME[rc & 0xFFFFFF] == "NOALLOC_TOO_LARGE"


def test_noalloc_rejects_wrapping_geometry(ctx, ia):
    """A shape whose chunk count times chunk size would overflow 64 bits is rejected, not
    wrapped into a small number that passes the limits."""
    import torch
    dummy = torch.zeros(64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _noalloc(ia, torch, (1 << 32, 1 << 32), (1, 1), (1, 1), 8, dummy, 64, out, 1 << 32)
    assert rc & ia.RC_ERROR_BIT
    assert ia.ERR_NAME[rc & 0xFFFFFF] in ("NOALLOC_TOO_LARGE", "INVALID_ARGUMENT")
