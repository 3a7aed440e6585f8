"""Frames on disk through the C ABI: a whole frame written by the reference's toolchain
(tests/data/test_binomial_int32_n1_p0.7.iarray, committed under tests/golden/) opened by
iarray_container_open and decoded on the GPU, and sparse (directory) frames written for
storage.contiguous = false, read back by iarray_container_open / _load and removed by
iarray_container_remove."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DIGESTS = json.load(open(os.path.join(GOLD, "golden_digests.json")))


@pytest.mark.parametrize("load", [False, True])
def test_reference_frame_opens_and_decodes(ctx, ia, load):
    name = "test_binomial_int32_n1_p0.7"
    path = os.path.join(GOLD, f"{name}.iarray")
    c = ia.Container.open(ctx, path, load=load)
    meta = DIGESTS[name]
    assert c.shape == (1000000,)
    assert c.dtype == np.int32
    x = c.to_numpy()
    chunk = 100000
    for k, w in enumerate(meta["chunks"]):
        piece = x[k * chunk:(k + 1) * chunk]
        assert hashlib.sha256(piece.tobytes()).hexdigest() == w["sha_decoded"], k
        assert hashlib.sha256(c.chunks()[k]).hexdigest() == w["sha_chunk"], k
    assert 0.69 < x.mean() < 0.71 and set(np.unique(x)) <= {0, 1}
    # the library writes it back as a frame the oracle reads, chunk for chunk
    fr = O.read_frame(c.to_cframe())
    assert [hashlib.sha256(b).hexdigest() for b in fr["chunks"]] == [w["sha_chunk"] for w in meta["chunks"]]


def test_sparse_frame_roundtrip(ctx, ia, tmp_path):
    rng = np.random.default_rng(31)
    a = np.round(rng.standard_normal((300, 257)), 2)
    d = str(tmp_path / "a.iarray")
    c = ia.Container.from_numpy(ctx, a, (128, 100), (32, 25), urlpath=d, contiguous=False)
    assert os.path.isdir(d)
    nch = 3 * 3
    assert sorted(os.listdir(d)) == sorted(["chunks.b2frame"] + [f"{k:08X}.chunk" for k in range(nch)])
    for k in range(nch):
        assert open(os.path.join(d, f"{k:08X}.chunk"), "rb").read() == c.chunks()[k]
    index = open(os.path.join(d, "chunks.b2frame"), "rb").read()
    assert index[:10] == b"\x9e\xa8b2frame\x00" and index[26] == 1        # directory frame type
    # the index frame carries the same header fields and metalayers as the contiguous frame
    contiguous = c.to_cframe()
    assert index[27:29] == contiguous[27:29]
    for load in (False, True):
        assert np.array_equal(ia.Container.open(ctx, d, load=load).to_numpy(), a)
    ia.Container.remove(d)
    assert not os.path.exists(d)


def test_matmul_output_as_sparse_frame(ctx, ia, tmp_path):
    rng = np.random.default_rng(32)
    A, B = rng.uniform(-1, 1, (120, 90)), rng.uniform(-1, 1, (90, 70))
    d = str(tmp_path / "c.iarray")
    C = ia.matmul(ctx, ia.Container.from_numpy(ctx, A, (40, 30), (20, 15)),
                  ia.Container.from_numpy(ctx, B, (30, 35), (15, 35)), (60, 35), (30, 35), urlpath=d, contiguous=False)
    back = ia.Container.open(ctx, d)
    assert back.chunks() == C.chunks()
    assert np.allclose(back.to_numpy(), A @ B, rtol=1e-13, atol=1e-13)
    ia.Container.remove(d)
    # a container already on disk is not saved again (src/iarray_container.c:63-66)
    with pytest.raises(ia.IArrayError) as e:
        C.save(str(tmp_path / "again.iarray"))
    assert e.value.name == "INVALID_STORAGE"
    # a contiguous frame file is removed too
    f = str(tmp_path / "f.iarray")
    ia.Container.from_numpy(ctx, A, (40, 30), (20, 15)).save(f)
    ia.Container.remove(f)
    assert not os.path.exists(f)


def test_compression_level_zero_writes_memcpyed_chunks(ia, tmp_path):
    """compression_level 0 (accepted by the reference's context, passed on to Blosc2 by
    src/iarray.c:391-439) stores every chunk memcpyed: the 32-byte header with the memcpyed
    flag, then the chunk's padded items unshuffled.  Products written with it read back."""
    cfg = ia.Config.defaults()
    cfg.compression_level = 0
    ctx = ia.Context(cfg)
    rng = np.random.default_rng(33)
    a = np.round(rng.standard_normal((130, 90)), 3)
    ch, bl = (64, 64), (32, 16)
    c = ia.Container.from_numpy(ctx, a, ch, bl)
    g = O.Geom(a.shape, ch, bl, 8)
    for k, chunk in enumerate(c.chunks()):
        assert chunk[2] & 0x02 and len(chunk) == g.chunk_nbytes + 32
        assert int.from_bytes(chunk[12:16], "little") == g.chunk_nbytes + 32
        assert chunk[32:] == g.chunk_from_array(a, k).tobytes()
        assert O.chunk_decompress(chunk) == g.chunk_from_array(a, k).tobytes()
    assert np.array_equal(c.to_numpy(), a)
    fr = c.to_cframe()
    assert fr[27] == 0x01                                # clevel 0 << 4 | LZ4
    C = ia.opt_gemm(ctx, c, ia.Container.from_numpy(ctx, a.T.copy(), (64, 64), (16, 32)), (64, 64), (32, 32))
    assert all(x[2] & 0x02 for x in C.chunks())
    np.testing.assert_allclose(C.to_numpy(), a @ a.T, rtol=1e-12, atol=1e-12)
    d = str(tmp_path / "z.iarray")
    c2 = ia.Container.from_numpy(ctx, a, ch, bl, urlpath=d)
    assert np.array_equal(ia.Container.open(ctx, d).to_numpy(), a)
    c2.free()
    ctx.close()
