"""CPU tests of the oracle: pinned against the reference's golden Blosc2 frames and
against liblz4 itself, and its GEMM/GEMV loop restatements against plain numpy."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
DIGESTS = json.load(open(os.path.join(GOLD, "golden_digests.json")))
CHUNK_FILES = sorted(f for f in os.listdir(GOLD) if f.startswith("chunk_") and f.endswith(".bin"))


def _golden_chunks():
    for f in CHUNK_FILES:
        name = f[len("chunk_"):-len("_0.bin")]
        yield name, open(os.path.join(GOLD, f), "rb").read()


@pytest.mark.parametrize("name,chunk", list(_golden_chunks()))
def test_golden_chunk_decodes_to_digest(name, chunk):
    d = DIGESTS[name]["chunks"][0]
    assert hashlib.sha256(chunk).hexdigest() == d["sha_chunk"]
    assert hashlib.sha256(O.chunk_decompress(chunk)).hexdigest() == d["sha_decoded"]


@pytest.mark.parametrize("name,chunk", list(_golden_chunks()))
def test_golden_chunk_reencodes_byte_identical(name, chunk):
    """Same header, and every block's streams byte-identical (bstarts order aside:
    the reference writes blocks in thread-completion order)."""
    h = O.chunk_header(chunk)
    re = O.chunk_compress(O.chunk_decompress(chunk), h["typesize"], h["blocksize"], True, O.SPLIT_AUTO)
    assert re[:12] == chunk[:12] and re[12:32] == chunk[12:32]
    gb, mb = O.chunk_blocks(chunk), O.chunk_blocks(re)
    assert len(gb) == len(mb)
    for (s, e), (s2, e2) in zip(gb, mb):
        assert chunk[s:e] == re[s2:e2]


def test_golden_digests_cover_every_frame():
    assert len(DIGESTS) == 10
    kinds = {"zero": 0, "raw": 0, "lz4": 0, "run": 0}
    for d in DIGESTS.values():
        assert d["typesize"] == 4 and d["blocksize"] == 40000 and d["chunksize"] == 400000
        assert len(d["chunks"]) == 10
        for c in d["chunks"]:
            for k, v in c["kinds"].items():
                kinds[k] += v
        # header layout pinned: magic, 64-bit offsets flag, LZ4 at clevel 5
        hb = bytes.fromhex(d["header_hex"])
        assert hb[:10] == b"\x9e\xa8b2frame\x00" and hb[25] == 0x12 and hb[27] == 0x51
    assert kinds["zero"] > 0 and kinds["raw"] > 0 and kinds["lz4"] > 0


@pytest.mark.skipif(not os.environ.get("IRONARRAY_REFERENCE_DIR"), reason="reference checkout not given")
def test_every_reference_frame_roundtrips():
    import glob
    ref = os.environ["IRONARRAY_REFERENCE_DIR"]
    for f in sorted(glob.glob(os.path.join(ref, "tests", "data", "test_*.iarray"))):
        name = os.path.basename(f)[:-len(".iarray")]
        fr = O.read_frame(open(f, "rb").read())
        for c, d in zip(fr["chunks"], DIGESTS[name]["chunks"]):
            assert hashlib.sha256(O.chunk_decompress(c)).hexdigest() == d["sha_decoded"]
            h = O.chunk_header(c)
            re = O.chunk_compress(O.chunk_decompress(c), h["typesize"], h["blocksize"])
            for (s, e), (s2, e2) in zip(O.chunk_blocks(c), O.chunk_blocks(re)):
                assert c[s:e] == re[s2:e2]


def _liblz4():
    try:
        return ctypes.CDLL("liblz4.so.1")
    except OSError:
        return None


@pytest.mark.skipif(_liblz4() is None, reason="liblz4.so.1 not present")
def test_lz4_encoder_matches_liblz4():
    lz = _liblz4()
    rng = np.random.default_rng(11)

    def ref(src, cap):
        dst = ctypes.create_string_buffer(cap + 64)
        n = lz.LZ4_compress_fast(src, dst, len(src), cap, 1)
        return dst.raw[:n]

    cases = 0
    for n in [13, 100, 4096, 10000, 65535, 65546, 65547, 70000, 250000]:
        for kind in range(5):
            if kind == 0:
                s = rng.integers(0, 256, n, dtype=np.uint8)
            elif kind == 1:
                s = rng.integers(0, 3, n, dtype=np.uint8)
            elif kind == 2:
                s = (np.arange(n) // 5 % 251).astype(np.uint8)
            elif kind == 3:
                s = rng.standard_normal(n // 4 + 1).astype(np.float32).view(np.uint8)[:n].copy()
            else:
                v = np.sin(0.001 * np.arange(n // 4 + 1)).astype(np.float32).view(np.uint8)
                s = v.reshape(-1, 4).T.copy().ravel()[:n]
            src = s.tobytes()
            full = ref(src, n + n // 255 + 32)
            for cap in {n, n - 1, len(full) - 1, len(full), len(full) + 1}:
                if cap <= 0:
                    continue
                assert O.lz4_compress(src, cap) == ref(src, cap), (n, kind, cap)
                cases += 1
    assert cases > 100


def test_lz4_roundtrip_and_malformed_streams():
    rng = np.random.default_rng(5)
    src = (rng.integers(0, 4, 5000, dtype=np.uint8)).tobytes()
    comp = O.lz4_compress(src, len(src))
    assert 0 < len(comp) < len(src)
    assert O.lz4_decompress(comp, len(src)) == src
    with pytest.raises(ValueError):
        O.lz4_decompress(comp[:-3], len(src))          # truncated
    bad = bytearray(comp)
    lit, p = bad[0] >> 4, 1
    if lit == 15:
        while bad[p] == 255:
            lit += 255
            p += 1
        lit += bad[p]
        p += 1
    bad[p + lit + 1] = 0xff                              # first offset beyond output start
    with pytest.raises(ValueError):
        O.lz4_decompress(bytes(bad), len(src))


@pytest.mark.parametrize("splitmode", [O.SPLIT_AUTO, O.SPLIT_NEVER, O.SPLIT_ALWAYS])
@pytest.mark.parametrize("kind", ["random", "smooth", "zeros", "const", "ints"])
def test_chunk_roundtrip_kinds(kind, splitmode):
    rng = np.random.default_rng(1)
    n = 4096
    a = {"random": np.frombuffer(rng.bytes(8 * n), np.float64), "smooth": np.sin(np.arange(n) * 0.01), "zeros": np.zeros(n),
         "const": np.full(n, 3.25), "ints": rng.integers(0, 5, n).astype(np.float64)}[kind]
    raw = a.tobytes()
    c = O.chunk_compress(raw, 8, 8 * 512, True, splitmode)
    assert O.chunk_decompress(c) == raw
    h = O.chunk_header(c)
    assert h["split"] == (splitmode != O.SPLIT_NEVER)
    if kind == "random" and splitmode != O.SPLIT_NEVER:
        assert h["memcpyed"]          # all-raw streams overflow nbytes + 32
    if kind == "const" and splitmode != O.SPLIT_NEVER:
        streams = O.chunk_streams(c)
        assert any(cs < 0 for blk in streams for cs, _ in blk)   # non-zero byte runs


def test_block_is_zeros_and_special_chunks():
    a = np.zeros(2048)
    a[1024:] = 1.0
    c = O.chunk_compress(a.tobytes(), 8, 8 * 256)
    assert O.LIB.ora_block_is_zeros(c, 0) == 1
    assert O.LIB.ora_block_is_zeros(c, 5) == 0
    z = bytearray(32)
    z[0], z[1], z[2], z[3] = 5, 1, 0x25, 8
    z[4:8] = (2048 * 8).to_bytes(4, "little")
    z[8:12] = (256 * 8).to_bytes(4, "little")
    z[12:16] = (32).to_bytes(4, "little")
    z[31] = 1 << 4
    assert O.LIB.ora_chunk_is_zeros(bytes(z)) == 1
    assert O.chunk_decompress(bytes(z)) == bytes(2048 * 8)


@pytest.mark.parametrize("M,K,N,ca,ba,cb,bb", [
    (50, 40, 30, (20, 16), (7, 5), (16, 13), (5, 6)),
    (33, 33, 33, (33, 33), (11, 11), (33, 33), (11, 11)),
    (64, 100, 17, (32, 50), (32, 25), (50, 17), (25, 17)),
])
def test_oracle_opt_gemm_matches_numpy(M, K, N, ca, ba, cb, bb):
    rng = np.random.default_rng(2)
    A, B = rng.uniform(-1, 1, (M, K)), rng.uniform(-1, 1, (K, N))
    ga, ach = O.encode_array(A, ca, ba)
    gb, bch = O.encode_array(B, cb, bb)
    gc = O.Geom((M, N), (ca[0], cb[1]), (ba[0], bb[1]), 8)
    C = O.opt_gemm(ga, ach, gb, bch, gc, O.DTYPE_DOUBLE)
    assert np.allclose(C, A @ B, rtol=1e-12, atol=1e-12)


def test_oracle_opt_gemv_matches_numpy():
    rng = np.random.default_rng(3)
    A, x = rng.uniform(-1, 1, (61, 47)), rng.uniform(-1, 1, 47)
    ga, ach = O.encode_array(A, (20, 16), (7, 5))
    gx, xch = O.encode_array(x, (16,), (5,))
    gc = O.Geom((61,), (20,), (7,), 8)
    y = O.opt_gemv(ga, ach, gx, xch, gc, O.DTYPE_DOUBLE)
    assert np.allclose(y, A @ x, rtol=1e-12, atol=1e-12)


def test_dd_rows_exact_on_integers():
    rng = np.random.default_rng(4)
    A = rng.integers(-1000, 1000, (6, 300)).astype(np.float64)
    B = rng.integers(-1000, 1000, (300, 40)).astype(np.float64)
    hi, lo = O.dd_rows(A, B, [0, 3, 5], nthreads=2)
    exact = (A.astype(object) @ B.astype(object))[[0, 3, 5]]
    assert np.array_equal(hi, exact.astype(np.float64)) and not lo.any()
    # and the error metric is 0 on the exact answer
    assert O.normwise_error(A @ B, hi, lo, [0, 3, 5]) == 0.0


def test_caterva_layout_roundtrip_ragged():
    rng = np.random.default_rng(6)
    A = rng.standard_normal((37, 53))
    g, chunks = O.encode_array(A, (10, 20), (3, 7))
    assert g.nchunks == 4 * 3 and g.extchunk == (12, 21)
    assert np.array_equal(O.decode_array(g, chunks, np.float64), A)


def test_cpu_baseline_whole_product_matches_oracle():
    """The timed CPU baseline (the reference's block-pair loop over every output chunk, with
    each block compressed by its worker) decodes to the oracle's product."""
    if O.openblas_dgemm() is None:
        pytest.skip("no cblas_dgemm in this environment")
    rng = np.random.default_rng(8)
    A, B = rng.uniform(-1, 1, (96, 80)), rng.uniform(-1, 1, (80, 70))
    A[:32, :40] = 0.0                                    # a zero chunk: skipped by the loop
    ga, ach = O.encode_array(A, (32, 40), (16, 20))
    gb, bch = O.encode_array(B, (40, 32), (20, 16))
    gc = O.Geom((96, 70), (32, 32), (16, 16), 8)
    chunks = O.cpu_opt_gemm(ga, ach, gb, bch, gc, 3)
    assert len(chunks) == gc.nchunks
    C = O.decode_array(gc, chunks, np.float64)
    ref = O.opt_gemm(ga, ach, gb, bch, gc, O.DTYPE_DOUBLE)
    assert np.allclose(C, ref, rtol=1e-13, atol=1e-13)
    for c in chunks:                                     # every chunk is valid Blosc2 for the oracle
        assert len(O.chunk_decompress(c)) == gc.chunk_nbytes


def test_committed_reference_frame_matches_digests():
    """The whole reference-written frame committed as a fixture: the oracle's frame reader
    finds every chunk, and each chunk and its decoding match the recorded digests."""
    import hashlib
    name = "test_binomial_int32_n1_p0.7"
    buf = open(os.path.join(GOLD, f"{name}.iarray"), "rb").read()
    fr = O.read_frame(buf)
    want = DIGESTS[name]["chunks"]
    assert len(fr["chunks"]) == len(want)
    for c, w in zip(fr["chunks"], want):
        assert hashlib.sha256(c).hexdigest() == w["sha_chunk"]
        assert hashlib.sha256(O.chunk_decompress(c)).hexdigest() == w["sha_decoded"]
