"""ORACLE — test infrastructure only.

ctypes wrapper over oracle/lib/libblosc_oracle.so (the plain-C restatement of the
reference's Blosc2 LZ4+SHUFFLE codec and blocked GEMM/GEMV loops) plus numpy helpers
for Caterva's padded blocked layout and for reading/writing Blosc2 contiguous frames.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module, always as the checker.  The product library never calls it.

Reference anchors:
  - chunk/block layout: Caterva, as configured by iarray_create_caterva_storage
    (src/iarray.c:532-552) and used by iarray_from_buffer (src/iarray_constructor.c:218-262);
  - "iarray" metalayer: _iarray_serialize_meta (src/iarray_private.h:364-387);
  - codec parameters: iarray_create_blosc_cparams (src/iarray.c:391-439);
  - frame layout: pinned on the reference's own frames tests/data/test_<dist>.iarray.
"""
from __future__ import annotations

import ctypes
import os
import struct

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libblosc_oracle.so")


def build():
    """Compile the oracle C restatement (make -C oracle)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    P, I, I64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    lib.ora_lz4_decompress.argtypes = [P, I, P, I]
    lib.ora_lz4_compress_limited.argtypes = [P, I, P, I]
    lib.ora_chunk_compress.argtypes = [P, I, I, I, I, I, P, I]
    lib.ora_chunk_decompress.argtypes = [P, I, P, I]
    lib.ora_chunk_is_zeros.argtypes = [P]
    lib.ora_block_is_zeros.argtypes = [P, I]
    lib.ora_split_decision.argtypes = [I, I, I, I, I]
    lib.ora_opt_gemm.argtypes = [P, P, P, I, P]
    lib.ora_opt_gemv.argtypes = [P, P, P, I, P]
    lib.ora_dense_gemm.argtypes = [I, I64, I64, I64, P, P, P]
    lib.ora_dd_rows.argtypes = [P, P, I64, I64, I64, P, I64, P, P, I]
    return lib


LIB = _load()

DTYPE_DOUBLE, DTYPE_FLOAT = 0, 1
NP_OF = {DTYPE_DOUBLE: np.float64, DTYPE_FLOAT: np.float32}
SPLIT_ALWAYS, SPLIT_NEVER, SPLIT_AUTO, SPLIT_FORWARD_COMPAT = 1, 2, 3, 4


def _ptr(a):
    if isinstance(a, (bytes, bytearray)):
        return ctypes.cast(ctypes.c_char_p(bytes(a)), ctypes.c_void_p)
    return ctypes.c_void_p(a.ctypes.data)


# ----------------------------------------------------------------------------- LZ4
def lz4_compress(src: bytes, cap: int) -> bytes:
    buf = ctypes.create_string_buffer(max(cap, 1) + 16)
    n = LIB.ora_lz4_compress_limited(src, len(src), buf, cap)
    return buf.raw[:n]


def lz4_decompress(src: bytes, n: int) -> bytes:
    buf = ctypes.create_string_buffer(max(n, 1))
    r = LIB.ora_lz4_decompress(src, len(src), buf, n)
    if r != n:
        raise ValueError(f"lz4 decode error {r}")
    return buf.raw[:n]


# ----------------------------------------------------------------------------- chunks
def chunk_compress(data: bytes, typesize: int, blocksize: int, shuffle: bool = True,
                   splitmode: int = SPLIT_AUTO) -> bytes:
    n = len(data)
    cap = n + 32 + 4 * (n // max(blocksize, 1) + 1) * (typesize + 1) + 64
    buf = ctypes.create_string_buffer(cap)
    # Blosc2's callers give dest capacity nbytes + BLOSC2_MAX_OVERHEAD (32).
    r = LIB.ora_chunk_compress(data, n, typesize, blocksize, int(shuffle), splitmode, buf, n + 32)
    if r < 0:
        raise ValueError(f"chunk compress error {r}")
    return buf.raw[:r]


def chunk_decompress(chunk: bytes) -> bytes:
    nbytes = struct.unpack_from("<i", chunk, 4)[0]
    buf = ctypes.create_string_buffer(max(nbytes, 1))
    r = LIB.ora_chunk_decompress(chunk, len(chunk), buf, nbytes)
    if r != nbytes:
        raise ValueError(f"chunk decode error {r}")
    return buf.raw[:nbytes]


def chunk_header(chunk: bytes) -> dict:
    flags, ts = chunk[2], chunk[3]
    nbytes, blocksize, cbytes = struct.unpack_from("<iii", chunk, 4)
    return dict(version=chunk[0], flags=flags, typesize=ts, nbytes=nbytes, blocksize=blocksize,
                cbytes=cbytes, memcpyed=bool(flags & 2), split=not (flags & 0x10),
                codec=flags >> 5, special=(chunk[31] >> 4) & 7)


def chunk_blocks(chunk: bytes) -> list[tuple[int, int]]:
    """(start, end) byte range of each block's stream data, in block order."""
    h = chunk_header(chunk)
    if h["memcpyed"] or h["special"]:
        return []
    nblocks = -(-h["nbytes"] // h["blocksize"])
    leftover = h["nbytes"] % h["blocksize"]
    out = []
    for b in range(nblocks):
        start = struct.unpack_from("<i", chunk, 32 + 4 * b)[0]
        bsize = leftover if (b == nblocks - 1 and leftover) else h["blocksize"]
        nstreams = h["typesize"] if (h["split"] and not (b == nblocks - 1 and leftover)) else 1
        p = start
        for _ in range(nstreams):
            cs = struct.unpack_from("<i", chunk, p)[0]
            p += 4 + (cs if cs > 0 else (1 if cs < 0 else 0))
        out.append((start, p))
    return out


def chunk_streams(chunk: bytes) -> list[list[tuple[int, bytes]]]:
    """Per block, per stream: (csize, payload bytes)."""
    h = chunk_header(chunk)
    res = []
    for (s, e) in chunk_blocks(chunk):
        p, streams = s, []
        while p < e:
            cs = struct.unpack_from("<i", chunk, p)[0]
            ln = cs if cs > 0 else (1 if cs < 0 else 0)
            streams.append((cs, chunk[p + 4:p + 4 + ln]))
            p += 4 + ln
        res.append(streams)
    return res


# ----------------------------------------------------------------------------- layout
def ceil_to(a, b):
    return -(-a // b) * b


class Geom:
    """Caterva partition: shape, chunkshape, blockshape (all ndim-long)."""

    def __init__(self, shape, chunkshape, blockshape, itemsize):
        self.shape = tuple(int(s) for s in shape)
        self.chunk = tuple(int(s) for s in chunkshape)
        self.block = tuple(int(s) for s in blockshape)
        self.itemsize = int(itemsize)
        self.ndim = len(self.shape)
        self.extshape = tuple(ceil_to(s, c) for s, c in zip(self.shape, self.chunk))
        self.extchunk = tuple(ceil_to(c, b) for c, b in zip(self.chunk, self.block))
        self.cgrid = tuple(e // c for e, c in zip(self.extshape, self.chunk))
        self.bgrid = tuple(e // b for e, b in zip(self.extchunk, self.block))
        self.nchunks = int(np.prod(self.cgrid))
        self.chunk_nbytes = int(np.prod(self.extchunk)) * self.itemsize
        self.blocksize = int(np.prod(self.block)) * self.itemsize

    def cstruct(self):
        class G(ctypes.Structure):
            _fields_ = [("ndim", ctypes.c_int), ("itemsize", ctypes.c_int),
                        ("shape", ctypes.c_int64 * 8), ("chunk", ctypes.c_int64 * 8),
                        ("block", ctypes.c_int64 * 8)]
        g = G()
        g.ndim, g.itemsize = self.ndim, self.itemsize
        for d in range(self.ndim):
            g.shape[d], g.chunk[d], g.block[d] = self.shape[d], self.chunk[d], self.block[d]
        return g

    def chunk_index(self, n):
        return np.unravel_index(n, self.cgrid)

    def chunk_from_array(self, arr: np.ndarray, n: int) -> np.ndarray:
        """Padded blocked item layout of chunk n (numpy, vectorised)."""
        ci = self.chunk_index(n)
        sl, pad = [], []
        for d in range(self.ndim):
            s = ci[d] * self.chunk[d]
            e = min(s + self.chunk[d], self.shape[d])
            sl.append(slice(s, e))
            pad.append((0, self.extchunk[d] - (e - s)))
        tile = np.pad(arr[tuple(sl)], pad)
        # split each axis into (bgrid, block) and move block-grid axes first
        shp = []
        for d in range(self.ndim):
            shp += [self.bgrid[d], self.block[d]]
        t = tile.reshape(shp)
        order = [2 * d for d in range(self.ndim)] + [2 * d + 1 for d in range(self.ndim)]
        return np.ascontiguousarray(t.transpose(order)).reshape(-1)

    def chunk_to_array(self, flat: np.ndarray, n: int, out: np.ndarray):
        ci = self.chunk_index(n)
        shp = list(self.bgrid) + list(self.block)
        t = flat.reshape(shp)
        order = []
        for d in range(self.ndim):
            order += [d, self.ndim + d]
        tile = t.transpose(order).reshape(self.extchunk)
        sl, tsl = [], []
        for d in range(self.ndim):
            s = ci[d] * self.chunk[d]
            e = min(s + self.chunk[d], self.shape[d])
            sl.append(slice(s, e))
            tsl.append(slice(0, e - s))
        out[tuple(sl)] = tile[tuple(tsl)]


def encode_array(arr: np.ndarray, chunkshape, blockshape, splitmode=SPLIT_AUTO):
    """numpy array -> list of Blosc2 chunks (LZ4 + SHUFFLE), row-major chunk order."""
    g = Geom(arr.shape, chunkshape, blockshape, arr.itemsize)
    return g, [chunk_compress(g.chunk_from_array(arr, n).tobytes(), g.itemsize, g.blocksize,
                              True, splitmode) for n in range(g.nchunks)]


def decode_array(g: Geom, chunks, dtype) -> np.ndarray:
    out = np.zeros(g.shape, dtype=dtype)
    for n, c in enumerate(chunks):
        flat = np.frombuffer(chunk_decompress(c), dtype=dtype)
        g.chunk_to_array(flat, n, out)
    return out


# ----------------------------------------------------------------------------- GEMM oracles
class _SChunk(ctypes.Structure):
    pass


def _schunk(g: Geom, chunks):
    gs = g.cstruct()

    class S(ctypes.Structure):
        _fields_ = [("g", type(gs)), ("chunks", ctypes.POINTER(ctypes.c_void_p)),
                    ("chunk_len", ctypes.POINTER(ctypes.c_int32))]
    bufs = [ctypes.create_string_buffer(bytes(c), len(c)) for c in chunks]
    arr = (ctypes.c_void_p * len(chunks))(*[ctypes.cast(b, ctypes.c_void_p) for b in bufs])
    lens = (ctypes.c_int32 * len(chunks))(*[len(c) for c in chunks])
    s = S(gs, arr, lens)
    s._keep = (bufs, arr, lens, gs)
    return s


def opt_gemm(ga: Geom, a_chunks, gb: Geom, b_chunks, gc: Geom, dtype: int, chunk_rule: int = 3) -> np.ndarray:
    """iarray_opt_gemm restated; returns C as a logical numpy array.  chunk_rule: which
    operands' special-zero chunks are skipped (bit 0 A, bit 1 B): 3 for iarray_opt_gemm, 2 for
    iarray_opt_gemm_a, 1 for iarray_opt_gemm_b."""
    sa, sb = _schunk(ga, a_chunks), _schunk(gb, b_chunks)
    cg = gc.cstruct()
    outs = [ctypes.create_string_buffer(gc.chunk_nbytes) for _ in range(gc.nchunks)]
    ptrs = (ctypes.c_void_p * gc.nchunks)(*[ctypes.cast(o, ctypes.c_void_p) for o in outs])
    if LIB.ora_opt_gemm_rule(ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(cg), dtype, ptrs, chunk_rule) != 0:
        raise ValueError("oracle opt_gemm failed")
    npdt = NP_OF[dtype]
    out = np.zeros(gc.shape, npdt)
    for n, o in enumerate(outs):
        gc.chunk_to_array(np.frombuffer(o.raw, npdt), n, out)
    return out


def opt_gemv(ga: Geom, a_chunks, gx: Geom, x_chunks, gc: Geom, dtype: int) -> np.ndarray:
    sa, sx = _schunk(ga, a_chunks), _schunk(gx, x_chunks)
    cg = gc.cstruct()
    outs = [ctypes.create_string_buffer(gc.chunk_nbytes) for _ in range(gc.nchunks)]
    ptrs = (ctypes.c_void_p * gc.nchunks)(*[ctypes.cast(o, ctypes.c_void_p) for o in outs])
    if LIB.ora_opt_gemv(ctypes.byref(sa), ctypes.byref(sx), ctypes.byref(cg), dtype, ptrs) != 0:
        raise ValueError("oracle opt_gemv failed")
    npdt = NP_OF[dtype]
    out = np.zeros(gc.shape, npdt)
    for n, o in enumerate(outs):
        gc.chunk_to_array(np.frombuffer(o.raw, npdt), n, out)
    return out


def dense_gemm(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """k-ascending dense product in the operands' own precision."""
    dt = DTYPE_DOUBLE if a.dtype == np.float64 else DTYPE_FLOAT
    a = np.ascontiguousarray(a)
    b2 = np.ascontiguousarray(b.reshape(b.shape[0], -1))
    c = np.zeros((a.shape[0], b2.shape[1]), a.dtype)
    LIB.ora_dense_gemm(dt, a.shape[0], b2.shape[1], a.shape[1], _ptr(a), _ptr(b2), _ptr(c))
    return c.reshape((a.shape[0],) + b.shape[1:])


def dd_rows(a: np.ndarray, b: np.ndarray, rows, nthreads: int | None = None):
    """Rows of A*B in double-double; returns (hi, lo) arrays of shape (len(rows), N)."""
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    rows = np.ascontiguousarray(rows, np.int64)
    n = b.shape[1]
    hi = np.zeros((len(rows), n))
    lo = np.zeros((len(rows), n))
    LIB.ora_dd_rows(_ptr(a), _ptr(b), a.shape[0], n, a.shape[1], _ptr(rows), len(rows),
                    _ptr(hi), _ptr(lo), nthreads or (os.cpu_count() or 1))
    return hi, lo


def normwise_error(c: np.ndarray, hi: np.ndarray, lo: np.ndarray, rows) -> float:
    """||C[rows] - C*||_F / ||C*||_F with C* = hi + lo (double-double)."""
    d = (c[rows].astype(np.float64) - hi) - lo
    return float(np.linalg.norm(d) / np.linalg.norm(hi))


# ----------------------------------------------------------------------------- frames
def _mp_int(buf, p):
    t = buf[p]
    if t < 0x80:
        return t, p + 1
    fmt = {0xcc: ">B", 0xcd: ">H", 0xce: ">I", 0xcf: ">Q", 0xd0: ">b", 0xd1: ">h", 0xd2: ">i", 0xd3: ">q"}[t]
    v = struct.unpack_from(fmt, buf, p + 1)[0]
    return v, p + 1 + struct.calcsize(fmt)


def read_frame(buf: bytes) -> dict:
    """Parse a Blosc2 contiguous frame: header fields, metalayers, chunks (in logical order)."""
    assert buf[0] == 0x9e and buf[1:10] == b"\xa8b2frame\x00", "not a blosc2 frame"
    header_size = struct.unpack_from(">i", buf, 11)[0]
    frame_size = struct.unpack_from(">Q", buf, 16)[0]
    flags = buf[25:29]
    nbytes = struct.unpack_from(">q", buf, 30)[0]
    cbytes = struct.unpack_from(">q", buf, 39)[0]
    typesize = struct.unpack_from(">i", buf, 48)[0]
    blocksize = struct.unpack_from(">i", buf, 53)[0]
    chunksize = struct.unpack_from(">i", buf, 58)[0]
    metas = {}
    p = 87
    assert buf[p] == 0x93
    p += 1
    _, p = _mp_int(buf, p)
    assert buf[p] == 0xde
    nmeta = struct.unpack_from(">H", buf, p + 1)[0]
    p += 3
    names = []
    for _ in range(nmeta):
        ln = buf[p] & 0x1f
        names.append(buf[p + 1:p + 1 + ln].decode())
        p += 1 + ln
        _, p = _mp_int(buf, p)
    assert buf[p] == 0xdc
    p += 3
    for nm in names:
        assert buf[p] == 0xc6
        ln = struct.unpack_from(">I", buf, p + 1)[0]
        metas[nm] = buf[p + 5:p + 5 + ln]
        p += 5 + ln
    # offsets chunk: the last chunk before the trailer; find it by walking data chunks
    nchunks = -(-nbytes // chunksize) if chunksize else 0
    pos = header_size
    for _ in range(nchunks):
        pos += struct.unpack_from("<i", buf, pos + 12)[0]
    off_chunk = buf[pos:pos + struct.unpack_from("<i", buf, pos + 12)[0]]
    offsets = np.frombuffer(chunk_decompress(off_chunk), np.int64)
    chunks = []
    for o in offsets:
        s = header_size + int(o)
        cb = struct.unpack_from("<i", buf, s + 12)[0]
        chunks.append(buf[s:s + cb])
    return dict(header_size=header_size, frame_size=frame_size, flags=flags, nbytes=nbytes,
                cbytes=cbytes, typesize=typesize, blocksize=blocksize, chunksize=chunksize,
                metalayers=metas, chunks=chunks, offsets=offsets)


def parse_caterva_meta(m: bytes):
    """[version, ndim, shape[int64], chunkshape[int32], blockshape[int32]]."""
    assert m[0] == 0x95
    ndim = m[2]
    p = 3

    def arr(p, code, fmt):
        assert m[p] == 0x90 + ndim
        p += 1
        vals = []
        for _ in range(ndim):
            assert m[p] == code
            vals.append(struct.unpack_from(fmt, m, p + 1)[0])
            p += 1 + struct.calcsize(fmt)
        return vals, p
    shape, p = arr(p, 0xd3, ">q")
    chunk, p = arr(p, 0xd2, ">i")
    block, p = arr(p, 0xd2, ">i")
    return ndim, shape, chunk, block


# ----------------------------------------------------------------------------- CPU baseline
def openblas_dgemm():
    """Address of OpenBLAS's cblas_dgemm (scipy's bundled copy), pinned to one thread,
    or None.  The reference calls MKL's cblas_dgemm with MKL pinned to one thread."""
    import glob
    try:
        import scipy
    except ImportError:
        return None
    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "libscipy_openblas*.so"))
    if not libs:
        return None
    lib = ctypes.CDLL(libs[0])
    try:
        lib.scipy_openblas_set_num_threads(1)
    except AttributeError:
        pass
    return ctypes.cast(lib.scipy_cblas_dgemm, ctypes.c_void_p).value, lib


def liblz4_decompress():
    try:
        lib = ctypes.CDLL("liblz4.so.1")
        return ctypes.cast(lib.LZ4_decompress_safe, ctypes.c_void_p).value, lib
    except OSError:
        return None


LIB.ora_cpu_opt_gemm_chunk.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


def cpu_opt_gemm_chunk(ga: Geom, a_chunks, gb: Geom, b_chunks, gc: Geom, cn: int, nthreads: int):
    """One output chunk of iarray_opt_gemm computed by the reference's loop on host cores
    (per-pair block decode, single-threaded OpenBLAS dgemm, Blosc2 re-encode).
    Returns the compressed chunk."""
    bl = openblas_dgemm()
    if bl is None:
        raise RuntimeError("no cblas_dgemm available for the CPU baseline")
    dec = liblz4_decompress()
    sa, sb = _schunk(ga, a_chunks), _schunk(gb, b_chunks)
    cg = gc.cstruct()
    out = ctypes.create_string_buffer(gc.chunk_nbytes + 64)
    r = LIB.ora_cpu_opt_gemm_chunk(ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(cg), cn, nthreads,
                                   bl[0], dec[0] if dec else None, out)
    if r < 0:
        raise RuntimeError(f"cpu baseline failed ({r})")
    return out.raw[:r]


LIB.ora_cpu_opt_gemm.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


def cpu_opt_gemm(ga: Geom, a_chunks, gb: Geom, b_chunks, gc: Geom, nthreads: int):
    """The whole iarray_opt_gemm product by the reference's loop on host cores
    (src/linalg/iarray_gemm.c:399-425: output chunk after output chunk, each one's blocks
    computed by `nthreads` workers with per-pair block decode and single-threaded OpenBLAS
    dgemm, each block compressed by its worker).  Returns the compressed output chunks."""
    bl = openblas_dgemm()
    if bl is None:
        raise RuntimeError("no cblas_dgemm available for the CPU baseline")
    dec = liblz4_decompress()
    sa, sb = _schunk(ga, a_chunks), _schunk(gb, b_chunks)
    cg = gc.cstruct()
    outs = [ctypes.create_string_buffer(gc.chunk_nbytes + 64) for _ in range(gc.nchunks)]
    ptrs = (ctypes.c_void_p * gc.nchunks)(*[ctypes.cast(o, ctypes.c_void_p) for o in outs])
    lens = (ctypes.c_int32 * gc.nchunks)()
    r = LIB.ora_cpu_opt_gemm(ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(cg), nthreads, bl[0],
                             dec[0] if dec else None, ptrs, lens)
    if r < 0:
        raise RuntimeError(f"cpu baseline failed ({r})")
    return [outs[i].raw[:lens[i]] for i in range(gc.nchunks)]
