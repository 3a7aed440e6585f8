"""ctypes binding of libiarray_b200.so (include/iarray_b200.h).

This is the Python-side stub a maintainer would add to bind the C ABI: it mirrors the
reference's C types (include/libiarray/iarray.h:214-240) and exposes each entry point
with the reference's argument meaning.  Containers stay on the GPU; numpy arrays cross
the boundary only through iarray_from_buffer / iarray_to_buffer.

The library has no CPU fallback: on a machine without a usable GPU, `init()` raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libiarray_b200.so")

DTYPE_DOUBLE, DTYPE_FLOAT = 0, 1
NP_DTYPE = {DTYPE_DOUBLE: np.float64, DTYPE_FLOAT: np.float32, 10: np.int64, 11: np.int32, 12: np.int16,
            13: np.int8, 16: np.uint64, 17: np.uint32, 18: np.uint16, 19: np.uint8}
IA_DTYPE = {np.dtype(v): k for k, v in NP_DTYPE.items()}
FORM_NATIVE, FORM_SPLIT = 0, 1
ENCODER_PARALLEL, ENCODER_LIBLZ4 = 0, 1
ALWAYS_SPLIT, NEVER_SPLIT, AUTO_SPLIT = 1, 2, 3

RC_ERROR_BIT = 1 << 63


def _code(c):
    return c << 16


NEGATE = 1 << 15
ES = 1024
ERR = {
    "INVALID_DTYPE": _code(1) | (ES + 6),
    "INVALID_SHAPE": _code(1) | (ES + 3),
    "INVALID_CHUNKSHAPE": _code(1) | (ES + 4),
    "INVALID_BLOCKSHAPE": _code(1) | (ES + 13),
    "INVALID_NDIM": _code(1) | (ES + 5),
    "INVALID_STORAGE": _code(1) | (ES + 7),
    "TOO_SMALL_BUFFER": _code(5) | (ES + 9),
    "BLOSC_FAILED": _code(2) | (ES + 11),
    "ASSERTION_FAILED": _code(2) | (ES + 12),
    "PERSISTENCY_FAILED": _code(2) | (ES + 8),
    "GPU_FAILED": _code(2) | (ES + 100),
    "GPU_OUT_OF_MEMORY": _code(9) | (ES + 100),
    "NOT_SUPPORTED": (_code(10) | NEGATE) | (ES + 1),
    "INVALID_ARGUMENT": _code(1) | 1,
    "NOT_INITIALIZED": (_code(11) | NEGATE),
    "NOALLOC_TOO_LARGE": _code(6) | (ES + 9),
}
ERR_NAME = {v: k for k, v in ERR.items()}


class Config(ctypes.Structure):
    _fields_ = [("compression_codec", ctypes.c_int), ("compression_level", ctypes.c_int),
                ("compression_favor", ctypes.c_int), ("use_dict", ctypes.c_int), ("splitmode", ctypes.c_int),
                ("filter_flags", ctypes.c_int), ("eval_method", ctypes.c_uint), ("max_num_threads", ctypes.c_int),
                ("fp_mantissa_bits", ctypes.c_uint8), ("btune", ctypes.c_bool), ("compression_meta", ctypes.c_uint8)]

    @classmethod
    def defaults(cls):
        # IARRAY_CONFIG_DEFAULTS (include/libiarray/iarray.h:275-287)
        return cls(1, 5, 0, 0, AUTO_SPLIT, 1, 2, 1, 0, True, 0)


class DtShape(ctypes.Structure):
    _fields_ = [("dtype", ctypes.c_int), ("dtype_size", ctypes.c_int32), ("ndim", ctypes.c_int8),
                ("shape", ctypes.c_int64 * 8)]


class Storage(ctypes.Structure):
    _fields_ = [("urlpath", ctypes.c_char_p), ("contiguous", ctypes.c_bool), ("chunkshape", ctypes.c_int64 * 8),
                ("blockshape", ctypes.c_int64 * 8)]


class IArrayError(RuntimeError):
    def __init__(self, rc, where):
        self.rc = rc
        self.msg = rc & 0xFFFFFF
        self.name = ERR_NAME.get(self.msg, hex(self.msg))
        super().__init__(f"{where}: {self.name} ({_lib().iarray_err_strerror(rc).decode()})")


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not built (run make -C iron-array_b200)")
        L = ctypes.CDLL(LIB_PATH)
        P, I64, RC = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64
        sig = {
            "iarray_init": ([], RC), "iarray_destroy": ([], None), "iarray_err_strerror": ([RC], ctypes.c_char_p),
            "iarray_context_new": ([P, P], RC), "iarray_context_free": ([P], None),
            "iarray_empty": ([P, P, P, P], RC), "iarray_zeros": ([P, P, P, P], RC),
            "iarray_arange": ([P, P, ctypes.c_double, ctypes.c_double, P, P], RC),
            "iarray_linspace": ([P, P, ctypes.c_double, ctypes.c_double, P, P], RC),
            "iarray_from_buffer": ([P, P, P, I64, P, P], RC), "iarray_to_buffer": ([P, P, P, I64], RC),
            "iarray_container_info": ([P, P, P], RC), "iarray_container_free": ([P, P], None),
            "iarray_get_dtshape": ([P, P, P], RC), "iarray_get_storage": ([P, P, P], RC),
            "iarray_is_view": ([P, P, P], RC), "iarray_container_almost_equal": ([P, P, ctypes.c_double], RC),
            "iarray_container_save": ([P, P, ctypes.c_char_p], RC),
            "iarray_container_open": ([P, ctypes.c_char_p, P], RC),
            "iarray_container_load": ([P, ctypes.c_char_p, P], RC),
            "iarray_container_remove": ([ctypes.c_char_p], RC),
            "iarray_expr_new": ([P, ctypes.c_int, P], RC), "iarray_expr_free": ([P, P], None),
            "iarray_expr_bind": ([P, ctypes.c_char_p, P], RC),
            "iarray_b200_expr_bind_matmul": ([P, ctypes.c_char_p, P, P], RC),
            "iarray_expr_bind_out_properties": ([P, P, P], RC),
            "iarray_expr_bind_scalar_double": ([P, ctypes.c_char_p, ctypes.c_double], RC),
            "iarray_expr_bind_scalar_float": ([P, ctypes.c_char_p, ctypes.c_float], RC),
            "iarray_expr_compile": ([P, ctypes.c_char_p], RC), "iarray_eval": ([P, P], RC),
            "iarray_expr_compile_udf": ([P, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p], RC),
            "iarray_to_cframe": ([P, P, P, P, P], RC), "iarray_from_cframe": ([P, P, I64, ctypes.c_bool, P], RC),
            "iarray_linalg_matmul": ([P, P, P, P, P], RC), "iarray_linalg_transpose": ([P, P, P], RC),
            "iarray_gemm": ([P, P, P, P], RC), "iarray_gemv": ([P, P, P, P], RC),
            "iarray_opt_gemm": ([P, P, P, P, P], RC), "iarray_opt_gemm_a": ([P, P, P, P, P], RC),
            "iarray_opt_gemm_b": ([P, P, P, P, P], RC), "iarray_opt_gemv": ([P, P, P, P, P], RC),
            "iarray_b200_set_form": ([P, ctypes.c_int], RC), "iarray_b200_set_encoder": ([P, ctypes.c_int], RC), "iarray_b200_set_split_terms": ([P, ctypes.c_int], RC),
            "iarray_b200_set_split_products_f32": ([P, ctypes.c_int], RC),
            "iarray_b200_last_timings": ([P, P], RC),
            "iarray_b200_from_chunks": ([P, P, P, I64, P, P, P], RC),
            "iarray_b200_get_chunk": ([P, P, I64, P, P], RC), "iarray_b200_nchunks": ([P, P], RC),
            "iarray_b200_decode_to_device": ([P, P, P, I64], RC),
            "iarray_b200_encode_from_device": ([P, P, P, I64, P, P], RC),
            "iarray_b200_dense_gemm": ([P, ctypes.c_int, I64, I64, I64, P, I64, P, I64, P, I64], RC),
            "iarray_b200_opt_gemm_cframes": ([P, P, I64, P, I64, P, P, I64, P], RC),
            "iarray_b200_synchronize": ([P], RC),
            "iarray_b200_kernel_launches": ([], ctypes.c_uint64),
            "iarray_b200_get_stream": ([P, P], RC),
            "iarray_b200_to_cframe_into": ([P, P, P, I64, P], RC),
            "iarray_b200_profile_kernels": ([ctypes.c_int], RC),
            "iarray_b200_batch_new": ([P, I64, P, P, P, P], RC),
            "iarray_b200_batch_run": ([P, P], RC),
            "iarray_b200_batch_info": ([P, P, P, P], RC),
            "iarray_b200_batch_split_tuning": ([P, P, P, P, P], RC),
            "iarray_b200_batch_free": ([P], None),
            "iarray_b200_kernel_profile": ([P, I64, P], RC),
            "iarray_b200_decode_noalloc": ([ctypes.c_int8, P, P, P, ctypes.c_int32, P, I64, P, I64, P], RC),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
    return _LIB


def lib():
    return _lib()


def profile_kernels(on):
    """Start (clearing the totals) or stop per-kernel CUDA-event timing."""
    check(_lib().iarray_b200_profile_kernels(1 if on else 0), "profile_kernels")


def kernel_profile():
    """{kernel name: (launches, total device ms)} since profiling was last started."""
    n = ctypes.c_int64()
    check(_lib().iarray_b200_kernel_profile(None, 0, ctypes.byref(n)), "kernel_profile")
    buf = ctypes.create_string_buffer(n.value + 1)
    check(_lib().iarray_b200_kernel_profile(buf, n.value + 1, ctypes.byref(n)), "kernel_profile")
    out = {}
    for ln in buf.value.decode().splitlines():
        name, cnt, ms = ln.split()
        out[name] = (int(cnt), float(ms))
    return out


def check(rc, where=""):
    if rc & RC_ERROR_BIT:
        raise IArrayError(rc, where)
    return rc


_initialized = False


def init():
    global _initialized
    if not _initialized:
        check(_lib().iarray_init(), "iarray_init")
        _initialized = True


def dtshape(shape, dtype):
    d = DtShape()
    d.dtype = IA_DTYPE[np.dtype(dtype)]
    d.ndim = len(shape)
    for i, s in enumerate(shape):
        d.shape[i] = s
    return d


def storage(chunkshape, blockshape, urlpath=None, contiguous=True):
    s = Storage()
    s.urlpath = urlpath.encode() if urlpath else None
    s.contiguous = contiguous
    for i, (c, b) in enumerate(zip(chunkshape, blockshape)):
        s.chunkshape[i] = c
        s.blockshape[i] = b
    return s


class Context:
    def __init__(self, cfg: Config | None = None, form: int = FORM_NATIVE, split_terms: int = 0,
                 encoder: int = ENCODER_LIBLZ4):
        init()
        self.cfg = cfg or Config.defaults()
        self.ptr = ctypes.c_void_p()
        check(_lib().iarray_context_new(ctypes.byref(self.cfg), ctypes.byref(self.ptr)), "iarray_context_new")
        self.set_form(form, split_terms)
        self.set_encoder(encoder)

    def set_encoder(self, encoder):
        check(_lib().iarray_b200_set_encoder(self.ptr, encoder), "set_encoder")

    def set_form(self, form, split_terms=0):
        check(_lib().iarray_b200_set_form(self.ptr, form), "set_form")
        check(_lib().iarray_b200_set_split_terms(self.ptr, split_terms), "set_split_terms")

    def set_split_products_f32(self, nproducts):
        """BF16 products of the float32 split form: 6 (three-word split), 3 (two-word
        split, "3xBF16"), 0 (automatic: 6)."""
        check(_lib().iarray_b200_set_split_products_f32(self.ptr, nproducts), "set_split_products_f32")

    def timings(self):
        t = (ctypes.c_double * 5)()
        check(_lib().iarray_b200_last_timings(self.ptr, t))
        return dict(decode_a=t[0], decode_b=t[1], product=t[2], encode=t[3], total=t[4])

    def stream(self) -> int:
        """The context's cudaStream_t handle (as an integer)."""
        s = ctypes.c_void_p()
        check(_lib().iarray_b200_get_stream(self.ptr, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self):
        check(_lib().iarray_b200_synchronize(self.ptr), "synchronize")

    def close(self):
        if self.ptr:
            _lib().iarray_context_free(ctypes.byref(self.ptr))
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Container:
    def __init__(self, ctx: Context, ptr: ctypes.c_void_p):
        self.ctx = ctx
        self.ptr = ptr

    # ------------------------------------------------------------------ constructors
    @classmethod
    def from_numpy(cls, ctx, arr, chunkshape, blockshape, urlpath=None, contiguous=True):
        """With `urlpath` the container is also written to disk: a contiguous frame file, or
        (contiguous=False) a sparse frame directory."""
        arr = np.ascontiguousarray(arr)
        d = dtshape(arr.shape, arr.dtype)
        s = storage(chunkshape, blockshape, urlpath, contiguous)
        p = ctypes.c_void_p()
        check(_lib().iarray_from_buffer(ctx.ptr, ctypes.byref(d), arr.ctypes.data, arr.nbytes, ctypes.byref(s),
                                        ctypes.byref(p)), "iarray_from_buffer")
        return cls(ctx, p)

    @classmethod
    def arange(cls, ctx, shape, dtype, start, step, chunkshape, blockshape):
        d, s, p = dtshape(shape, dtype), storage(chunkshape, blockshape), ctypes.c_void_p()
        check(_lib().iarray_arange(ctx.ptr, ctypes.byref(d), start, step, ctypes.byref(s), ctypes.byref(p)),
              "iarray_arange")
        return cls(ctx, p)

    @classmethod
    def linspace(cls, ctx, shape, dtype, start, stop, chunkshape, blockshape):
        d, s, p = dtshape(shape, dtype), storage(chunkshape, blockshape), ctypes.c_void_p()
        check(_lib().iarray_linspace(ctx.ptr, ctypes.byref(d), start, stop, ctypes.byref(s), ctypes.byref(p)),
              "iarray_linspace")
        return cls(ctx, p)

    @classmethod
    def empty(cls, ctx, shape, dtype, chunkshape, blockshape):
        d, s, p = dtshape(shape, dtype), storage(chunkshape, blockshape), ctypes.c_void_p()
        check(_lib().iarray_empty(ctx.ptr, ctypes.byref(d), ctypes.byref(s), ctypes.byref(p)), "iarray_empty")
        return cls(ctx, p)

    @classmethod
    def from_chunks(cls, ctx, shape, dtype, chunkshape, blockshape, chunks):
        d, s, p = dtshape(shape, dtype), storage(chunkshape, blockshape), ctypes.c_void_p()
        bufs = [ctypes.create_string_buffer(bytes(c), len(c)) for c in chunks]
        ptrs = (ctypes.c_void_p * len(chunks))(*[ctypes.cast(b, ctypes.c_void_p) for b in bufs])
        lens = (ctypes.c_int64 * len(chunks))(*[len(c) for c in chunks])
        check(_lib().iarray_b200_from_chunks(ctx.ptr, ctypes.byref(d), ctypes.byref(s), len(chunks), ptrs, lens,
                                             ctypes.byref(p)), "iarray_b200_from_chunks")
        return cls(ctx, p)

    @classmethod
    def from_cframe(cls, ctx, frame):
        """frame: bytes, or a numpy uint8 array (e.g. in pinned memory); not copied."""
        if isinstance(frame, np.ndarray):
            ptr, n = frame.ctypes.data, frame.nbytes
        else:
            ptr, n = ctypes.cast(ctypes.c_char_p(frame), ctypes.c_void_p), len(frame)
        p = ctypes.c_void_p()
        check(_lib().iarray_from_cframe(ctx.ptr, ptr, n, True, ctypes.byref(p)), "iarray_from_cframe")
        return cls(ctx, p)

    @classmethod
    def open(cls, ctx, path, load=False):
        p = ctypes.c_void_p()
        fn = _lib().iarray_container_load if load else _lib().iarray_container_open
        check(fn(ctx.ptr, path.encode(), ctypes.byref(p)), "iarray_container_open")
        return cls(ctx, p)

    @staticmethod
    def remove(path):
        """iarray_container_remove: a frame file, or a sparse frame directory."""
        check(_lib().iarray_container_remove(path.encode()), "iarray_container_remove")

    # ------------------------------------------------------------------ accessors
    def decode_to_device(self, dptr, ld):
        """Decode into device memory at `dptr` (row-major, leading dimension `ld` items)
        on the context's stream."""
        check(_lib().iarray_b200_decode_to_device(self.ctx.ptr, self.ptr, dptr, ld), "decode_to_device")

    def dtshape(self):
        d = DtShape()
        check(_lib().iarray_get_dtshape(self.ctx.ptr, self.ptr, ctypes.byref(d)))
        return d

    @property
    def shape(self):
        d = self.dtshape()
        return tuple(d.shape[i] for i in range(d.ndim))

    @property
    def dtype(self):
        return np.dtype(NP_DTYPE[self.dtshape().dtype])

    def to_numpy(self):
        out = np.empty(self.shape, self.dtype)
        check(_lib().iarray_to_buffer(self.ctx.ptr, self.ptr, out.ctypes.data, out.nbytes), "iarray_to_buffer")
        return out

    def info(self):
        nb, cb = ctypes.c_int64(), ctypes.c_int64()
        check(_lib().iarray_container_info(self.ptr, ctypes.byref(nb), ctypes.byref(cb)))
        return nb.value, cb.value

    def nchunks(self):
        n = ctypes.c_int64()
        check(_lib().iarray_b200_nchunks(self.ptr, ctypes.byref(n)))
        return n.value

    def chunk(self, n) -> bytes:
        ln = ctypes.c_int64()
        check(_lib().iarray_b200_get_chunk(self.ctx.ptr, self.ptr, n, None, ctypes.byref(ln)))
        buf = ctypes.create_string_buffer(ln.value)
        check(_lib().iarray_b200_get_chunk(self.ctx.ptr, self.ptr, n, buf, ctypes.byref(ln)), "get_chunk")
        return buf.raw[:ln.value]

    def chunks(self):
        return [self.chunk(i) for i in range(self.nchunks())]

    def to_cframe(self) -> bytes:
        fp, ln, nf = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_int64(), ctypes.c_bool()
        check(_lib().iarray_to_cframe(self.ctx.ptr, self.ptr, ctypes.byref(fp), ctypes.byref(ln), ctypes.byref(nf)),
              "iarray_to_cframe")
        data = ctypes.string_at(fp, ln.value)
        if nf.value:
            ctypes.CDLL(None).free(fp)
        return data

    def cframe_len(self) -> int:
        n = ctypes.c_int64()
        check(_lib().iarray_b200_to_cframe_into(self.ctx.ptr, self.ptr, None, 0, ctypes.byref(n)))
        return n.value

    def to_cframe_into(self, buf: np.ndarray) -> int:
        """Write the frame into a caller numpy uint8 buffer; returns its length."""
        n = ctypes.c_int64()
        check(_lib().iarray_b200_to_cframe_into(self.ctx.ptr, self.ptr, buf.ctypes.data, buf.nbytes, ctypes.byref(n)),
              "iarray_b200_to_cframe_into")
        return n.value

    def save(self, path):
        check(_lib().iarray_container_save(self.ctx.ptr, self.ptr, path.encode()), "iarray_container_save")

    def transpose(self):
        p = ctypes.c_void_p()
        check(_lib().iarray_linalg_transpose(self.ctx.ptr, self.ptr, ctypes.byref(p)), "iarray_linalg_transpose")
        return Container(self.ctx, p)

    def free(self):
        if self.ptr:
            _lib().iarray_container_free(self.ctx.ptr, ctypes.byref(self.ptr))
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _product(fn, name, ctx, a, b, chunkshape, blockshape, urlpath=None, contiguous=True):
    s = storage(chunkshape, blockshape, urlpath, contiguous)
    p = ctypes.c_void_p()
    check(fn(ctx.ptr, a.ptr, b.ptr, ctypes.byref(s), ctypes.byref(p)), name)
    return Container(ctx, p)


def matmul(ctx, a, b, chunkshape, blockshape, urlpath=None, contiguous=True):
    return _product(_lib().iarray_linalg_matmul, "iarray_linalg_matmul", ctx, a, b, chunkshape, blockshape, urlpath,
                    contiguous)


def opt_gemm(ctx, a, b, chunkshape, blockshape):
    return _product(_lib().iarray_opt_gemm, "iarray_opt_gemm", ctx, a, b, chunkshape, blockshape)


def opt_gemm_cframes(ctx, a_frame, b_frame, chunkshape, blockshape, out=None):
    """iarray_b200_opt_gemm_cframes: A and B as contiguous frames in host memory (bytes or
    uint8 numpy arrays, ideally pinned), C's frame written into `out` (a uint8 numpy array;
    allocated with the documented upper bound when None).  Returns (out, frame length)."""
    def buf(x):
        if isinstance(x, np.ndarray):
            return x.ctypes.data_as(ctypes.c_void_p), x.nbytes
        b = ctypes.create_string_buffer(bytes(x), len(x))
        return ctypes.cast(b, ctypes.c_void_p), len(x), b
    pa, pb = buf(a_frame), buf(b_frame)
    s = storage(chunkshape, blockshape)
    n = ctypes.c_int64()
    if out is None:
        hdr = read_frame_shapes(a_frame, b_frame)
        out = np.empty(hdr, np.uint8)
    check(_lib().iarray_b200_opt_gemm_cframes(ctx.ptr, pa[0], pa[1], pb[0], pb[1], ctypes.byref(s),
                                              out.ctypes.data_as(ctypes.c_void_p), out.nbytes, ctypes.byref(n)),
          "iarray_b200_opt_gemm_cframes")
    return out, n.value


def read_frame_shapes(a_frame, b_frame):
    """Upper bound of the C frame size for two operand frames (their containers' shapes)."""
    ctx = Context()
    a = Container.from_cframe(ctx, bytes(a_frame))
    b = Container.from_cframe(ctx, bytes(b_frame))
    (m, _), (_, n) = a.shape, b.shape
    isz = np.dtype(a.dtype).itemsize
    return m * n * isz * 2 + 64 * 1024 + (1 << 20)


def opt_gemm_a(ctx, a, b, chunkshape, blockshape):
    return _product(_lib().iarray_opt_gemm_a, "iarray_opt_gemm_a", ctx, a, b, chunkshape, blockshape)


def opt_gemm_b(ctx, a, b, chunkshape, blockshape):
    return _product(_lib().iarray_opt_gemm_b, "iarray_opt_gemm_b", ctx, a, b, chunkshape, blockshape)


def opt_gemv(ctx, a, b, chunkshape, blockshape):
    return _product(_lib().iarray_opt_gemv, "iarray_opt_gemv", ctx, a, b, chunkshape, blockshape)


class Batch:
    """Batched float64 products C_i = A_i * B_i (iarray_b200_batch_*): built once (autotuned
    grouped product, captured CUDA graph), run any number of times."""

    def __init__(self, ctx, As, Bs, chunkshapes, blockshapes):
        n = len(As)
        self.ctx, self.n = ctx, n
        self._keep = (list(As), list(Bs))
        a = (ctypes.c_void_p * n)(*[x.ptr for x in As])
        b = (ctypes.c_void_p * n)(*[x.ptr for x in Bs])
        st = (Storage * n)()
        for i in range(n):
            st[i] = storage(chunkshapes[i], blockshapes[i])
        self.ptr = ctypes.c_void_p()
        check(_lib().iarray_b200_batch_new(ctx.ptr, n, a, b, st, ctypes.byref(self.ptr)), "iarray_b200_batch_new")

    def run(self):
        out = (ctypes.c_void_p * self.n)()
        check(_lib().iarray_b200_batch_run(self.ptr, out), "iarray_b200_batch_run")
        return [Container(self.ctx, ctypes.c_void_p(out[i])) for i in range(self.n)]

    def info(self):
        cfg = ctypes.c_int()
        ms = (ctypes.c_double * 8)()             # IARRAY_B200_BATCH_TILE_CONFIGS
        nodes = ctypes.c_int64()
        check(_lib().iarray_b200_batch_info(self.ptr, ctypes.byref(cfg), ms, ctypes.byref(nodes)))
        return {"tile_config": cfg.value, "tune_ms": list(ms), "graph_nodes": nodes.value}

    def split_tuning(self):
        """Moduli count of a split-form batch, the native product's error (the bar's base) and
        the tuner's time and error for 16, 15, 14, 13, 12 moduli."""
        n, en = ctypes.c_int(), ctypes.c_double()
        ms, err = (ctypes.c_double * 5)(), (ctypes.c_double * 5)()
        check(_lib().iarray_b200_batch_split_tuning(self.ptr, ctypes.byref(n), ctypes.byref(en), ms, err),
              "batch_split_tuning")
        return {"nterms": n.value, "err_native": en.value, "tune_ms": list(ms), "tune_err": list(err)}

    def free(self):
        if self.ptr:
            _lib().iarray_b200_batch_free(ctypes.byref(self.ptr))
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def almost_equal(a, b, tol):
    return _lib().iarray_container_almost_equal(a.ptr, b.ptr, tol)


class Expression:
    """iarray_expr_* / iarray_eval: an element-wise expression over containers of the output's
    shape, evaluated on the GPU; bind_matmul feeds a matrix product in as an operand."""

    def __init__(self, ctx, dtype=np.float64):
        self.ctx = ctx
        self.ptr = ctypes.c_void_p()
        check(_lib().iarray_expr_new(ctx.ptr, IA_DTYPE[np.dtype(dtype)], ctypes.byref(self.ptr)), "iarray_expr_new")

    def bind(self, var, container):
        check(_lib().iarray_expr_bind(self.ptr, var.encode(), container.ptr), "iarray_expr_bind")

    def bind_matmul(self, var, a, b):
        check(_lib().iarray_b200_expr_bind_matmul(self.ptr, var.encode(), a.ptr, b.ptr), "iarray_b200_expr_bind_matmul")

    def bind_scalar(self, var, value, single=False):
        fn = _lib().iarray_expr_bind_scalar_float if single else _lib().iarray_expr_bind_scalar_double
        check(fn(self.ptr, var.encode(), value), "iarray_expr_bind_scalar")

    def bind_out(self, shape, dtype, chunkshape, blockshape, urlpath=None, contiguous=True):
        d = dtshape(shape, dtype)
        s = storage(chunkshape, blockshape, urlpath, contiguous)
        check(_lib().iarray_expr_bind_out_properties(self.ptr, ctypes.byref(d), ctypes.byref(s)),
              "iarray_expr_bind_out_properties")

    def compile(self, text):
        check(_lib().iarray_expr_compile(self.ptr, text.encode()), "iarray_expr_compile")

    def eval(self):
        p = ctypes.c_void_p()
        check(_lib().iarray_eval(self.ptr, ctypes.byref(p)), "iarray_eval")
        return Container(self.ctx, p)

    def free(self):
        if self.ptr:
            _lib().iarray_expr_free(self.ctx.ptr, ctypes.byref(self.ptr))
            self.ptr = ctypes.c_void_p()
