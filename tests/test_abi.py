"""CPU checks of the C-ABI library: it loads, exports every entry point the public
header declares, and fails loudly (no CPU fallback) when no GPU is usable."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "iarray_b200.h")
LIB = os.path.join(ROOT, "iron-array_b200", "lib", "libiarray_b200.so")


def declared_functions():
    text = "\n".join(ln for ln in open(HEADER).read().splitlines() if not ln.lstrip().startswith("#"))
    return re.findall(r"INA_API\([^)]*\)\s*(\w+)\s*\(", text)


def test_header_declares_reference_entry_points():
    names = set(declared_functions())
    for ref in ["iarray_linalg_matmul", "iarray_opt_gemm", "iarray_opt_gemm_a", "iarray_opt_gemm_b",
                "iarray_opt_gemv", "iarray_gemm", "iarray_gemv", "iarray_init", "iarray_destroy",
                "iarray_context_new", "iarray_context_free", "iarray_from_buffer", "iarray_to_buffer",
                "iarray_empty", "iarray_container_free", "iarray_container_info", "iarray_container_save",
                "iarray_container_open", "iarray_container_load", "iarray_to_cframe", "iarray_from_cframe",
                "iarray_linalg_transpose", "iarray_err_strerror"]:
        assert ref in names, ref


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_only_declared_symbols_are_exported():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    ours = {n for n in exported if n.startswith("iarray_")}
    assert ours == set(declared_functions())


def test_header_constants_match_the_binding():
    """The binding's fixed-size buffers follow the header's constants."""
    text = open(HEADER).read()
    configs = int(re.search(r"#define IARRAY_B200_BATCH_TILE_CONFIGS (\d+)", text).group(1))
    src = open(os.path.join(ROOT, "iron-array_b200", "iarray_b200.py")).read()
    assert f"ms = (ctypes.c_double * {configs})()" in src
    assert configs == 8


def test_error_strings(ia=None):
    import iarray_b200 as m
    lib = m.lib()
    assert lib.iarray_err_strerror(0) == b"Success"
    assert b"GPU" in lib.iarray_err_strerror(m.RC_ERROR_BIT | m.ERR["GPU_FAILED"])
    assert b"chunkshape" in lib.iarray_err_strerror(m.RC_ERROR_BIT | m.ERR["INVALID_CHUNKSHAPE"])


def test_context_requires_init():
    import iarray_b200 as m
    if m._initialized:
        pytest.skip("library already initialised in this process")
    cfg = m.Config.defaults()
    p = ctypes.c_void_p()
    rc = m.lib().iarray_context_new(ctypes.byref(cfg), ctypes.byref(p))
    assert rc & m.RC_ERROR_BIT and (rc & 0xFFFFFF) == m.ERR["NOT_INITIALIZED"]


@pytest.mark.skipif(gpu_available(), reason="a GPU is present")
def test_init_fails_loudly_without_gpu():
    import iarray_b200 as m
    rc = m.lib().iarray_init()
    assert rc & m.RC_ERROR_BIT and (rc & 0xFFFFFF) == m.ERR["GPU_FAILED"]
    with pytest.raises(m.IArrayError):
        m.init()
