"""The C ABI library loads and exports every entry point include/hulkcuda.h
declares; calls that need no GPU behave (no compute is run here)."""
import ctypes as C
import subprocess

import pytest

from hulktracer_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    syms = _lib.exported_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(syms) <= exported


def test_status_codes_match_reference_enum():
    # EHulkResult, HulkEngine/public/hulk_assert.h:42-50
    assert [_lib.STATUS_NAMES[i] for i in range(6)] == ["HK_OK", "HK_E_ALLOC", "HK_E_FILE_OPEN", "HK_E_FILE_CLOSE",
                                                      "HK_E_ILLEGAL_INPUT", "HK_E_NODE_NOT_FOUND"]


def test_config_default():
    L = _lib.load()
    c = _lib.Config()
    assert L.hk_config_default(C.byref(c)) == 0
    assert (c.traverse_cost, c.intersect_cost, c.max_depth, c.leaf_size, c.bins) == (1.0, 1.5, 24, 4, 32)
    assert L.hk_config_default(None) == 4


def test_null_arguments_rejected():
    L = _lib.load()
    assert L.hk_create(None, None) == 4
    assert L.hk_destroy(None) == 4
    assert L.hk_trace(None, None, 0, 0, None) == 4


@pytest.mark.parametrize("block,ok", [(256, True), (288, False), (512, False), (1024, False), (48, False)])
def test_block_size_beyond_the_launch_bound_rejected(block, ok):
    """The trace kernel is compiled for at most 256 threads per block; a
    larger block_size is refused when the context is created (HK_E_ILLEGAL_INPUT)
    instead of failing every later launch. Validation runs before any CUDA call."""
    L = _lib.load()
    c = _lib.Config()
    L.hk_config_default(C.byref(c))
    c.block_size = block
    h = C.c_void_p()
    st = L.hk_create(C.byref(h), C.byref(c))
    if ok:
        assert st in (0, 16)   # 16: no GPU in this process
        if st == 0:
            L.hk_destroy(h)
    else:
        assert st == 4


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.load()
    h = C.c_void_p()
    assert L.hk_create(C.byref(h), None) == 16
