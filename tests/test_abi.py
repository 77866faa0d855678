"""The C-ABI library builds for sm_100a, loads on a machine without a GPU, and exports every
entry point include/mcb200.h declares."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "mcb200.h")).read()
    return sorted(set(re.findall(r"\b(mcb_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_expected_entry_points():
    from mcmatlab_b200 import native
    assert set(native.EXPORTS) == set(declared())


def test_library_exports_all_symbols():
    from mcmatlab_b200 import build, native
    build.build()
    L = C.CDLL(native.LIB_PATH)
    for name in declared():
        assert hasattr(L, name), name


def test_context_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from mcmatlab_b200 import native
    L = native.lib()
    p = C.c_void_p()
    st = L.mcb_ctx_create(0, C.byref(p))
    assert st in (1, 3)  # MCB_EINVAL / MCB_ECUDA, never a crash


def test_python_context_raises_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from mcmatlab_b200 import native
    with pytest.raises(native.MCBError):
        native.context(0)
    with pytest.raises(native.MCBError):
        native.context(0)
