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


@pytest.mark.parametrize("name", ["c0_small", "radial_lens_ff", "broadband", "plane_bt2", "xy_custom_fiber_cyclic"])
def test_tally_count_layout(name):
    """mcb_mc_tally_count (host only, no GPU): per wavelength the voxel tallies, image, far field
    and escape-face tallies (boundaryType 2: a 5x-wide z < 0 face), then two packet counts."""
    import sys
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import mccases
    from mcmatlab_b200 import abi, mexargs, native
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    mb = abi.McModelBuffers(mc_in)
    m = mb.model
    nx, ny, nz, nL = m.nx, m.ny, m.nz, m.nL
    nT = m.LC_nTimeBins + 2 if m.LC_nTimeBins else 1
    Lim = m.LC_res ** 2 * nT if m.useLightCollector else 0
    Lzn = 25 * nx * ny if m.boundaryType == 2 else nx * ny
    per = (nx * ny * nz if m.calcNFR else 0) + Lim + m.farFieldRes ** 2 + 2 * ny * nz + 2 * nx * nz + nx * ny + Lzn + 2
    assert native.lib().mcb_mc_tally_count(C.byref(m)) == per * nL
    shapes = abi.result_shapes(mc_in)
    if "NFR" in shapes:
        assert int(np.prod(shapes["NFR"])) == nx * ny * nz * nL


def test_size_class():
    """mcb_mc_size_class (host only): voxels in powers of 4, +16 gradient, +32 batched."""
    from mcmatlab_b200 import abi, native
    m = abi.mcb_mc_model()
    for (nx, ny, nz), want in (((2, 2, 2), 1), ((100, 100, 100), 9), ((256, 256, 256), 12), ((1024, 1024, 1024), 15)):
        m.nx, m.ny, m.nz = nx, ny, nz
        assert native.lib().mcb_mc_size_class(C.byref(m), 0, 0) == want
        assert native.lib().mcb_mc_size_class(C.byref(m), 1, 1) == want + 48
