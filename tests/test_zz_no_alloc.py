"""mcb_heat_forward_static, the heat entry that allocates nothing (its working set is a 32 MiB
static device array), against mcb_heat_forward on the same inputs: two calls in a row, each
within the tolerance below of the allocating entry; its size limit; and no change of free
device memory across a call. Kept last in collection so that it also runs after every other
GPU test has used the context."""
import numpy as np
import pytest

import heatcases

pytestmark = pytest.mark.gpu

TOL_T = 1e-5      # relative, temperatures, sensors and maxima (both paths run the same FP32 kernels)
TOL_OMEGA = 1e-5  # relative to the damage accumulated in the call


def _compare(a, b, case):
    Ta, Oa, Sa, Ma = a
    Tb, Ob, Sb, Mb = b
    assert np.max(np.abs(Tb - Ta) / np.abs(Ta)) <= TOL_T
    if Sa.size:
        assert np.max(np.abs(Sb - Sa) / np.abs(Sa)) <= TOL_T
    np.testing.assert_allclose(Mb, Ma, rtol=TOL_T)
    if Oa is not None:
        inc = np.max(np.abs(Oa - case["Omega0"]))
        assert np.max(np.abs(Ob - Oa)) <= TOL_OMEGA * inc + 2 * np.finfo(np.float32).eps * np.max(np.abs(Oa))


def _c1_like():
    # 64^3 with damage and three sensors, 40 steps: past the 16-step graph chunks of the allocating path
    return heatcases._base(64, 9, 0, True, 40, 0.9, True)


@pytest.mark.parametrize("name", sorted(heatcases.CASES) + ["c1_like_64"])
def test_static_entry_matches_allocating_entry_twice(name):
    from mcmatlab_b200 import native
    case = _c1_like() if name == "c1_like_64" else heatcases.CASES[name]()
    nx, ny, nz = case["n"]
    ref = native.heat_forward(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    first = native.heat_forward_static(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    second = native.heat_forward_static(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    _compare(ref, first, case)
    _compare(ref, second, case)


def test_static_entry_allocates_no_device_memory():
    import torch
    from mcmatlab_b200 import native
    case = _c1_like()
    nx, ny, nz = case["n"]
    native.heat_forward_static(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)  # set-up call
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    native.heat_forward_static(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_entry_rejects_grids_beyond_its_scratch():
    from mcmatlab_b200 import native
    big = heatcases._base(128, 5, 0, True, 1, 0.9, True)  # 2.1e6 voxels: beyond 32 MiB
    with pytest.raises(native.MCBError, match="static limit"):
        native.heat_forward_static(big["T0"], big["Omega0"], big["hp"], 128, 128, 128)
    # a small grid whose sensor history (8 B per sensor and step) alone exceeds the scratch
    long = heatcases._base(8, 6, 0, True, 2_000_000, 0.9, False)
    with pytest.raises(native.MCBError, match="static limit"):
        native.heat_forward_static(long["T0"], None, long["hp"], 8, 8, 8)
    # the context stays usable, and the same grid runs through the allocating entry
    case = heatcases.CASES["insulated_on"]()
    nx, ny, nz = case["n"]
    ref = native.heat_forward(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    _compare(ref, native.heat_forward_static(case["T0"], case["Omega0"], case["hp"], nx, ny, nz), case)
    native.heat_forward(big["T0"], big["Omega0"], big["hp"], 128, 128, 128)
