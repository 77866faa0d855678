"""Sub-media binning on the device (mcb_downsample_params) against the oracle restatement, which
is pinned bit for bit to the reference build: identical bins and representatives."""
import numpy as np
import pytest

import dscases

pytestmark = pytest.mark.gpu


def test_gpu_binning_matches_oracle_bit_for_bit(oracle_lib):
    from mcmatlab_b200 import native
    from oracle import orc
    for i, (par, nb) in enumerate(dscases.cases()):
        a = orc.oracle_downsample(par, nb)
        b = native.downsample_params(par, nb)
        np.testing.assert_array_equal(b[1], a[1], err_msg="labels, case %d" % i)
        np.testing.assert_array_equal(b[0], a[0], err_msg="representatives, case %d" % i)


def test_gpu_binning_large_medium(oracle_lib):
    """A million voxels into 64 bins (the serial reference takes seconds here)."""
    from mcmatlab_b200 import native
    from oracle import orc
    rng = np.random.default_rng(11)
    n = 1_000_000
    T = rng.normal(60, 15, n)
    par = np.stack([2.0 + 0.05 * T, 100.0 - 0.3 * T, np.full(n, 0.9)]).astype(np.float32)
    a = orc.oracle_downsample(par, 64)
    b = native.downsample_params(par, 64)
    np.testing.assert_array_equal(b[1], a[1])
    np.testing.assert_array_equal(b[0], a[0])


def test_gpu_binning_rejects_bad_sizes():
    from mcmatlab_b200 import native
    par = np.ones((3, 10), np.float32)
    for nb in (0, 256):
        with pytest.raises(native.MCBError):
            native.downsample_params(par, nb)
