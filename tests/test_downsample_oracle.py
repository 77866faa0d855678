"""The oracle's restatement of the sub-media binning against the reference's own
getDownsampledParamVals.c built with its flags (oracle/_ref/libref_downsample.so): bins and
representatives bit for bit."""
import numpy as np
import pytest

import dscases


def test_oracle_binning_matches_reference_build(ref_available, oracle_lib):
    if not ref_available:
        pytest.skip("reference build absent")
    from oracle import orc, ref
    R = ref.RefDownsample()
    for i, (par, nb) in enumerate(dscases.cases()):
        a = R.run(par, nb)
        b = orc.oracle_downsample(par, nb)
        np.testing.assert_array_equal(b[1], a[1], err_msg="labels, case %d" % i)
        np.testing.assert_array_equal(b[0], a[0], err_msg="representatives, case %d" % i)


def test_oracle_binning_properties(oracle_lib):
    from oracle import orc
    rng = np.random.default_rng(5)
    par = rng.uniform(1, 2, (3, 400)).astype(np.float32)
    reps, lab = orc.oracle_downsample(par, 10)
    assert lab.min() >= 1 and lab.max() <= 10
    # every representative is one of the points, and each point is labelled with its nearest one
    span = par.max(axis=1) - par.min(axis=1)
    nv = par / span[:, None]
    rv = reps / span[:, None]
    for k in range(10):
        assert np.any(np.all(np.abs(par - reps[:, [k]]) <= 1e-6 * np.abs(reps[:, [k]]), axis=0))
    d = ((nv[:, :, None] - rv[:, None, :]) ** 2).sum(axis=0)
    np.testing.assert_allclose(d[np.arange(400), lab.astype(int) - 1], d.min(axis=1), rtol=1e-5, atol=1e-7)
