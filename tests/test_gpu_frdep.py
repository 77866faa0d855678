"""Fluence-rate dependent media end to end on the GPU (runMonteCarlo.m:81-113 with
getOpticalMediaProperties' sub-media binning on the device): a saturable absorber re-binned over
three iterations with 1/4, 1/2 and all of the requested packets."""
import numpy as np
import pytest

from mcmatlab_b200 import mexargs
from mcmatlab_b200 import model as mm

pytestmark = pytest.mark.gpu


def _saturable(n=32, nph=1e5):
    def media(p):
        return [mm.mediumProperties(name="air", mua=1e-8, mus=1e-8, g=1.0, n=1.0),
                mm.mediumProperties(name="absorber", mua=lambda wl, FR, T, FD: 50.0 / (1.0 + FR / 200.0) + 0 * T,
                                    mus=100.0, g=0.9, n=1.0, nBins=8)]

    def geom(X, Y, Z, p):
        M = np.full(X.shape, 2.0)
        M[Z < 0.01] = 1
        return M
    m = mm.model()
    m.G.nx = m.G.ny = m.G.nz = n
    m.G.Lx = m.G.Ly = m.G.Lz = 0.1
    m.G.mediaPropertiesFunc = media
    m.G.geomFunc = geom
    m.MC.nPhotonsRequested = nph
    m.MC.matchedInterfaces = True
    m.MC.silentMode = True
    m.MC.wavelength = 532.0
    m.MC.lightSource.sourceType = 0
    m.MC.P = 50.0
    m.MC.FRdepIterations = 3
    return m


def test_fr_dependent_iterations_rebin_the_absorber(oracle_lib):
    from mcmatlab_b200 import native
    from oracle import orc
    m = _saturable()
    m.runMonteCarlo()
    MC = m.MC
    assert MC.nPhotonsRequested == 1e5 and MC.nPhotons == 1e5
    NFR = np.asarray(MC.NFR)
    assert NFR.shape == (32, 32, 32) and np.all(np.isfinite(NFR)) and NFR.max() > 0
    mua = np.asarray(MC.mediaProperties["mua"])[:, 0]
    assert mua.shape == (9,)
    sub = np.unique(np.asarray(MC.M)[np.asarray(m.G.M_raw) == 2])
    assert sub.size >= 4  # the absorber is split by its fluence rate
    assert np.all(mua[1:] <= 50.0) and mua[1:].min() < 45.0  # saturated bins absorb less
    assert np.all(np.diff(mua[1:]) >= 0)
    # the device binning inside the host flow equals the oracle's on the same model state
    a = mexargs.prepare_mc(m, 1, downsample=native.downsample_params)
    b = mexargs.prepare_mc(m, 1, downsample=orc.oracle_downsample)
    np.testing.assert_array_equal(a["M"], b["M"])
    np.testing.assert_array_equal(a["mua"], b["mua"])
