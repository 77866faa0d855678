"""Heat simulation with temperature-dependent media on the GPU: every mediaPropRecalcPeriod
updates the MC is re-run at the current temperatures and the thermal media are re-binned
(simulateHeatDistribution.m:295-296, :356-357, :417-418, heatSimParamsRecalc :516-541)."""
import numpy as np
import pytest

from mcmatlab_b200 import model as mm
from mcmatlab_b200 import prep

pytestmark = pytest.mark.gpu


def _model(recalc):
    def media(p):
        return [mm.mediumProperties(name="air", mua=1e-8, mus=1e-8, g=1.0, n=1.0, VHC=1.2e-3, TC=2.6e-4),
                mm.mediumProperties(name="chromic", mua=lambda wl, FR, T, FD: 20.0 * (1.0 + 0.05 * (T - 37.0)) + 0 * FR,
                                    mus=100.0, g=0.9, n=1.0, VHC=lambda T, FD: 3.9 * (1.0 + 0.002 * (T - 37.0)),
                                    TC=0.0037, nBins=4)]

    def geom(X, Y, Z, p):
        M = np.full(X.shape, 2.0)
        M[Z < 0.01] = 1
        return M
    m = mm.model()
    m.G.nx = m.G.ny = m.G.nz = 24
    m.G.Lx = m.G.Ly = m.G.Lz = 0.1
    m.G.mediaPropertiesFunc = media
    m.G.geomFunc = geom
    m.MC.nPhotonsRequested = 5e4
    m.MC.matchedInterfaces = True
    m.MC.silentMode = True
    m.MC.wavelength = 532.0
    m.MC.lightSource.sourceType = 0
    m.MC.P = 2.0
    m.HS.silentMode = True
    m.HS.durationOn = 0.02
    m.HS.durationEnd = 0.01
    m.HS.nUpdates = 4
    m.HS.T = 37.0
    m.HS.mediaPropRecalcPeriod = 2 if recalc else 0
    return m


def test_heat_with_media_recalculation():
    m = _model(True)
    m.runMonteCarlo()
    mua0 = np.asarray(m.MC.mediaProperties["mua"])[:, 0].copy()
    m.simulateHeatDistribution()
    T = np.asarray(m.HS.T)
    assert np.all(np.isfinite(T)) and T.max() > 40.0
    # the MC was re-run at the heated temperatures: the chromic medium is split and absorbs more
    mua1 = np.asarray(m.MC.mediaProperties["mua"])[:, 0]
    assert mua1.shape == (5,) and mua1[1:].max() > mua0[1:].max()
    assert np.unique(np.asarray(m.MC.M)[np.asarray(m.G.M_raw) == 2]).size >= 2
    # the thermal media were re-binned by temperature
    VHC = np.asarray(m.HS.mediaProperties["VHC"])
    assert VHC.shape == (5,) and VHC[1:].max() > VHC[1:].min()
    # without recalculation the properties stay at their 37 C values
    m2 = _model(False)
    m2.runMonteCarlo()
    m2.simulateHeatDistribution()
    assert np.all(np.asarray(m2.HS.mediaProperties["VHC"])[1:] == np.float32(3.9))
    assert not np.allclose(np.asarray(m2.HS.T), T)
