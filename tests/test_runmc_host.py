"""Host flow of runMonteCarlo (runMonteCarlo.m:81-113) with the transport replaced by the
oracle: the fluence-rate iterations' packet schedule (1/4, 1/2, all of the requested packets for
three iterations), re-binning on the previous iteration's fluence rate, and the restored request;
the fluorescence step's results landing in model.FMC."""
import numpy as np
import pytest

import mccases
from mcmatlab_b200 import model as mm


@pytest.fixture
def oracle_transport(monkeypatch, oracle_lib):
    from mcmatlab_b200 import native
    from oracle import orc
    calls = []

    def mc_run(mc_in, device=0, example_cap=100000):
        calls.append(dict(nPhotons=mc_in["nPhotonsRequested"], mua=np.array(mc_in["mua"]), M=np.array(mc_in["M"])))
        return orc.oracle_mc(mc_in, 0)
    monkeypatch.setattr(native, "mc_run", mc_run)
    monkeypatch.setattr(native, "interface_normals", lambda *a, device=0, **k: pytest.fail("normals not expected"))
    monkeypatch.setattr(native, "downsample_params", lambda par, nb, device=0: orc.oracle_downsample(par, nb))
    return calls


def _saturable():
    def media(p):
        return [mm.mediumProperties(name="air", mua=1e-8, mus=1e-8, g=1.0, n=1.0),
                mm.mediumProperties(name="absorber", mua=lambda wl, FR, T, FD: 50.0 / (1.0 + FR / 200.0) + 0 * T,
                                    mus=100.0, g=0.9, n=1.0, nBins=6)]

    def geom(X, Y, Z, p):
        M = np.full(X.shape, 2.0)
        M[Z < 0.01] = 1
        return M
    m = mm.model()
    m.G.nx = m.G.ny = m.G.nz = 16
    m.G.Lx = m.G.Ly = m.G.Lz = 0.1
    m.G.mediaPropertiesFunc = media
    m.G.geomFunc = geom
    m.MC.nPhotonsRequested = 8e3
    m.MC.matchedInterfaces = True
    m.MC.silentMode = True
    m.MC.wavelength = 532.0
    m.MC.lightSource.sourceType = 0
    m.MC.P = 50.0
    m.MC.FRdepIterations = 3
    return m


def test_fr_iterations_schedule_and_rebinning(oracle_transport):
    m = _saturable()
    m.runMonteCarlo()
    calls = oracle_transport
    assert [c["nPhotons"] for c in calls] == [2e3, 4e3, 8e3]
    assert m.MC.nPhotonsRequested == 8e3 and m.MC.nPhotons == 8e3
    # first iteration: no fluence rate yet, one value for the absorber; later ones re-binned
    assert np.unique(calls[0]["M"][calls[0]["M"] > 1]).size == 1
    assert np.unique(calls[2]["M"][calls[2]["M"] > 1]).size > 1
    assert calls[2]["mua"][1:, 0].min() < 50.0
    FR = np.asarray(m.MC.FR)  # P x NFR of the second iteration (runMonteCarlo.m:107)
    assert FR.shape == (16, 16, 16) and np.all(FR >= 0) and FR.max() > 0


def test_fluorescence_results_land_in_fmc(oracle_transport):
    m = mccases.fluorescence_excited()
    m.FMC.matchedInterfaces = True
    m.runMonteCarlo("fluorescence")
    F = m.FMC
    assert np.asarray(F.NFR).shape == (24, 24, 24, 2) and F.nPhotons == 2e4
    assert np.asarray(F.sourceDistribution).shape == (24, 24, 24, 2)
    assert np.asarray(F.farField).shape == (8, 8, 2)
    assert np.isnan(m.MC.nPhotons)  # the excitation object is untouched


class _OracleHeatState:
    """Stands in for native.HeatState with the FP64 oracle stepper (host flow tests only)."""
    created = 0

    def __init__(self, T, Omega, hp, nx, ny, nz, device=0):
        type(self).created += 1
        self.n = (nx, ny, nz)
        self.T = np.asarray(T, dtype=np.float64).reshape(self.n, order="F")
        self.O = None if Omega is None else np.asarray(Omega, dtype=np.float64).reshape(self.n, order="F")

    def step(self, hp):
        from oracle import orc
        self.T, self.O, sens, mx = orc.oracle_heat(self.T, self.O, hp, *self.n)
        return (sens if sens is not None else np.zeros((0, 0))), np.asarray(mx, dtype=np.float32).reshape(1, -1)

    def read(self):
        return self.T.astype(np.float32), (None if self.O is None else self.O.astype(np.float32))

    def close(self):
        pass


def _chromic(period):
    def media(p):
        return [mm.mediumProperties(name="air", mua=1e-8, mus=1e-8, g=1.0, n=1.0, VHC=1.2e-3, TC=2.6e-4),
                mm.mediumProperties(name="chromic", mua=lambda wl, FR, T, FD: 20.0 * (1.0 + 0.05 * (T - 37.0)) + 0 * FR,
                                    mus=100.0, g=0.9, n=1.0, VHC=lambda T, FD: 3.9 * (1.0 + 0.002 * (T - 37.0)),
                                    TC=0.0037, nBins=3)]

    def geom(X, Y, Z, p):
        M = np.full(X.shape, 2.0)
        M[Z < 0.01] = 1
        return M
    m = mm.model()
    m.G.nx = m.G.ny = m.G.nz = 12
    m.G.Lx = m.G.Ly = m.G.Lz = 0.1
    m.G.mediaPropertiesFunc = media
    m.G.geomFunc = geom
    m.MC.nPhotonsRequested = 4e3
    m.MC.matchedInterfaces = True
    m.MC.silentMode = True
    m.MC.wavelength = 532.0
    m.MC.lightSource.sourceType = 0
    m.MC.P = 20.0
    m.HS.silentMode = True
    m.HS.durationOn = 0.1
    m.HS.durationOff = 0.05
    m.HS.durationEnd = 0.05
    m.HS.nPulses = 2
    m.HS.nUpdates = 4
    m.HS.mediaPropRecalcPeriod = period
    return m


def test_heat_recalculation_schedule(oracle_transport, monkeypatch):
    """nUpdates = 4 splits into 3 on and 1 off update per pulse and 1 end update
    (simulateHeatDistribution.m:80-110): 2 pulses give 9 updates, and every 3rd re-runs the MC
    and rebuilds the stepper, after updates 3, 6 and 9, as the update index of :280, :341, :401
    runs through the pulses and the end phase."""
    from mcmatlab_b200 import native
    monkeypatch.setattr(native, "HeatState", _OracleHeatState)
    _OracleHeatState.created = 0
    m = _chromic(3)
    m.runMonteCarlo()
    n0 = len(oracle_transport)
    m.simulateHeatDistribution()
    assert len(oracle_transport) - n0 == 3
    assert _OracleHeatState.created == 1 + 3
    assert np.asarray(m.HS.T).max() > 37.0
    assert np.asarray(m.HS.mediaProperties["VHC"]).shape == (4,)
    _OracleHeatState.created = 0
    m2 = _chromic(0)
    m2.runMonteCarlo()
    n1 = len(oracle_transport)
    m2.simulateHeatDistribution()
    assert len(oracle_transport) == n1 and _OracleHeatState.created == 1
