"""End-to-end through the Python mirror of MCmatlab.model: runMonteCarlo then
simulateHeatDistribution, checked against the CPU oracle run on the same inputs."""
import math

import numpy as np
import pytest

import mcstats
from mcmatlab_b200 import configs, mexargs, prep

pytestmark = pytest.mark.gpu


def test_run_mc_and_heat_match_oracle(oracle_lib):
    from oracle import orc
    m = configs.standard_tissue_cube(n=30, nPhotons=1e5, seed=5)
    m.runMonteCarlo()
    NFR = m.MC.NFR
    assert NFR.shape == (30, 30, 30) and m.MC.nPhotons == 1e5
    assert m.MC.NI_zneg.shape == (30, 30)
    mc_in = mexargs.prepare_mc(m)
    o = orc.oracle_mc(mc_in, 0)
    sg = mcstats.summaries({"NFR": NFR[..., None], "NI_zneg": m.MC.NI_zneg[..., None]}, mc_in)
    so = mcstats.summaries(o, mc_in)
    for k in ("abs_m1_l0", "abs_m2_l0", "abs_m3_l0", "NI_zneg_l0"):
        assert abs(sg[k] - so[k]) <= 0.03 * abs(so[k]) + 1e-4, (k, sg[k], so[k])

    HS = m.HS
    HS.durationOn, HS.durationOff, HS.durationEnd = 2e-4, 1e-4, 0.0
    HS.nUpdates = 4
    HS.T = 37.0
    HS.tempSensorPositions = np.array([[0.0, 0.0, 0.04], [0.0, 0.0, 0.012]])
    m.simulateHeatDistribution()
    Tg = HS.T
    # the same schedule through the FP64 oracle
    G = m.G
    th = prep.thermal_media_properties(G.mediaPropertiesFunc([]), G.M_raw)
    NA = np.asarray(m.MC.normalizedAbsorption)[..., 0]
    c, Q = prep.calc_dTdt_arrays(th["VHC"], th["TC"], G.dx, G.dy, G.dz, NA, m.MC.P, th["M"])
    dtmax = prep.calc_dtmax(th["M"], th["TC"], th["VHC"], G.dx, G.dy, G.dz) * 1.5
    sched = prep.heat_schedule(2e-4, 1e-4, 0.0, 4, dtmax)
    li, w = prep.convert_temp_sensor_pos(HS.tempSensorPositions, G.x, G.y, G.z)
    T = np.full((30, 30, 30), 37.0)
    Om = np.zeros((30, 30, 30))
    for phase, lights in (("on", True), ("off", False)):
        nU, nT, dt = sched[phase]
        for _ in range(nU):
            hp = mexargs.heat_mex_params(th["M"], th["A"], th["E"], c, Q, True, 0, li, w, lights, nT, dt)
            T, Om, S, Mx = orc.oracle_heat(T, Om, hp, 30, 30, 30)
    assert np.max(np.abs(Tg - T) / T) <= 1e-5
    assert HS.sensorTemps.shape[0] == 2
    assert len(HS.sensorsTimeVector) == HS.sensorTemps.shape[1]
    np.testing.assert_allclose(HS.sensorTemps[:, -1], S[:, -1], rtol=1e-5)
    assert HS.maxMediaTemps[3] >= 37.0
