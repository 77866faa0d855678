"""combineModels (+MCmatlab/@model/combineModels.m): weighted merging of finished runs, its
checks, and MATLAB's single-precision arithmetic."""
import copy
import math

import numpy as np
import pytest

from mcmatlab_b200 import model as mm

FACES = ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")


def _finished(seed, nPhotons, base=None):
    m = copy.deepcopy(base) if base is not None else mm.model()
    if base is None:
        m.G.nx, m.G.ny, m.G.nz = 4, 3, 2
    rng = np.random.default_rng(seed)
    MC = m.MC
    MC.nPhotons = float(nPhotons)
    MC.nPhotonsCollected = float(nPhotons // 10)
    MC.simulationTime = 0.5 * seed
    MC.normalizedFluenceRate = rng.uniform(0, 10, (4, 3, 2)).astype(np.float32)
    MC.farFieldRes = 3
    MC.farField = rng.uniform(0, 1, (3, 3)).astype(np.float32)
    for f in FACES:
        setattr(MC, "normalizedIrradiance_" + f, rng.uniform(0, 1, (3, 2)).astype(np.float32))
    MC.examplePaths = rng.uniform(0, 1, (4, 2))
    return m


def test_merge_weights_by_packets_in_single_precision():
    a = _finished(1, 100)
    b = _finished(2, 300, base=a)
    c = mm.combineModels([a, b], "MC")
    w = np.float32(300 / 100)
    want = ((a.MC.NFR + w * b.MC.NFR) * np.float32(100)) / np.float32(400)
    assert c.MC.NFR.dtype == np.float32
    np.testing.assert_array_equal(c.MC.NFR, want)
    np.testing.assert_allclose(c.MC.NFR, (100 * a.MC.NFR.astype(float) + 300 * b.MC.NFR.astype(float)) / 400, rtol=1e-6)
    for f in FACES:
        k = "normalizedIrradiance_" + f
        np.testing.assert_allclose(getattr(c.MC, k), (getattr(a.MC, k) + 3.0 * getattr(b.MC, k)) / 4.0, rtol=1e-6)
    assert c.MC.nPhotons == 400 and c.MC.nPhotonsCollected == 40 and c.MC.simulationTime == 1.5
    assert c.MC.examplePaths.shape == (4, 4)
    assert math.isnan(c.MC.lightCollector.image)
    # the inputs are left as they were
    assert a.MC.nPhotons == 100


def test_merge_weights_by_power_when_sources_differ():
    a = _finished(1, 100)
    b = _finished(2, 300, base=a)
    b.MC.lightSource.xFocus = 0.01
    a.MC.P, b.MC.P = 2.0, 1.0
    c = mm.combineModels([a, b], "MC")
    np.testing.assert_allclose(c.MC.NFR, (2 * a.MC.NFR.astype(float) + 1 * b.MC.NFR.astype(float)) / 3, rtol=1e-6)
    assert c.MC.P == 3.0 and c.MC.lightSource is None
    b.MC.P = math.nan
    with pytest.raises(ValueError, match="MC.P"):
        mm.combineModels([a, b], "MC")


def test_checks():
    a = _finished(1, 100)
    b = _finished(2, 300, base=a)
    b.G.nx = 5
    with pytest.raises(ValueError, match="G nx"):
        mm.combineModels([a, b], "MC")
    b = _finished(2, 300, base=a)
    b.MC.boundaryType = 2
    with pytest.raises(ValueError, match="MC boundaryType"):
        mm.combineModels([a, b], "MC")
    b = _finished(2, 300, base=a)
    b.MC.lightCollector.f = 0.5
    with pytest.raises(ValueError, match="light collector f"):
        mm.combineModels([a, b], "MC")
    b = _finished(2, 300, base=a)
    b.MC.nPhotons = math.nan
    with pytest.raises(ValueError, match="MC simulation executed"):
        mm.combineModels([a, b], "MC")
    with pytest.raises(ValueError, match="simType"):
        mm.combineModels([a, a], "HS")


def test_fluorescence_merge_needs_identical_excitation():
    a = _finished(1, 100)
    b = copy.deepcopy(a)
    rng = np.random.default_rng(7)
    for m, n in ((a, 50), (b, 150)):
        m.FMC.nPhotons = float(n)
        m.FMC.nPhotonsCollected = 0.0
        m.FMC.simulationTime = 1.0
        m.FMC.normalizedFluenceRate = rng.uniform(0, 1, (4, 3, 2, 2)).astype(np.float32)
    c = mm.combineModels([a, b], "FMC")
    np.testing.assert_allclose(c.FMC.NFR, (a.FMC.NFR.astype(float) + 3 * b.FMC.NFR.astype(float)) / 4, rtol=1e-6)
    assert c.FMC.nPhotons == 200
    b.MC.NFR = b.MC.NFR * 2
    with pytest.raises(ValueError, match="MC objects must all be identical"):
        mm.combineModels([a, b], "FMC")
