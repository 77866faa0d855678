"""Small seeded MC models that together exercise every branch of the transport path.

Each case returns a model (mcmatlab_b200.model.model); tests turn it into MEX-level
inputs with mexargs.prepare_mc and run it through the reference build, the CPU
oracle and the GPU library with the same inputs.
"""
from __future__ import annotations

import math

import numpy as np

from mcmatlab_b200 import configs
from mcmatlab_b200 import model as mm


def _slab_media(params):
    return [mm.mediumProperties(name="top", mua=2.0, mus=80.0, g=0.8, n=1.0),
            mm.mediumProperties(name="mid", mua=5.0, mus=120.0, g=0.9, n=1.37),
            mm.mediumProperties(name="bottom", mua=1.0, mus=60.0, g=0.7, n=1.4)]


def _slab_geom(X, Y, Z, p):
    M = np.full(X.shape, 3.0)
    M[Z < 0.06] = 2
    M[Z < 0.02] = 1
    return M


def _slab(n=24, nph=2e4):
    m = mm.model()
    m.G.nx = m.G.ny = m.G.nz = n
    m.G.Lx = m.G.Ly = m.G.Lz = 0.1
    m.G.mediaPropertiesFunc = _slab_media
    m.G.geomFunc = _slab_geom
    m.MC.nPhotonsRequested = nph
    m.MC.silentMode = True
    m.MC.wavelength = 600.0
    return m


def c0_small():
    return configs.standard_tissue_cube(n=30, nPhotons=2e4)


def c0_matched():
    m = configs.standard_tissue_cube(n=24, nPhotons=2e4, matched=True)
    return m


def iso_point_bt0():
    m = _slab()
    m.MC.matchedInterfaces = True
    m.MC.boundaryType = 0
    m.MC.LS.sourceType = 1
    m.MC.LS.xFocus, m.MC.LS.yFocus, m.MC.LS.zFocus = 0.01, -0.005, 0.05
    m.MC.LS.theta, m.MC.LS.phi = 0.4, 0.3
    m.MC.LS.emitterLength = 0.02
    m.MC.nPhotonsRequested = 5e3
    return m


def plane_bt2():
    m = _slab()
    m.MC.matchedInterfaces = True
    m.MC.boundaryType = 2
    m.MC.LS.sourceType = 2
    m.MC.LS.theta = 0.2
    m.MC.nPhotonsRequested = 2e4
    return m


def lg01_bt1():
    m = _slab()
    m.MC.matchedInterfaces = False
    m.MC.LS.sourceType = 3
    m.MC.LS.FPID.radialWidth = 0.02
    m.MC.LS.AID.radialWidth = 0.1
    m.MC.LS.zFocus = 0.03
    return m


def radial_lens_ff():
    m = _slab()
    m.MC.matchedInterfaces = False
    m.MC.LS.sourceType = 4
    m.MC.LS.FPID.radialDistr = 1
    m.MC.LS.FPID.radialWidth = 0.015
    m.MC.LS.AID.radialDistr = 0
    m.MC.LS.AID.radialWidth = 0.2
    m.MC.LS.theta = 0.1
    m.MC.farFieldRes = 12
    m.MC.useLightCollector = True
    lc = m.MC.LC
    lc.x, lc.y, lc.z = 0.0, 0.0, -0.05
    lc.theta, lc.phi = 0.0, math.pi / 2
    lc.f = 0.05
    lc.diam = 0.1
    lc.fieldSize = 0.08
    lc.res = 8
    lc.tStart, lc.tEnd, lc.nTimeBins = -2e-12, 8e-12, 10
    return m


def radial_custom_lambertian():
    m = _slab()
    m.MC.matchedInterfaces = True
    m.MC.LS.sourceType = 4
    r = np.linspace(0, 1, 1000)
    m.MC.LS.FPID.radialDistr = np.exp(-4 * r ** 2) + 0.2
    m.MC.LS.FPID.radialWidth = 0.02
    m.MC.LS.AID.radialDistr = 2
    m.MC.LS.AID.radialWidth = 0.0
    return m


def xy_custom_fiber_cyclic():
    m = _slab()
    m.MC.matchedInterfaces = False
    m.MC.boundaryType = 3
    m.MC.LS.sourceType = 5
    m.MC.LS.psi = 0.3
    x = np.linspace(-1, 1, 1000)
    m.MC.LS.FPID.XDistr = 1.0 + 0.5 * x
    m.MC.LS.FPID.XWidth = 0.02
    m.MC.LS.FPID.YDistr = 1
    m.MC.LS.FPID.YWidth = 0.01
    m.MC.LS.AID.XDistr = np.abs(x) + 0.1
    m.MC.LS.AID.XWidth = 0.2
    m.MC.LS.AID.YDistr = 0
    m.MC.LS.AID.YWidth = 0.1
    m.MC.useLightCollector = True
    lc = m.MC.LC
    lc.x, lc.y, lc.z = 0.0, 0.0, -0.02
    lc.theta, lc.phi = 0.0, math.pi / 2
    lc.f = math.inf
    lc.diam = 0.2
    lc.NA = 0.6
    lc.res = 1
    lc.tStart, lc.tEnd, lc.nTimeBins = 0.0, 2e-11, 16
    return m


def custom_phase():
    m = _slab()

    def media(p):
        base = _slab_media(p)
        base[1] = mm.mediumProperties(name="mid", mua=5.0, mus=120.0, g=math.nan,
                                      customPhaseFunc=lambda wl, th: 1.0 + 3.0 * math.cos(th) ** 2 + 4.0 * math.exp(-10 * th),
                                      n=1.0)
        return base
    m.G.mediaPropertiesFunc = media
    m.MC.matchedInterfaces = True
    m.MC.LS.sourceType = 0
    m.MC.farFieldRes = 10
    return m


def dc_end_of_life():
    m = radial_lens_ff()
    m.MC.farFieldRes = 0
    dc = m.MC.depositionCriteria
    dc.minScatterings = 2
    dc.maxScatterings = 40
    dc.onlyCollected = True
    dc.evaluateOnlyAtEndOfLife = True
    m.MC.nPhotonsRequested = 4e4
    return m


def dc_running():
    m = _slab()
    m.MC.matchedInterfaces = False
    dc = m.MC.depositionCriteria
    dc.minScatterings = 1
    dc.maxRefractions = 2
    dc.minMediumIdxToConsider = 2
    dc.evaluateOnlyAtEndOfLife = False
    return m


def distributed_source():
    m = _slab()
    m.MC.matchedInterfaces = False
    X, Y, Z = np.meshgrid(m.G.x, m.G.y, m.G.z, indexing="ij")
    m.MC.sourceDistribution = np.exp(-((X ** 2 + Y ** 2) / 0.02 ** 2 + (Z - 0.05) ** 2 / 0.01 ** 2)).astype(np.float32)
    return m


def broadband():
    m = configs.standard_tissue_cube(n=20, nPhotons=2e4)

    def media(p):
        return [mm.mediumProperties(name="air", mua=1e-8, mus=1e-8, g=1.0, n=1.0),
                mm.mediumProperties(name="epidermis", mua=lambda wl: 10.0 * (wl / 500.0) ** -2, mus=150.0, g=0.9, n=1.3),
                mm.mediumProperties(name="dermis", mua=lambda wl: 1.0 + wl / 1000.0, mus=lambda wl: 100.0 * (wl / 500.0) ** -1,
                                    g=0.9, n=1.3),
                mm.mediumProperties(name="vessel", mua=200.0, mus=100.0, g=0.9, n=1.3)]
    m.G.mediaPropertiesFunc = media
    m.MC.wavelength = np.array([450.0, 650.0])
    m.MC.spectrumFunc = lambda wl: 1.0 + (wl > 500)
    return m


def _fluo_media(params):
    return [mm.mediumProperties(name="top", mua=2.0, mus=80.0, g=0.8, n=1.0),
            mm.mediumProperties(name="mid", mua=lambda wl: 5.0 if wl < 500 else 2.0, mus=120.0, g=0.9, n=1.37,
                                QY=0.4, ES=lambda wl: math.exp(-((wl - 560.0) / 40.0) ** 2)),
            mm.mediumProperties(name="bottom", mua=1.0, mus=60.0, g=0.7, n=1.4,
                                QY=lambda wl, FR, T, FD: 0.1 * (1 + 0.01 * (T - 37.0)) + 0 * FR,
                                ES=lambda wl, FR, T, FD: wl / 600.0 + 0 * T)]


def fluorescence_excited(nph=2e4):
    """A slab whose excitation step (450 nm) has a seeded synthetic fluence-rate field in place of
    a transport run, so that the fluorescence inputs are identical wherever they are built. The
    middle medium emits with a constant yield and a Gaussian spectrum, the bottom one with a
    temperature-dependent yield (HS.T = 40) and a linear spectrum; the top one does not emit."""
    from mcmatlab_b200 import mexargs
    m = _slab(nph=nph)
    m.G.mediaPropertiesFunc = _fluo_media
    m.MC.wavelength = 450.0
    m.MC.matchedInterfaces = False
    m.HS.T = 40.0
    ex = mexargs.prepare_mc(m, 1)
    X, Y, Z = np.meshgrid(m.G.x, m.G.y, m.G.z, indexing="ij")
    m.MC.M = ex["M"]
    m.MC.mediaProperties = {"name": ex["mediaNames"], "mua": ex["mua"], "mus": ex["mus"], "g": ex["g"], "n": ex["n"],
                            "CDFidx": ex["CDFidx"]}
    m.MC.normalizedFluenceRate = (np.exp(-Z / 0.03) * np.exp(-(X ** 2 + Y ** 2) / 0.03 ** 2)).astype(np.float32)
    F = m.FMC
    F.wavelength = np.array([550.0, 650.0])
    F.nPhotonsRequested = nph
    F.silentMode = True
    F.matchedInterfaces = False
    F.boundaryType = 1
    F.farFieldRes = 8
    return m


# fluorescence runs (simType 2): prepared with mexargs.prepare_mc(model, 2)
FLUO_CASES = {"fluorescence": fluorescence_excited}

CASES = {
    "c0_small": c0_small,
    "c0_matched": c0_matched,
    "iso_point_bt0": iso_point_bt0,
    "plane_bt2": plane_bt2,
    "lg01_bt1": lg01_bt1,
    "radial_lens_ff": radial_lens_ff,
    "radial_custom_lambertian": radial_custom_lambertian,
    "xy_custom_fiber_cyclic": xy_custom_fiber_cyclic,
    "custom_phase": custom_phase,
    "dc_end_of_life": dc_end_of_life,
    "dc_running": dc_running,
    "distributed_source": distributed_source,
    "broadband": broadband,
}
