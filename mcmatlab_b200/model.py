"""Python mirror of the reference's MCmatlab.model object API.

The reference user API is a set of MATLAB value classes (+MCmatlab/@<name>/<name>.m)
holding inputs and results; model.runMonteCarlo and model.simulateHeatDistribution
prepare MEX inputs and call the native code. This module keeps the same class names,
property names, defaults and validation messages for the properties that feed the two
hot paths, and routes the native calls to the sm_100a library through its C ABI
(mcmatlab_b200.native). Property aliases the reference keeps for backward
compatibility (LS, LC, FPID, AID, NFR, NA, NI_*) are provided as well.

Out of scope here (they do not feed either hot path): plotting, movies,
FR/T/FD-dependent media (sub-media splitting), fluorescence source construction and
model merging.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Callable, List, Optional

import numpy as np

from . import prep


def _nan():
    return math.nan


@dataclass
class mediumProperties:
    """+MCmatlab/@mediumProperties/mediumProperties.m:1-20 (properties and defaults)."""
    name: str = "Unlabeled medium"
    mua: Any = math.nan
    mus: Any = math.nan
    g: Any = math.nan
    customPhaseFunc: Any = None
    n: Any = 1.0
    QY: Any = 0.0
    ES: Any = 1.0
    VHC: Any = math.nan
    TC: Any = math.nan
    E: float = 0.0
    A: float = 0.0
    nBins: int = 1


@dataclass
class geometry:
    """+MCmatlab/@geometry/geometry.m:1-40, 110-138."""
    silentMode: bool = False
    nx: int = 100
    ny: int = 100
    nz: int = 100
    Lx: float = 1.0
    Ly: float = 1.0
    Lz: float = 1.0
    mediaPropertiesFunc: Callable = field(default=lambda p: [mediumProperties()])
    mediaPropParams: list = field(default_factory=list)
    geomFunc: Callable = field(default=lambda X, Y, Z, p: np.ones(X.shape))
    geomFuncParams: list = field(default_factory=list)
    M_raw: Optional[np.ndarray] = None

    @property
    def dx(self):
        return self.Lx / self.nx

    @property
    def dy(self):
        return self.Ly / self.ny

    @property
    def dz(self):
        return self.Lz / self.nz

    @property
    def x(self):
        return prep.geometry_axes(self.nx, self.ny, self.nz, self.Lx, self.Ly, self.Lz)[0]

    @property
    def y(self):
        return prep.geometry_axes(self.nx, self.ny, self.nz, self.Lx, self.Ly, self.Lz)[1]

    @property
    def z(self):
        return prep.geometry_axes(self.nx, self.ny, self.nz, self.Lx, self.Ly, self.Lz)[2]

    def updateGeometry(self):
        for name, v in (("nx", self.nx), ("ny", self.ny), ("nz", self.nz)):
            if int(v) != v or v <= 1:
                raise ValueError("Error: %s must be an integer greater than 1." % name)
        self.M_raw = prep.evaluate_geometry(self)
        return self


@dataclass
class sourceIntensityDistribution:
    """+MCmatlab/@sourceIntensityDistribution/sourceIntensityDistribution.m:4-10.

    Distr values: 0 top-hat, 1 Gaussian, 2 cosine (Lambertian), or a custom array.
    """
    radialDistr: Any = math.nan
    radialWidth: float = math.nan
    XDistr: Any = math.nan
    XWidth: float = math.nan
    YDistr: Any = math.nan
    YWidth: float = math.nan


@dataclass
class lightSource:
    """+MCmatlab/@lightSource/lightSource.m:6-21.

    sourceType 0 pencil beam, 1 isotropic point/line, 2 infinite plane wave,
    3 Laguerre-Gaussian LG01, 4 radially factorizable, 5 X/Y factorizable.
    """
    sourceType: int = 0
    xFocus: float = 0.0
    yFocus: float = 0.0
    zFocus: float = 0.0
    theta: float = 0.0
    phi: float = 0.0
    psi: float = 0.0
    emitterLength: float = 0.0
    focalPlaneIntensityDistribution: sourceIntensityDistribution = field(default_factory=sourceIntensityDistribution)
    angularIntensityDistribution: sourceIntensityDistribution = field(default_factory=sourceIntensityDistribution)

    @property
    def FPID(self):
        return self.focalPlaneIntensityDistribution

    @FPID.setter
    def FPID(self, v):
        self.focalPlaneIntensityDistribution = v

    @property
    def AID(self):
        return self.angularIntensityDistribution

    @AID.setter
    def AID(self, v):
        self.angularIntensityDistribution = v


@dataclass
class lightCollector:
    """+MCmatlab/@lightCollector/lightCollector.m:5-28."""
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0
    theta: float = 0.0
    phi: float = math.pi / 2
    f: float = math.inf
    diam: float = 1.0
    fieldSize: float = 1.0
    NA: float = 0.22
    res: int = 0
    tStart: float = 0.0
    tEnd: float = 1e-12
    nTimeBins: int = 0
    image: Any = math.nan
    X: Any = math.nan
    Y: Any = math.nan
    t: Any = math.nan


@dataclass
class depositionCriteria:
    """+MCmatlab/@depositionCriteria/depositionCriteria.m:31-52."""
    minScatterings: float = 0
    maxScatterings: float = math.inf
    minRefractions: float = 0
    maxRefractions: float = math.inf
    minReflections: float = 0
    maxReflections: float = math.inf
    minInterfaceTransitions: float = 0
    maxInterfaceTransitions: float = math.inf
    minMediumIdxToConsider: float = 1
    maxMediumIdxToConsider: float = math.inf
    onlyCollected: bool = False
    evaluateOnlyAtEndOfLife: bool = True
    minSubmediaIdx: float = 1
    maxSubmediaIdx: float = math.inf


@dataclass
class monteCarloSimulation:
    """+MCmatlab/@monteCarloSimulation/monteCarloSimulation.m:5-70 (inputs and results).

    `seed` is an addition: the transport RNG here is counter-based (Philox-4x32-10)
    and reproducible for a given seed; the reference seeds from the clock.
    """
    silentMode: bool = False
    useAllCPUs: bool = False
    useGPU: bool = True
    GPUdevice: int = 0
    simulationTimeRequested: float = 0.1
    nPhotonsRequested: float = math.nan
    requestCollectedPhotons: bool = False
    calcNormalizedFluenceRate: bool = True
    nExamplePaths: int = 0
    farFieldRes: int = 0
    matchedInterfaces: bool = True
    smoothingLengthScale: float = 0.1
    boundaryType: int = 1
    wavelength: Any = 800.0
    P: float = 1.0
    spectrumFunc: Callable = field(default=lambda wl: 1.0)
    FRinitial: Any = math.nan
    FRdepIterations: int = 0
    lightSource: lightSource = field(default_factory=lightSource)
    useLightCollector: bool = False
    lightCollector: lightCollector = field(default_factory=lightCollector)
    depositionCriteria: depositionCriteria = field(default_factory=depositionCriteria)
    sourceDistribution: Any = math.nan
    seed: int = 1
    # results
    simulationTime: float = math.nan
    nPhotons: float = math.nan
    nPhotonsCollected: float = math.nan
    nThreads: float = math.nan
    mediaProperties: Any = math.nan
    CDFs: Any = None
    M: Any = math.nan
    interfaceNormals: Any = math.nan
    spectrum: Any = math.nan
    examplePaths: Any = math.nan
    normalizedFluenceRate: Any = 0
    FR: Any = 0
    farField: Any = math.nan
    farFieldTheta: Any = math.nan
    farFieldPhi: Any = math.nan
    normalizedIrradiance_xpos: Any = math.nan
    normalizedIrradiance_xneg: Any = math.nan
    normalizedIrradiance_ypos: Any = math.nan
    normalizedIrradiance_yneg: Any = math.nan
    normalizedIrradiance_zpos: Any = math.nan
    normalizedIrradiance_zneg: Any = math.nan
    kernelStats: Any = None

    # aliases kept by the reference (monteCarloSimulation.m:72-90, 130-170)
    LS = property(lambda s: s.lightSource, lambda s, v: setattr(s, "lightSource", v))
    LC = property(lambda s: s.lightCollector, lambda s, v: setattr(s, "lightCollector", v))
    NFR = property(lambda s: s.normalizedFluenceRate, lambda s, v: setattr(s, "normalizedFluenceRate", v))
    calcNFR = property(lambda s: s.calcNormalizedFluenceRate, lambda s, v: setattr(s, "calcNormalizedFluenceRate", v))
    NI_xpos = property(lambda s: s.normalizedIrradiance_xpos)
    NI_xneg = property(lambda s: s.normalizedIrradiance_xneg)
    NI_ypos = property(lambda s: s.normalizedIrradiance_ypos)
    NI_yneg = property(lambda s: s.normalizedIrradiance_yneg)
    NI_zpos = property(lambda s: s.normalizedIrradiance_zpos)
    NI_zneg = property(lambda s: s.normalizedIrradiance_zneg)

    @property
    def normalizedAbsorption(self):
        """NA = mua(M) .* NFR per wavelength (monteCarloSimulation.m:98-108)."""
        NFR = np.asarray(self.normalizedFluenceRate)
        if NFR.size <= 1:
            return 0
        mua = np.asarray(self.mediaProperties["mua"])
        M = np.asarray(self.M).astype(np.int64) - 1
        NA = np.empty(NFR.shape if NFR.ndim == 4 else NFR.shape + (1,), dtype=np.float64)
        NFR4 = NFR if NFR.ndim == 4 else NFR[..., None]
        for iL in range(NA.shape[3]):
            NA[..., iL] = (mua[:, iL][M].astype(np.float32) * NFR4[..., iL]).astype(np.float32)
        return NA

    NA = property(lambda s: s.normalizedAbsorption)


@dataclass
class heatSimulation:
    """+MCmatlab/@heatSimulation/heatSimulation.m:5-45."""
    silentMode: bool = False
    useAllCPUs: bool = False
    useGPU: bool = True
    largeTimeSteps: bool = False
    heatBoundaryType: int = 0
    durationOn: float = 0.0
    durationOff: float = 0.0
    durationEnd: float = 0.0
    nPulses: int = 1
    nUpdates: int = 10
    mediaPropRecalcPeriod: int = 0
    tempSensorPositions: Any = None
    T: Any = 37.0
    mediaProperties: Any = math.nan
    M: Any = math.nan
    Omega: Any = 0.0
    maxMediaTemps: Any = math.nan
    sensorsTimeVector: Any = math.nan
    sensorTemps: Any = math.nan
    # explicit time step override (the reference derives dt from calcdtmax; see simulateHeatDistribution)
    dtFactor: float = math.nan


class model:
    """+MCmatlab/@model/model.m: the top-level object holding G, MC, FMC and HS."""

    def __init__(self):
        self.name = "model"
        self.G = geometry()
        self.MC = monteCarloSimulation()
        self.FMC = monteCarloSimulation()
        self.HS = heatSimulation()

    def runMonteCarlo(self, *args):
        from .runmc import runMonteCarlo
        return runMonteCarlo(self, *args)

    def simulateHeatDistribution(self):
        from .heatsim import simulateHeatDistribution
        return simulateHeatDistribution(self)


def combineModels(modelArray, simType):
    """+MCmatlab/@model/combineModels.m: one model holding the merged results of several runs."""
    from .combine import combineModels as _combine
    return _combine(modelArray, simType)
