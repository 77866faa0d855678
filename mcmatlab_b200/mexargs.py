"""The MEX-level view of a model: what the reference's MEX functions read.

`prepare_mc(model, simType)` performs the MATLAB-side steps of runMonteCarlo
(+MCmatlab/@model/runMonteCarlo.m:51-66, :145-176) that happen before the MEX call and
returns a flat dict `mc_in` of numpy arrays and scalars. `mex_model_tree(mc_in)`
turns that dict into the nested property tree the MEX function reads with
mxGetPropertyShared (+MCmatlab/src/MCmatlab.c:317-616), with MATLAB's types:
Python bool -> logical, number -> double, numpy arrays keep their dtype.
The same tree drives the reference MEX (through the oracle's mx shim) and this
library's MEX shim, so both see identical inputs.

`heat_mex_params(...)` builds the heatSimParameters struct of
+MCmatlab/@model/simulateHeatDistribution.m:209-211 as read by
+MCmatlab/src/finiteElementHeatPropagator.c:688-739.
"""
from __future__ import annotations

import math

import numpy as np

from . import prep


def _distr(v):
    return np.atleast_1d(np.asarray(v, dtype=np.float64)).reshape(1, -1)


_RESTRICTIVE = ("minScatterings", "maxScatterings", "minRefractions", "maxRefractions", "minReflections",
                "maxReflections", "minInterfaceTransitions", "maxInterfaceTransitions")


def _fr_t_fd(mdl):
    """Fluence rate, temperature and fractional damage grids of the model (getOpticalMediaProperties.m:23-30)."""
    G = mdl.G
    shape = G.M_raw.shape
    T = np.broadcast_to(np.asarray(mdl.HS.T, dtype=np.float32), shape)
    FD = np.broadcast_to((1 - np.exp(-np.asarray(mdl.HS.Omega, dtype=np.float64))).astype(np.float32), shape)
    NFR = np.asarray(mdl.MC.NFR, dtype=np.float32)
    FR = np.broadcast_to((mdl.MC.P * (NFR.sum(axis=3) if NFR.ndim == 4 else NFR)).astype(np.float32), shape)
    return FR, T, FD


def prepare_mc(mdl, simType=1, normals=None, downsample=None):
    """Flat MEX-level inputs for one MC run (runMonteCarlo.m + getOpticalMediaProperties.m).

    simType 1 reads model.MC; simType 2 (fluorescence) reads model.FMC, as MCmatlab.c:322-323
    does, and builds the fluorescence source from the excitation run's model.MC results
    (runMonteCarlo.m:119-166, prep.fluorescence_source), which it also stores in
    model.FMC.sourceDistribution. `normals` replaces prep.interface_normals (runMonteCarlo
    passes the device version); `downsample` performs the sub-media binning of media whose optical
    properties depend on fluence rate, temperature or damage (runMonteCarlo passes
    native.downsample_params)."""
    if simType not in (1, 2):
        raise ValueError("simType must be 1 (MC) or 2 (fluorescence MC)")
    G = mdl.G
    MC = mdl.FMC if simType == 2 else mdl.MC
    if G.M_raw is None:
        G.updateGeometry()
    wl = np.atleast_1d(np.asarray(MC.wavelength, dtype=np.float64))
    if np.any(np.isnan(wl)):
        raise ValueError("Error: No wavelength defined")
    if simType == 1:
        spectrum = np.array([float(MC.spectrumFunc(w)) for w in wl])
        spectrum = spectrum / spectrum.sum()
    else:
        spectrum = np.ones(wl.size)  # not read by the MEX when a source distribution is given
        if np.size(mdl.MC.NFR) <= 1:
            raise ValueError("Error: normalizedFluenceRate matrix not calculated for excitation light")
        eDC = mdl.MC.depositionCriteria
        if (any(getattr(eDC, k) != (0 if k.startswith("min") else math.inf) for k in _RESTRICTIVE)
                or eDC.onlyCollected):
            raise ValueError("The excitation step must be calculated without restrictive deposition criteria in order to calculate fluorescence.")
    DC = MC.depositionCriteria
    if DC.onlyCollected and not DC.evaluateOnlyAtEndOfLife:
        raise ValueError("Error: depositionCriteria.onlyCollected = true requires depositionCriteria.evaluateOnlyAtEndOfLife = true.")
    if MC.nExamplePaths != 0 and wl.size != 1:
        raise ValueError("Error: Example paths are not supported when simulating broadband illumination.")
    if DC.onlyCollected and not MC.useLightCollector:
        raise ValueError("Error: depositionCriteria.onlyCollected is true, but no light collector is defined")
    if MC.farFieldRes and MC.boundaryType == 0:
        raise ValueError("Error: If boundaryType == 0, no photons can escape to be registered in the far field. Set farFieldRes to zero or change boundaryType.")
    if MC.useLightCollector and MC.boundaryType == 0:
        raise ValueError("Error: If boundaryType == 0, no photons can escape to be registered on the light collector. Disable light collector or change boundaryType.")
    media = G.mediaPropertiesFunc(G.mediaPropParams)
    FR, T, FD = _fr_t_fd(mdl)
    mp = prep.optical_media_properties(media, G.M_raw, wl, MC.matchedInterfaces, G.dx, G.dy, G.dz, DC,
                                       MC.smoothingLengthScale, normals, FR=FR, T=T, FD=FD, downsample=downsample)
    if simType == 2:
        MC.sourceDistribution = prep.fluorescence_source(media, G.M_raw, mdl.MC.NA, mdl.MC.wavelength, wl, FR, T, FD)
    SD = MC.sourceDistribution
    if np.ndim(SD) == 0:
        sd = None
    else:
        sd = np.asarray(SD, dtype=np.float32)
        if sd.ndim == 3:
            sd = sd[..., None]
        if sd.shape != (G.nx, G.ny, G.nz, wl.size):
            raise ValueError("Error: model.MC.sourceDistribution must be of size [nx, ny, nz, nLambda]")
        if np.any(~np.isfinite(sd)) or np.any(sd < 0):
            raise ValueError("Error: model.MC.sourceDistribution must be real, finite and non-negative")
        if simType == 1:
            # runMonteCarlo.m:65 normalises the excitation source to unit integral; the
            # fluorescence source keeps its scale (each wavelength's power is its integral)
            sd = (sd / (G.dx * G.dy * G.dz * sd.sum(dtype=np.float64))).astype(np.float32)
        sd = np.asfortranarray(sd)
    LS = MC.lightSource
    if sd is None and LS.sourceType in (3, 4, 5):
        FP, AI = LS.FPID, LS.AID
        if LS.sourceType == 3 and (math.isnan(FP.radialWidth) or math.isnan(AI.radialWidth)):
            raise ValueError("Error: lightSource.focalPlaneIntensityDistribution.radialWidth and lightSource.angularIntensityDistribution.radialWidth must both be specified when sourceType is 3")
        if LS.sourceType == 4 and (np.isnan(_distr(FP.radialDistr)[0, 0]) or np.isnan(_distr(AI.radialDistr)[0, 0])):
            raise ValueError("Error: lightSource.focalPlaneIntensityDistribution.radialDistr and lightSource.angularIntensityDistribution.radialDistr must both be specified when sourceType is 4")
        if LS.sourceType == 5 and (np.isnan(_distr(FP.XDistr)[0, 0]) or np.isnan(_distr(FP.YDistr)[0, 0])
                                   or np.isnan(_distr(AI.XDistr)[0, 0]) or np.isnan(_distr(AI.YDistr)[0, 0])):
            raise ValueError("Error: X and Y distributions must be specified when sourceType is 5")
    LC = MC.lightCollector
    if MC.useLightCollector:
        if math.isfinite(LC.f):
            xLCC = LC.x - LC.f * math.sin(LC.theta) * math.cos(LC.phi)
            yLCC = LC.y - LC.f * math.sin(LC.theta) * math.sin(LC.phi)
            zLCC = LC.z - LC.f * math.cos(LC.theta)
        else:
            xLCC, yLCC, zLCC = LC.x, LC.y, LC.z
            if LC.res != 1:
                raise ValueError("Error: lightCollector.res must be 1 when lightCollector.f is Inf")
        if (abs(xLCC) < G.nx * G.dx / 2 and abs(yLCC) < G.ny * G.dy / 2 and abs(zLCC - G.nz * G.dz / 2) < G.nz * G.dz / 2):
            raise ValueError("Error: Light collector center (%.4f,%.4f,%.4f) is inside cuboid" % (xLCC, yLCC, zLCC))
    return dict(
        nx=G.nx, ny=G.ny, nz=G.nz, dx=G.dx, dy=G.dy, dz=G.dz,
        M=mp["M"], mua=mp["mua"], mus=mp["mus"], g=mp["g"], n=mp["n"], CDFidx=mp["CDFidx"],
        CDFs=mp["CDFs"], interfaceNormals=mp["interfaceNormals"], sourceDistribution=sd,
        spectrum=spectrum, wavelength=wl,
        nPhotonsRequested=float(MC.nPhotonsRequested), simulationTimeRequested=float(MC.simulationTimeRequested),
        requestCollectedPhotons=bool(MC.requestCollectedPhotons), calcNFR=bool(MC.calcNormalizedFluenceRate),
        useLightCollector=bool(MC.useLightCollector), silentMode=True, useAllCPUs=bool(MC.useAllCPUs),
        farFieldRes=int(MC.farFieldRes), boundaryType=int(MC.boundaryType), nExamplePaths=int(MC.nExamplePaths),
        GPUdevice=int(MC.GPUdevice), seed=int(MC.seed),
        LS=dict(sourceType=int(LS.sourceType), xFocus=float(LS.xFocus), yFocus=float(LS.yFocus), zFocus=float(LS.zFocus),
                theta=float(LS.theta), phi=float(LS.phi), psi=float(LS.psi), emitterLength=float(LS.emitterLength),
                FPID=dict(radialDistr=_distr(LS.FPID.radialDistr), radialWidth=float(LS.FPID.radialWidth),
                          XDistr=_distr(LS.FPID.XDistr), XWidth=float(LS.FPID.XWidth),
                          YDistr=_distr(LS.FPID.YDistr), YWidth=float(LS.FPID.YWidth)),
                AID=dict(radialDistr=_distr(LS.AID.radialDistr), radialWidth=float(LS.AID.radialWidth),
                         XDistr=_distr(LS.AID.XDistr), XWidth=float(LS.AID.XWidth),
                         YDistr=_distr(LS.AID.YDistr), YWidth=float(LS.AID.YWidth))),
        LC=dict(x=float(LC.x), y=float(LC.y), z=float(LC.z), theta=float(LC.theta), phi=float(LC.phi), f=float(LC.f),
                diam=float(LC.diam), fieldSize=float(LC.fieldSize), NA=float(LC.NA), res=float(LC.res),
                tStart=float(LC.tStart), tEnd=float(LC.tEnd), nTimeBins=float(LC.nTimeBins)),
        DC=dict(minScatterings=float(DC.minScatterings), maxScatterings=float(DC.maxScatterings),
                minRefractions=float(DC.minRefractions), maxRefractions=float(DC.maxRefractions),
                minReflections=float(DC.minReflections), maxReflections=float(DC.maxReflections),
                minInterfaceTransitions=float(DC.minInterfaceTransitions),
                maxInterfaceTransitions=float(DC.maxInterfaceTransitions),
                minSubmediaIdx=float(mp["minSubmediaIdx"]), maxSubmediaIdx=float(mp["maxSubmediaIdx"]),
                onlyCollected=bool(DC.onlyCollected), evaluateOnlyAtEndOfLife=bool(DC.evaluateOnlyAtEndOfLife)),
        mediaNames=mp["names"], simType=simType,
    )


def mex_model_tree(mc_in):
    """Nested property tree of an MCmatlab.model as MCmatlab.c's mexFunction reads it."""
    f32nan = np.array([[np.nan]], dtype=np.float32)
    MC = dict(
        silentMode=True, calcNFR=bool(mc_in["calcNFR"]),
        LS=dict(mc_in["LS"]),
        sourceDistribution=f32nan if mc_in["sourceDistribution"] is None else mc_in["sourceDistribution"],
        nPhotonsRequested=mc_in["nPhotonsRequested"], simulationTimeRequested=mc_in["simulationTimeRequested"],
        requestCollectedPhotons=mc_in["requestCollectedPhotons"],
        mediaProperties=dict(mua=np.asfortranarray(mc_in["mua"]), mus=np.asfortranarray(mc_in["mus"]),
                             g=np.asfortranarray(mc_in["g"]), n=np.asfortranarray(mc_in["n"]),
                             CDFidx=np.asfortranarray(mc_in["CDFidx"])),
        M=mc_in["M"], farFieldRes=float(mc_in["farFieldRes"]), boundaryType=float(mc_in["boundaryType"]),
        interfaceNormals=f32nan if mc_in["interfaceNormals"] is None else mc_in["interfaceNormals"],
        CDFs=np.asfortranarray(mc_in["CDFs"]) if np.size(mc_in["CDFs"]) else np.zeros((0, 0)),
        depositionCriteria=dict(mc_in["DC"]), LC=dict(mc_in["LC"]),
        useLightCollector=mc_in["useLightCollector"], nExamplePaths=float(mc_in["nExamplePaths"]),
        spectrum=np.asarray(mc_in["spectrum"], dtype=np.float64).reshape(1, -1),
        useAllCPUs=mc_in["useAllCPUs"], GPUdevice=float(mc_in["GPUdevice"]), seed=float(mc_in["seed"]),
    )
    G = dict(dx=float(mc_in["dx"]), dy=float(mc_in["dy"]), dz=float(mc_in["dz"]))
    if mc_in.get("simType", 1) == 2:
        return dict(MC=dict(), G=G, FMC=MC)
    return dict(MC=MC, G=G, FMC=dict())


def heat_mex_params(M1, A, E, c, dTdt_abs, useAllCPUs, heatBoundaryType, sensorIdx, sensorW,
                    lightsOn, steps, dt):
    """heatSimParameters as passed to finiteElementHeatPropagator (simulateHeatDistribution.m:209-211, :254-256)."""
    nS = 0 if sensorIdx is None else len(sensorIdx)
    return dict(
        M=np.asfortranarray((M1.astype(np.int16) - 1).astype(np.uint8)),
        A=np.asarray(A, dtype=np.float64).reshape(-1, 1),
        E=np.asarray(E, dtype=np.float64).reshape(-1, 1),
        dTdtperdeltaT=np.asfortranarray(np.asarray(c, dtype=np.float32)),
        dTdt_abs=np.asfortranarray(np.asarray(dTdt_abs, dtype=np.float32)),
        useAllCPUs=bool(useAllCPUs), heatBoundaryType=float(heatBoundaryType),
        tempSensorCornerIdxs=(np.zeros((0, 0)) if nS == 0 else np.asarray(sensorIdx, dtype=np.float64).reshape(-1, 1)),
        tempSensorInterpWeights=(np.zeros((0, 0)) if nS == 0 else np.asfortranarray(np.asarray(sensorW, dtype=np.float64))),
        lightsOn=bool(lightsOn), steps=float(steps), dt=float(dt),
    )
