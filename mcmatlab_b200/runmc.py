"""model.runMonteCarlo: host flow of +MCmatlab/@model/runMonteCarlo.m on the B200 library.

Steps (runMonteCarlo.m line numbers): geometry update (:51-52), spectrum and distributed-source
normalisation (:59-65), input checks (:220-375) and media preparation
(getOpticalMediaProperties) in mexargs.prepare_mc, the MEX call (:174) replaced by
mcb_mc_run, then the light-collector and far-field axes (:182-216).

`runMonteCarlo(model, 'fluorescence')` (simType 2) runs the fluorescence step: the source is
built from the excitation results in model.MC (:119-166) and the run's settings and results
live in model.FMC, as in the reference.
"""
from __future__ import annotations

import math

import numpy as np

from . import mexargs, native


def _squeeze_last(a, nL):
    return a[..., 0] if (a is not None and nL == 1 and a.ndim >= 3) else a


def runMonteCarlo(model, *args):
    simType = 2 if "fluorescence" in args else 1
    MC = model.FMC if simType == 2 else model.MC
    model.G.updateGeometry()
    if simType == 1 and MC.FRdepIterations > 0:
        # fluence-rate dependent media: nIterations runs with 1/2^(n-1), ..., 1/2, 1 of the
        # requested packets (or time), each re-binning the media on the previous fluence rate
        # (runMonteCarlo.m:81-113)
        nIt = int(MC.FRdepIterations)
        timed = math.isnan(MC.nPhotonsRequested)
        req = MC.simulationTimeRequested if timed else MC.nPhotonsRequested
        for i in range(nIt):
            part = req * 0.5 ** (nIt - 1 - i)
            if timed:
                MC.simulationTimeRequested = part
            else:
                MC.nPhotonsRequested = part
            _run_once(model, simType)
            if i < nIt - 1:
                MC.FR = MC.P * np.asarray(MC.NFR)
        if timed:
            MC.simulationTimeRequested = req
        else:
            MC.nPhotonsRequested = req
        return model
    return _run_once(model, simType)


def _run_once(model, simType):
    MC = model.FMC if simType == 2 else model.MC
    dev = MC.GPUdevice
    mc_in = mexargs.prepare_mc(model, simType, normals=lambda *a: native.interface_normals(*a, device=dev),
                               downsample=lambda par, nb: native.downsample_params(par, nb, device=dev))
    out = native.mc_run(mc_in, device=dev)
    nL = np.asarray(mc_in["mua"]).shape[1]
    if simType == 1:
        MC.spectrum = mc_in["spectrum"]
    MC.mediaProperties = {"name": mc_in["mediaNames"], "mua": mc_in["mua"], "mus": mc_in["mus"], "g": mc_in["g"],
                          "n": mc_in["n"], "CDFidx": mc_in["CDFidx"]}
    MC.M = mc_in["M"]
    MC.CDFs = mc_in["CDFs"]
    MC.interfaceNormals = mc_in["interfaceNormals"] if mc_in["interfaceNormals"] is not None else np.float32(np.nan)
    if mc_in["calcNFR"]:
        MC.normalizedFluenceRate = _squeeze_last(out["NFR"], nL)
    if mc_in["farFieldRes"]:
        MC.farField = out["farField"][..., 0] if nL == 1 else out["farField"]
        r = mc_in["farFieldRes"]
        MC.farFieldTheta = np.linspace(math.pi / r / 2, math.pi - math.pi / r / 2, r)
        MC.farFieldPhi = np.linspace(-math.pi + 2 * math.pi / r / 2, math.pi - 2 * math.pi / r / 2, r)
    for face in ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg"):
        k = "NI_" + face
        if k in out:
            setattr(MC, "normalizedIrradiance_" + face, out[k][..., 0] if nL == 1 else out[k])
    if mc_in["useLightCollector"]:
        img = out["image"]
        LC = MC.lightCollector
        LC.image = float(img.ravel()[0]) if img.size == 1 else np.squeeze(img)
        if LC.res > 1:
            LC.X = np.linspace(LC.fieldSize * (1 / LC.res - 1), LC.fieldSize * (1 - 1 / LC.res), LC.res) / 2
            LC.Y = LC.X
        if LC.nTimeBins > 0:
            LC.t = (np.arange(-0.5, LC.nTimeBins + 1.5)) * (LC.tEnd - LC.tStart) / LC.nTimeBins + LC.tStart
    MC.nPhotons = out["nPhotons"]
    MC.nPhotonsCollected = out["nPhotonsCollected"]
    MC.nThreads = out["nThreads"]
    MC.simulationTime = out["simulationTime"]
    if mc_in["nExamplePaths"]:
        MC.examplePaths = out["examplePaths"]
    MC.kernelStats = {"propagationSteps": out["propagationSteps"], "kernelMs": out["kernelMs"]}
    return model
