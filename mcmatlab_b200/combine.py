"""combineModels: merging the results of several runs of one model
(+MCmatlab/@model/combineModels.m:1-196).

The runs must share the geometry (:7-17), have run (:20-24) and share the listed MC (or FMC)
settings and light-collector settings (:27-57, :121-157). For 'MC', outputs are averaged with
weights nPhotons, or with weights P when the light sources or powers differ (then P adds up
and the light source is left empty, :40-112); for 'FMC' the excitation MC objects must be
identical and the weights are nPhotons (:117-195). Times and packet counts add, example paths
concatenate. The arithmetic follows MATLAB's for single-precision outputs and double weights:
the weight ratio is rounded to single, products and sums are single.

The reference's `reset(model,'FMC')` / `reset(model,'HS')` calls (:62-63, :160) discard their
result (the model is a value object), so the first model's other sub-objects are kept, as here.
"""
from __future__ import annotations

import copy
import dataclasses
import math

import numpy as np

_G_PROPS = ("nx", "ny", "nz", "Lx", "Ly", "Lz", "mediaPropertiesFunc", "mediaPropParams", "geomFunc", "geomFuncParams")
_MC_PROPS = ("calcNormalizedFluenceRate", "farFieldRes", "matchedInterfaces", "smoothingLengthScale", "boundaryType",
             "wavelength", "useLightCollector", "depositionCriteria")
_FMC_PROPS = _MC_PROPS[:-1]
_LC_PROPS = ("x", "y", "z", "theta", "phi", "f", "diam", "fieldSize", "NA", "res", "tStart", "tEnd", "nTimeBins")
_OUTPUTS = ("normalizedFluenceRate", "farField", "normalizedIrradiance_xpos", "normalizedIrradiance_xneg",
            "normalizedIrradiance_ypos", "normalizedIrradiance_yneg", "normalizedIrradiance_zpos",
            "normalizedIrradiance_zneg")


def isequaln(a, b):
    """MATLAB's isequaln: equal values, NaN equal to NaN, compared through nested objects."""
    if a is b:
        return True
    if callable(a) or callable(b):
        return False
    if dataclasses.is_dataclass(a) and dataclasses.is_dataclass(b):
        return type(a) is type(b) and all(isequaln(getattr(a, f.name), getattr(b, f.name))
                                          for f in dataclasses.fields(a))
    if isinstance(a, dict) and isinstance(b, dict):
        return a.keys() == b.keys() and all(isequaln(a[k], b[k]) for k in a)
    if isinstance(a, (list, tuple)) and isinstance(b, (list, tuple)):
        return len(a) == len(b) and all(isequaln(x, y) for x, y in zip(a, b))
    if isinstance(a, str) or isinstance(b, str):
        return a == b
    try:
        x, y = np.asarray(a), np.asarray(b)
    except Exception:
        return a == b
    if x.shape != y.shape and not (x.size == y.size == 1):
        return False
    if x.dtype.kind in "fc" or y.dtype.kind in "fc":
        return bool(np.array_equal(x.reshape(-1), y.reshape(-1), equal_nan=True))
    return bool(np.array_equal(x.reshape(-1), y.reshape(-1)))


def _f32(x):
    return np.asarray(x, dtype=np.float32) if np.ndim(x) else np.float32(x)


def _check_same(objs, props, what):
    for p in props:
        if not all(isequaln(getattr(o, p), getattr(objs[0], p)) for o in objs[1:]):
            raise ValueError("Error: The %s %s properties are not identical, so the objects cannot be combined." % (what, p))


def _merge(sims, weights, out):
    """Weighted sum of the normalised outputs of `sims` into `out` (MATLAB single arithmetic),
    then renormalised by w1 / wTot."""
    w1 = weights[0]
    for s, w in zip(sims[1:], weights[1:]):
        out.simulationTime = out.simulationTime + s.simulationTime
        out.nPhotons = out.nPhotons + s.nPhotons
        out.nPhotonsCollected = out.nPhotonsCollected + s.nPhotonsCollected
        out.examplePaths = np.concatenate([np.atleast_2d(out.examplePaths), np.atleast_2d(s.examplePaths)], axis=1)
        r = np.float32(w / w1)
        out.lightCollector.image = _f32(out.lightCollector.image) + r * _f32(s.lightCollector.image)
        for k in _OUTPUTS:
            setattr(out, k, _f32(getattr(out, k)) + r * _f32(getattr(s, k)))
    return w1


def _renormalise(out, w1, wTot):
    a, b = np.float32(w1), np.float32(wTot)
    out.lightCollector.image = (_f32(out.lightCollector.image) * a) / b
    for k in _OUTPUTS:
        setattr(out, k, (_f32(getattr(out, k)) * a) / b)


def combineModels(modelArray, simType):
    """Returns a new model holding the merged results of modelArray (simType 'MC' or 'FMC')."""
    models = list(modelArray)
    if not models:
        raise ValueError("Error: no models to combine")
    _check_same([m.G for m in models], _G_PROPS, "G")
    for m in models:
        if m.MC.nPhotons is None or (isinstance(m.MC.nPhotons, float) and math.isnan(m.MC.nPhotons)):
            raise ValueError("Error: All input models must have had their MC simulation executed using runMonteCarlo() before combining.")
    _check_same([m.MC for m in models], _MC_PROPS, "MC")
    same_sources = all(isequaln(m.MC.lightSource, models[0].MC.lightSource) and isequaln(m.MC.P, models[0].MC.P)
                       for m in models[1:])
    _check_same([m.MC.lightCollector for m in models], _LC_PROPS, "light collector")
    out = copy.deepcopy(models[0])
    if simType == "MC":
        if not same_sources:
            for m in models:
                if m.MC.P is None or math.isnan(m.MC.P):
                    raise ValueError("Error: If the light source definitions are not identical, all input models must have the MC.P (power) property specified. These do not need to be the correct absolute power values, but must have the correct relative power values.")
            weights = [m.MC.P for m in models]
        else:
            weights = [m.MC.nPhotons for m in models]
        w1 = _merge([m.MC for m in models], weights, out.MC)
        if not same_sources:
            out.MC.P = sum(weights)
            out.MC.lightSource = None  # a combination of light sources is represented by none
            wTot = out.MC.P
        else:
            wTot = out.MC.nPhotons
        _renormalise(out.MC, w1, wTot)
    elif simType == "FMC":
        for m in models[1:]:
            if not isequaln(m.MC, models[0].MC):
                raise ValueError("Error: The MC objects must all be identical for the FMC objects to be combined.")
        for m in models:
            if m.FMC.nPhotons is None or (isinstance(m.FMC.nPhotons, float) and math.isnan(m.FMC.nPhotons)):
                raise ValueError("Error: All input models must have had their FMC simulation executed using runMonteCarlo() before combining.")
        _check_same([m.FMC for m in models], _FMC_PROPS, "FMC")
        _check_same([m.FMC.lightCollector for m in models], _LC_PROPS, "FMC light collector")
        weights = [m.FMC.nPhotons for m in models]
        w1 = _merge([m.FMC for m in models], weights, out.FMC)
        _renormalise(out.FMC, w1, out.FMC.nPhotons)
    else:
        raise ValueError("Error: simType must be 'MC' or 'FMC'")
    return out


def merge_tallies(mc_in, runs, device=0):
    """Exact merging of runs of one model (MEX-level inputs mc_in) on disjoint packet ranges, e.g.
    a run continued later with packetOffset = the packets already run: the runs' FP64 tallies
    (native.mc_run(..., tallies=True)) are added and normalised once (mcb_mc_normalize), which
    gives the outputs of one run over the union of the packets up to FP64 summation order.
    combineModels merges the runs' normalised single-precision outputs instead."""
    from . import native
    total = None
    for r in runs:
        t = np.asarray(r["tallies"], dtype=np.float64)
        total = t.copy() if total is None else total + t
    return native.mc_normalize(mc_in, total, device=device)
