"""model.simulateHeatDistribution: host flow of +MCmatlab/@model/simulateHeatDistribution.m on
the B200 stepper.

Follows the reference: thermal media (:31), per-medium initial maxima (:39-49), Omega set-up
(:52-59), time-step schedule (:61-110; dt limit x1.5, x15 with largeTimeSteps, or
HS.dtFactor when set), time vectors (:112-128), dT/dt arrays (:132), sensors (:135-150), then
for each pulse the illumination and diffusion phases and the end phase, each as nUpdates
stepper calls (:240-420). The grids stay resident on the GPU across the update calls
(mcb_heat_state_*); the reference re-uploads them on every MEX call. Every
HS.mediaPropRecalcPeriod updates the media are recalculated as heatSimParamsRecalc does
(:516-541): with temperature or damage dependent optical properties the MC (and the fluorescence
MC, if it ran) is re-run on the GPU at the current T and Omega, then the thermal media are
re-binned and the heat source rebuilt, and the stepper continues from the current grids.
Plotting and movies are not part of this library.
"""
from __future__ import annotations

import math

import numpy as np

from . import mexargs, native, prep


def initial_max_media_temps(T, M_raw, nM):
    """maxMediaTemps of a first heat run, one entry per unsplit medium present in the model
    (simulateHeatDistribution.m:38-47). As in the reference, entry i (1-based) is the maximum of T
    over the voxels whose raw medium index equals i, or -Inf where there is none."""
    M_raw = np.asarray(M_raw)
    T = np.asarray(T)
    out = np.full(nM, -np.inf)
    for i in range(1, nM + 1):
        sel = M_raw == i
        if sel.any():
            out[i - 1] = float(T[sel].max())
    return out


def fold_max_media_temps(maxT, new, nBins):
    """Folds the stepper's per-sub-medium maxima `new` into the per-medium maxima `maxT` in place:
    medium iM takes the maximum over its sub-media iSM .. iSM + nBins[iM] - 1
    (simulateHeatDistribution.m:268-272, :329-333, :390-394)."""
    new = np.asarray(new, dtype=np.float64).ravel()
    iSM = 0
    for iM, nb in enumerate(nBins):
        maxT[iM] = max(maxT[iM], float(new[iSM:iSM + nb].max()))
        iSM += nb
    return maxT


def simulateHeatDistribution(model):
    G = model.G
    HS = model.HS
    MC = model.MC
    if np.size(MC.normalizedFluenceRate) <= 1:
        raise ValueError("Error: MC.NFR was not calculated")
    G.updateGeometry()
    T = np.empty((G.nx, G.ny, G.nz), dtype=np.float32, order="F")
    T[...] = np.asarray(HS.T, dtype=np.float32)
    first = np.ndim(HS.maxMediaTemps) == 0 and math.isnan(HS.maxMediaTemps)
    media = G.mediaPropertiesFunc(G.mediaPropParams)
    dev = MC.GPUdevice

    def binning(par, nb):
        return native.downsample_params(par, nb, device=dev)

    def fd_grid():
        return (1 - np.exp(-np.asarray(HS.Omega, dtype=np.float64))).astype(np.float32) if np.ndim(HS.Omega) else np.float32(0.0)
    th = prep.thermal_media_properties(media, G.M_raw, T, fd_grid(), downsample=binning)
    HS.mediaProperties = {"name": th["names"], "VHC": th["VHC"], "TC": th["TC"], "A": th["A"], "E": th["E"]}
    HS.M = th["M"]
    if first:
        HS.maxMediaTemps = initial_max_media_temps(T, G.M_raw, len(th["nBins"]))
    damage = bool(np.any(th["A"]))
    if damage:
        if first or np.ndim(HS.Omega) == 0:
            HS.Omega = np.zeros((G.nx, G.ny, G.nz), dtype=np.float32, order="F")
    else:
        HS.Omega = np.float32(np.nan)
    if HS.nPulses != 1 and (HS.durationOn == 0 or HS.durationOff == 0):
        raise ValueError("Error: If either on-duration or off-duration is 0, nPulses must be 1")
    factor = HS.dtFactor if not math.isnan(HS.dtFactor) else (15.0 if HS.largeTimeSteps else 1.5)
    dtmax = prep.calc_dtmax(th["M"], th["TC"], th["VHC"], G.dx, G.dy, G.dz) * factor
    sched = prep.heat_schedule(HS.durationOn, HS.durationOff, HS.durationEnd, HS.nUpdates, dtmax)
    (nUon, nTon, dtOn), (nUoff, nToff, dtOff), (nUend, nTend, dtEnd) = sched["on"], sched["off"], sched["end"]
    t_off = 0.0 if first or np.ndim(HS.sensorsTimeVector) == 0 else float(np.asarray(HS.sensorsTimeVector)[-1])
    tv = [0.0]
    for j in range(HS.nPulses):
        base = (HS.durationOn + HS.durationOff) * j
        tv += list(base + np.arange(1, nUon * nTon + 1) * dtOn)
        tv += list(base + HS.durationOn + np.arange(1, nUoff * nToff + 1) * dtOff)
    tv += list((HS.durationOn + HS.durationOff) * HS.nPulses + np.arange(1, nUend * nTend + 1) * dtEnd)
    tv = t_off + np.array(tv)
    if first or np.ndim(HS.sensorsTimeVector) == 0:
        HS.sensorsTimeVector = tv
    else:
        HS.sensorsTimeVector = np.concatenate([np.asarray(HS.sensorsTimeVector)[:-1], tv])
    NA = np.asarray(MC.normalizedAbsorption, dtype=np.float64)
    NA_sum = NA.sum(axis=3) if NA.ndim == 4 else NA
    c, Q = prep.calc_dTdt_arrays(th["VHC"], th["TC"], G.dx, G.dy, G.dz, NA_sum, MC.P, th["M"])
    pos = HS.tempSensorPositions
    if pos is not None and np.size(pos):
        pos = np.atleast_2d(np.asarray(pos, dtype=np.float64))
        if (np.any(np.abs(pos[:, 0]) > G.dx * G.nx / 2) or np.any(np.abs(pos[:, 1]) > G.dy * G.ny / 2)
                or np.any(np.abs(pos[:, 2]) - G.dz * G.nz / 2 > G.dz * G.nz / 2)):
            raise ValueError("Error: A temperature sensor is outside the cuboid.")
        li, w = prep.convert_temp_sensor_pos(pos, G.x, G.y, G.z)
    else:
        li, w = None, None
    sensorTemps = None if first or np.ndim(HS.sensorTemps) == 0 else np.asarray(HS.sensorTemps)

    def params(lightsOn, steps, dt):
        return mexargs.heat_mex_params(th["M"], th["A"], th["E"], c, Q, HS.useAllCPUs, HS.heatBoundaryType, li, w,
                                       lightsOn, steps, dt)

    state = native.HeatState(T, HS.Omega if damage else None, params(True, 1, dtOn), G.nx, G.ny, G.nz,
                             device=dev)
    maxT = np.asarray(HS.maxMediaTemps, dtype=np.float64).copy()
    period = int(HS.mediaPropRecalcPeriod)
    FRd, Td, FDd = prep.dependence_flags([media[int(m) - 1] for m in np.unique(G.M_raw)])
    thmT, thmFD = prep.thermal_dependence_flags([media[int(m) - 1] for m in np.unique(G.M_raw)])
    opt_dep = bool(np.any(Td | FDd))
    thm_dep = bool(np.any(thmT | thmFD))

    def recalc():
        """heatSimParamsRecalc (simulateHeatDistribution.m:516-541) at the current grids."""
        nonlocal state, th, c, Q, generation
        generation += 1
        Tc, Oc = state.read()
        HS.T = Tc
        if damage:
            HS.Omega = Oc
        if opt_dep:
            silent = MC.silentMode
            MC.silentMode = True
            model.runMonteCarlo()
            MC.silentMode = silent
            if not math.isnan(model.FMC.simulationTime):
                model.runMonteCarlo("fluorescence")
        if opt_dep or thm_dep:
            th = prep.thermal_media_properties(media, G.M_raw, Tc, fd_grid(), downsample=binning)
            HS.mediaProperties = {"name": th["names"], "VHC": th["VHC"], "TC": th["TC"], "A": th["A"], "E": th["E"]}
            HS.M = th["M"]
        NA = np.asarray(MC.normalizedAbsorption, dtype=np.float64)
        c, Q = prep.calc_dTdt_arrays(th["VHC"], th["TC"], G.dx, G.dy, G.dz, NA.sum(axis=3) if NA.ndim == 4 else NA,
                                     MC.P, th["M"])
        state.close()
        state = native.HeatState(Tc, Oc if damage else None, params(True, 1, dtOn), G.nx, G.ny, G.nz, device=dev)

    generation = 0

    def run(n_updates, steps, dt, lights, first_idx):
        nonlocal sensorTemps
        hp, built = params(lights, steps, dt), generation
        for i in range(n_updates):
            if built != generation:  # media recalculated: new media grid, coefficients and source
                hp, built = params(lights, steps, dt), generation
            sens, mx = state.step(hp)
            fold_max_media_temps(maxT, mx, th["nBins"])
            if li is not None:
                sensorTemps = sens if sensorTemps is None else np.concatenate([sensorTemps[:, :-1], sens], axis=1)
            if period > 0 and (first_idx + i + 1) % period == 0:
                recalc()

    try:
        per_pulse = nUon + nUoff
        for j in range(HS.nPulses):
            if HS.durationOn != 0:
                run(nUon, nTon, dtOn, True, j * per_pulse)
            if HS.durationOff != 0:
                run(nUoff, nToff, dtOff, False, j * per_pulse + nUon)
        run(nUend, nTend, dtEnd, False, HS.nPulses * per_pulse)
        Tn, On = state.read()
    finally:
        state.close()
    HS.T = Tn
    if damage:
        HS.Omega = On
    HS.maxMediaTemps = maxT
    HS.sensorTemps = sensorTemps if sensorTemps is not None else np.nan
    return model
