"""ctypes mirrors of the POD structs in include/mcb200.h and fillers from MEX-level inputs.

`McModelBuffers(mc_in)` converts the flat dict produced by mexargs.prepare_mc into an
mcb_mc_model (keeping the numpy buffers alive), and `McResultBuffers` allocates the
output arrays with the sizes MCmatlab.c's mexFunction allocates (MCmatlab.c:461-493).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

KILLRANGE = 5
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)


class mcb_distr(C.Structure):
    _fields_ = [("values", _dp), ("n", C.c_int64), ("width", C.c_double)]


class mcb_mc_model(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("M", C.POINTER(C.c_uint8)),
        ("nM", C.c_int32), ("nL", C.c_int32),
        ("mua", _dp), ("mus", _dp), ("g", _dp), ("n", _dp), ("CDFidx", _dp),
        ("CDFs", _dp), ("nCDFelems", C.c_int64),
        ("interfaceNormals", _fp), ("sourceDistribution", _fp), ("spectrum", _dp),
        ("nPhotonsRequested", C.c_double), ("simulationTimeRequested", C.c_double),
        ("requestCollectedPhotons", C.c_int32), ("calcNFR", C.c_int32), ("useLightCollector", C.c_int32),
        ("farFieldRes", C.c_int32), ("boundaryType", C.c_int32), ("nExamplePaths", C.c_int32),
        ("seed", C.c_uint64),
        ("sourceType", C.c_int32),
        ("xFocus", C.c_double), ("yFocus", C.c_double), ("zFocus", C.c_double),
        ("theta", C.c_double), ("phi", C.c_double), ("psi", C.c_double), ("emitterLength", C.c_double),
        ("FPID_radial", mcb_distr), ("FPID_X", mcb_distr), ("FPID_Y", mcb_distr),
        ("AID_radial", mcb_distr), ("AID_X", mcb_distr), ("AID_Y", mcb_distr),
        ("LC_x", C.c_double), ("LC_y", C.c_double), ("LC_z", C.c_double), ("LC_theta", C.c_double),
        ("LC_phi", C.c_double), ("LC_f", C.c_double), ("LC_diam", C.c_double), ("LC_fieldSize", C.c_double),
        ("LC_NA", C.c_double), ("LC_tStart", C.c_double), ("LC_tEnd", C.c_double),
        ("LC_res", C.c_int32), ("LC_nTimeBins", C.c_int32),
        ("DC_minScatterings", C.c_double), ("DC_maxScatterings", C.c_double),
        ("DC_minRefractions", C.c_double), ("DC_maxRefractions", C.c_double),
        ("DC_minReflections", C.c_double), ("DC_maxReflections", C.c_double),
        ("DC_minInterfaceTransitions", C.c_double), ("DC_maxInterfaceTransitions", C.c_double),
        ("DC_minSubmediaIdx", C.c_double), ("DC_maxSubmediaIdx", C.c_double),
        ("DC_onlyCollected", C.c_int32), ("DC_evaluateOnlyAtEndOfLife", C.c_int32),
        ("packetOffset", C.c_uint64), ("packetStride", C.c_uint64),
    ]


class mcb_mc_result(C.Structure):
    _fields_ = [
        ("NFR", _fp), ("image", _fp), ("farField", _fp),
        ("NI_xpos", _fp), ("NI_xneg", _fp), ("NI_ypos", _fp), ("NI_yneg", _fp), ("NI_zpos", _fp), ("NI_zneg", _fp),
        ("examplePaths", _dp), ("examplePathsCap", C.c_int64),
        ("examplePathsN", C.c_int64),
        ("nPhotons", C.c_double), ("nPhotonsCollected", C.c_double), ("nThreads", C.c_double),
        ("simulationTime", C.c_double),
        ("propagationSteps", C.c_uint64), ("kernelMs", C.c_double),
        ("freeStepCuts", C.c_double), ("freeStepCutWeight", C.c_double),
        ("tallies", _dp),
    ]


class mcb_mc_launch(C.Structure):
    _fields_ = [("refillMin", C.c_int32), ("scatterMin", C.c_int32)]


class mcb_mc_objectives(C.Structure):
    _fields_ = [("nRadialBins", C.c_int32), ("radialBinWidth", C.c_double), ("box", C.c_int32 * 6)]


class mcb_mc_grad_result(C.Structure):
    _fields_ = [("R", _dp), ("dR_dmua", _dp), ("dR_dmus", _dp), ("F", C.c_double), ("dF_dmua", _dp), ("dF_dmus", _dp)]


class GradBuffers:
    """Objectives and derivative outputs of a perturbation-MC run."""

    def __init__(self, nM, nRadialBins, radialBinWidth, box):
        self.obj = mcb_mc_objectives()
        self.obj.nRadialBins = int(nRadialBins)
        self.obj.radialBinWidth = float(radialBinWidth)
        for q in range(6):
            self.obj.box[q] = int(box[q]) if box is not None else 0
        nR = max(int(nRadialBins), 1)
        self.R = np.zeros(nR)
        self.dR_dmua = np.zeros(nR * nM)
        self.dR_dmus = np.zeros(nR * nM)
        self.dF_dmua = np.zeros(nM)
        self.dF_dmus = np.zeros(nM)
        g = mcb_mc_grad_result()
        g.R = _ptr(self.R, C.c_double)
        g.dR_dmua = _ptr(self.dR_dmua, C.c_double)
        g.dR_dmus = _ptr(self.dR_dmus, C.c_double)
        g.dF_dmua = _ptr(self.dF_dmua, C.c_double)
        g.dF_dmus = _ptr(self.dF_dmus, C.c_double)
        self.res = g
        self.nR = int(nRadialBins)
        self.nM = nM

    def outputs(self):
        nR, nM = self.nR, self.nM
        return {"R": self.R[:nR].copy(), "dR_dmua": self.dR_dmua[:nR * nM].reshape(nR, nM, order="F"),
                "dR_dmus": self.dR_dmus[:nR * nM].reshape(nR, nM, order="F"), "F": self.res.F,
                "dF_dmua": self.dF_dmua.copy(), "dF_dmus": self.dF_dmus.copy()}


class mcb_heat_params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("nM", C.c_int32),
        ("M", C.POINTER(C.c_uint8)), ("dTdtperdeltaT", _fp), ("dTdt_abs", _fp),
        ("A", _dp), ("E", _dp),
        ("lightsOn", C.c_int32), ("heatBoundaryType", C.c_int32),
        ("steps", C.c_int64), ("dt", C.c_double),
        ("nSensors", C.c_int32),
        ("tempSensorCornerIdxs", _dp), ("tempSensorInterpWeights", _dp),
    ]


class mcb_heat_objective(C.Structure):
    _fields_ = [("damageWeight", _fp), ("peakWeight", _fp)]


class mcb_heat_grad(C.Structure):
    _fields_ = [("J", C.c_double), ("J_damage", C.c_double), ("J_peak", C.c_double), ("dJ_dc", _dp),
                ("dJ_dQ", _fp), ("dJ_dT0", _fp), ("forwardMs", C.c_double), ("adjointMs", C.c_double)]


def _ptr(a, ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


def _col(a, dtype):
    """Column-major contiguous copy (MATLAB order) flattened to 1-D."""
    return np.ascontiguousarray(np.asarray(a, dtype=dtype).reshape(-1, order="F"))


class McModelBuffers:
    """An mcb_mc_model filled from a prepare_mc dict; holds references to every buffer it points at."""

    def __init__(self, mc_in):
        self.keep = []
        m = mcb_mc_model()
        m.nx, m.ny, m.nz = mc_in["nx"], mc_in["ny"], mc_in["nz"]
        m.dx, m.dy, m.dz = mc_in["dx"], mc_in["dy"], mc_in["dz"]
        M = _col(mc_in["M"], np.uint8)
        self.keep.append(M)
        m.M = _ptr(M, C.c_uint8)
        nM, nL = np.asarray(mc_in["mua"]).shape
        m.nM, m.nL = nM, nL
        for name in ("mua", "mus", "g", "n", "CDFidx"):
            a = _col(mc_in[name], np.float64)
            self.keep.append(a)
            setattr(m, name, _ptr(a, C.c_double))
        if np.size(mc_in["CDFs"]):
            cd = _col(mc_in["CDFs"], np.float64)
            self.keep.append(cd)
            m.CDFs, m.nCDFelems = _ptr(cd, C.c_double), cd.size
        else:
            m.CDFs, m.nCDFelems = _ptr(None, C.c_double), 0
        if mc_in["interfaceNormals"] is not None:
            nrm = _col(mc_in["interfaceNormals"], np.float32)
            self.keep.append(nrm)
            m.interfaceNormals = _ptr(nrm, C.c_float)
        else:
            m.interfaceNormals = _ptr(None, C.c_float)
        if mc_in["sourceDistribution"] is not None:
            sd = _col(mc_in["sourceDistribution"], np.float32)
            self.keep.append(sd)
            m.sourceDistribution = _ptr(sd, C.c_float)
        else:
            m.sourceDistribution = _ptr(None, C.c_float)
        sp = np.ascontiguousarray(np.asarray(mc_in["spectrum"], dtype=np.float64).ravel())
        self.keep.append(sp)
        m.spectrum = _ptr(sp, C.c_double)
        m.nPhotonsRequested = mc_in["nPhotonsRequested"]
        m.simulationTimeRequested = mc_in["simulationTimeRequested"]
        m.requestCollectedPhotons = int(mc_in["requestCollectedPhotons"])
        m.calcNFR = int(mc_in["calcNFR"])
        m.useLightCollector = int(mc_in["useLightCollector"])
        m.farFieldRes = int(mc_in["farFieldRes"])
        m.boundaryType = int(mc_in["boundaryType"])
        m.nExamplePaths = int(mc_in["nExamplePaths"])
        m.seed = int(mc_in["seed"]) & 0xFFFFFFFFFFFFFFFF
        LS = mc_in["LS"]
        m.sourceType = LS["sourceType"]
        for k in ("xFocus", "yFocus", "zFocus", "theta", "phi", "psi", "emitterLength"):
            setattr(m, k, LS[k])
        for grp, key in (("FPID", "FPID"), ("AID", "AID")):
            for ax, wk in (("radial", "radialWidth"), ("X", "XWidth"), ("Y", "YWidth")):
                vals = np.ascontiguousarray(np.asarray(LS[key][ax + "Distr"], dtype=np.float64).ravel())
                self.keep.append(vals)
                d = mcb_distr(_ptr(vals, C.c_double), vals.size, LS[key][wk])
                setattr(m, "%s_%s" % (grp, ax), d)
        LC = mc_in["LC"]
        m.LC_x, m.LC_y, m.LC_z = LC["x"], LC["y"], LC["z"]
        m.LC_theta, m.LC_phi, m.LC_f = LC["theta"], LC["phi"], LC["f"]
        m.LC_diam, m.LC_fieldSize, m.LC_NA = LC["diam"], LC["fieldSize"], LC["NA"]
        m.LC_tStart, m.LC_tEnd = LC["tStart"], LC["tEnd"]
        m.LC_res, m.LC_nTimeBins = int(LC["res"]), int(LC["nTimeBins"])
        DC = mc_in["DC"]
        for k in ("minScatterings", "maxScatterings", "minRefractions", "maxRefractions", "minReflections",
                  "maxReflections", "minInterfaceTransitions", "maxInterfaceTransitions", "minSubmediaIdx",
                  "maxSubmediaIdx"):
            setattr(m, "DC_" + k, float(DC[k]))
        m.DC_onlyCollected = int(DC["onlyCollected"])
        m.DC_evaluateOnlyAtEndOfLife = int(DC["evaluateOnlyAtEndOfLife"])
        m.packetOffset = int(mc_in.get("packetOffset", 0))
        m.packetStride = int(mc_in.get("packetStride", 1))
        self.model = m
        self.mc_in = mc_in


def result_shapes(mc_in):
    """MATLAB shapes of the tallied outputs of one MC call, as MCmatlab.c allocates them
    (:461-493); every shape carries the wavelength as its last axis."""
    nx, ny, nz = mc_in["nx"], mc_in["ny"], mc_in["nz"]
    nL = np.asarray(mc_in["mua"]).shape[1]
    bt = mc_in["boundaryType"]
    sd = mc_in["sourceDistribution"] is not None
    LC = mc_in["LC"]
    nTB = 0 if sd else int(LC["nTimeBins"])
    res = int(LC["res"])
    shapes = {}
    if mc_in["calcNFR"]:
        shapes["NFR"] = (nx, ny, nz, nL)
    if mc_in["useLightCollector"]:
        shapes["image"] = (res, res, nTB + 2 if nTB else 1, nL)
    ffr = int(mc_in["farFieldRes"])
    if ffr:
        shapes["farField"] = (ffr, ffr, nL)
    if bt == 1:
        shapes.update(NI_xpos=(ny, nz, nL), NI_xneg=(ny, nz, nL), NI_ypos=(nx, nz, nL),
                      NI_yneg=(nx, nz, nL), NI_zpos=(nx, ny, nL), NI_zneg=(nx, ny, nL))
    elif bt == 2:
        shapes["NI_zneg"] = (KILLRANGE * nx, KILLRANGE * ny, nL)
    elif bt == 3:
        shapes.update(NI_zpos=(nx, ny, nL), NI_zneg=(nx, ny, nL))
    return shapes


class McResultBuffers:
    """Output arrays sized as MCmatlab.c allocates them (:461-493), returned in MATLAB shapes."""

    def __init__(self, mc_in, example_cap=0, tally_count=0):
        self.shapes = result_shapes(mc_in)
        self.arrays = {k: np.zeros(int(np.prod(s)), dtype=np.float32) for k, s in self.shapes.items()}
        r = mcb_mc_result()
        for k, a in self.arrays.items():
            setattr(r, k, _ptr(a, C.c_float))
        self.paths = np.zeros(4 * max(example_cap, 1), dtype=np.float64)
        r.examplePaths = _ptr(self.paths, C.c_double)
        r.examplePathsCap = example_cap
        self.tallies = np.zeros(tally_count, dtype=np.float64) if tally_count else None
        if tally_count:
            r.tallies = _ptr(self.tallies, C.c_double)
        self.result = r

    def outputs(self):
        out = {k: self.arrays[k].reshape(s, order="F") for k, s in self.shapes.items()}
        r = self.result
        out["nPhotons"] = r.nPhotons
        out["nPhotonsCollected"] = r.nPhotonsCollected
        out["nThreads"] = r.nThreads
        out["simulationTime"] = r.simulationTime
        out["propagationSteps"] = int(r.propagationSteps)
        out["kernelMs"] = r.kernelMs
        out["freeStepCuts"] = r.freeStepCuts
        out["freeStepCutWeight"] = r.freeStepCutWeight
        if self.tallies is not None:
            out["tallies"] = self.tallies
        n = int(r.examplePathsN)
        out["examplePaths"] = self.paths[:4 * n].reshape(4, n, order="F") if n else np.zeros((4, 0))
        return out


class HeatParamBuffers:
    """An mcb_heat_params filled from the heatSimParameters dict of mexargs.heat_mex_params."""

    def __init__(self, nx, ny, nz, hp):
        self.keep = []
        p = mcb_heat_params()
        p.nx, p.ny, p.nz = nx, ny, nz
        c = _col(hp["dTdtperdeltaT"], np.float32)
        nM = int(round((c.size // 3) ** 0.5))
        p.nM = nM
        M = _col(hp["M"], np.uint8)
        Q = _col(hp["dTdt_abs"], np.float32)
        A = _col(hp["A"], np.float64)
        E = _col(hp["E"], np.float64)
        self.keep += [c, M, Q, A, E]
        p.M, p.dTdtperdeltaT, p.dTdt_abs = _ptr(M, C.c_uint8), _ptr(c, C.c_float), _ptr(Q, C.c_float)
        p.A, p.E = _ptr(A, C.c_double), _ptr(E, C.c_double)
        p.lightsOn = int(bool(hp["lightsOn"]))
        p.heatBoundaryType = int(hp["heatBoundaryType"])
        p.steps = int(hp["steps"])
        p.dt = float(hp["dt"])
        idx = np.asarray(hp["tempSensorCornerIdxs"], dtype=np.float64).ravel()
        nS = idx.size
        p.nSensors = nS
        if nS:
            w = _col(hp["tempSensorInterpWeights"], np.float64)
            idx = np.ascontiguousarray(idx)
            self.keep += [idx, w]
            p.tempSensorCornerIdxs, p.tempSensorInterpWeights = _ptr(idx, C.c_double), _ptr(w, C.c_double)
        else:
            p.tempSensorCornerIdxs = _ptr(None, C.c_double)
            p.tempSensorInterpWeights = _ptr(None, C.c_double)
        self.params = p
        self.nM = nM
        self.nS = nS
