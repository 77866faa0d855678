"""ctypes access to the FP64 CPU restatements in oracle/_ref/liboracle.so.

TEST INFRASTRUCTURE ONLY (the checker): imported by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg.

  oracle_mc(mc_in, nthreads)             mc_oracle.c:orc_mc_run on MEX-level inputs
  oracle_heat(T, Omega, heat_params)     heat_oracle.c:orc_heat_run (FP64 DG-ADI)
  oracle_mc_grad(mc_in, ...)             mc_oracle.c:orc_mc_grad (perturbation MC)
  oracle_heat_adjoint(T0, hp, ...)       heat_oracle.c:orc_heat_adjoint (FP64 adjoint of the stepper)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from mcmatlab_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_ref", "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError("oracle/_ref/liboracle.so is missing; run `make -C oracle oracle`")
        L = C.CDLL(path)
        L.orc_mc_run.argtypes = [C.POINTER(abi.mcb_mc_model), C.POINTER(abi.mcb_mc_result), C.c_int]
        L.orc_mc_run.restype = C.c_int
        dp = C.POINTER(C.c_double)
        L.orc_heat_run.argtypes = [C.c_long, C.c_long, C.c_long, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), dp, dp, C.c_int, C.c_int, C.c_long, C.c_double,
                                   dp, dp, C.c_int, dp, dp, dp, dp]
        L.orc_heat_run.restype = C.c_int
        L.orc_mc_grad.argtypes = [C.POINTER(abi.mcb_mc_model), C.POINTER(abi.mcb_mc_objectives),
                                  C.POINTER(abi.mcb_mc_result), C.POINTER(abi.mcb_mc_grad_result), C.c_int]
        L.orc_mc_grad.restype = C.c_int
        u8p = C.POINTER(C.c_uint8)
        L.orc_heat_adjoint.argtypes = [C.c_long, C.c_long, C.c_long, C.c_int, u8p, dp, dp, dp, dp, C.c_int, C.c_int,
                                       C.c_long, C.c_double, dp, dp, dp, dp, dp, dp, dp]
        L.orc_heat_adjoint.restype = C.c_int
        L.orc_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_lambert_wm1.argtypes = [C.c_double]
        L.orc_lambert_wm1.restype = C.c_double
        for f in ("orc_sizeof_mc_model", "orc_sizeof_mc_result", "orc_sizeof_heat_params"):
            getattr(L, f).restype = C.c_size_t
        _LIB = L
    return _LIB


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return list(o)


def oracle_downsample(paramVals, nBins):
    """CPU restatement of the sub-media binning: ([3 x n] float32, nBins) -> (downsampled [3 x nBins]
    float32, binidx [n] uint8, 1-based)."""
    par = np.asfortranarray(np.asarray(paramVals, dtype=np.float32))
    n = par.shape[1]
    out = np.zeros((3, int(nBins)), dtype=np.float32, order="F")
    idx = np.zeros(n, dtype=np.uint8)
    L = lib()
    rc = L.orc_downsample(par.ctypes.data_as(C.POINTER(C.c_float)), C.c_long(n), C.c_int(int(nBins)),
                          out.ctypes.data_as(C.POINTER(C.c_float)), idx.ctypes.data_as(C.POINTER(C.c_uint8)))
    if rc != 0:
        raise RuntimeError("oracle binning failed (%d)" % rc)
    return out, idx


def oracle_mc(mc_in, nthreads=0, example_cap=100000):
    """FP64 transport on MEX-level inputs; with nExamplePaths > 0 also the example paths (packets
    0, 1, 2, ... replayed one after another, as the CUDA path records them)."""
    mb = abi.McModelBuffers(mc_in)
    rb = abi.McResultBuffers(mc_in, example_cap if mc_in["nExamplePaths"] else 0)
    rc = lib().orc_mc_run(C.byref(mb.model), C.byref(rb.result), int(nthreads))
    if rc != 0:
        raise RuntimeError("oracle MC run failed (%d)" % rc)
    return rb.outputs()


def oracle_mc_grad(mc_in, nRadialBins=32, radialBinWidth=0.01, box=None, nthreads=0):
    """FP64 perturbation-MC run (same estimator as the GPU) -> (outputs, grad dict)."""
    mb = abi.McModelBuffers(mc_in)
    rb = abi.McResultBuffers(mc_in)
    gb = abi.GradBuffers(int(np.asarray(mc_in["mua"]).shape[0]), nRadialBins, radialBinWidth, box)
    rc = lib().orc_mc_grad(C.byref(mb.model), C.byref(gb.obj), C.byref(rb.result), C.byref(gb.res), int(nthreads))
    if rc != 0:
        raise RuntimeError("oracle gradient run failed (%d)" % rc)
    return rb.outputs(), gb.outputs()


def oracle_heat(T, Omega, hp, nx, ny, nz):
    """FP64 DG-ADI over hp['steps'] steps. Returns (T, Omega or None, sensorTemps [nS, nt+1], maxMediaTemps)."""
    hb = abi.HeatParamBuffers(nx, ny, nz, hp)
    p = hb.params
    Td = np.ascontiguousarray(np.asarray(T, dtype=np.float64).reshape(-1, order="F"))
    Od = None if Omega is None else np.ascontiguousarray(np.asarray(Omega, dtype=np.float64).reshape(-1, order="F"))
    nt = int(p.steps)
    sens = np.zeros(hb.nS * (nt + 1)) if hb.nS else None
    mx = np.zeros(hb.nM)
    dp = C.POINTER(C.c_double)
    nul = C.cast(None, dp)
    lib().orc_heat_run(nx, ny, nz, hb.nM, p.M, p.dTdtperdeltaT, p.dTdt_abs, p.A, p.E, p.lightsOn, p.heatBoundaryType,
                       nt, p.dt, Td.ctypes.data_as(dp), Od.ctypes.data_as(dp) if Od is not None else nul, hb.nS,
                       p.tempSensorCornerIdxs, p.tempSensorInterpWeights,
                       sens.ctypes.data_as(dp) if sens is not None else nul, mx.ctypes.data_as(dp))
    shp = (nx, ny, nz)
    return (Td.reshape(shp, order="F"), None if Od is None else Od.reshape(shp, order="F"),
            None if sens is None else sens.reshape(hb.nS, nt + 1, order="F"), mx)


def oracle_heat_adjoint(T0, hp, nx, ny, nz, wd=None, wp=None, c=None, Q=None, grads=True):
    """FP64 objective J = sum wd * (damage gained) + sum wp * max_n T^n of hp['steps'] DG-ADI steps and,
    with grads, (J, Jd, Jp), dJ/dc [nM, nM, 3], dJ/dQ and dJ/dT0 (grid shaped). c and Q default to
    hp's float32 tables and may be given in float64 (finite differences)."""
    c = np.asarray(hp["dTdtperdeltaT"] if c is None else c, dtype=np.float64)
    nM = c.shape[0]
    cd = np.ascontiguousarray(c.reshape(-1, order="F"))
    Qd = np.ascontiguousarray(np.asarray(hp["dTdt_abs"] if Q is None else Q, dtype=np.float64).reshape(-1, order="F"))
    M = np.ascontiguousarray(np.asarray(hp["M"], dtype=np.uint8).reshape(-1, order="F"))
    A = np.ascontiguousarray(np.asarray(hp["A"], dtype=np.float64).ravel())
    E = np.ascontiguousarray(np.asarray(hp["E"], dtype=np.float64).ravel())
    T = np.ascontiguousarray(np.asarray(T0, dtype=np.float64).reshape(-1, order="F"))
    L = T.size
    dp = C.POINTER(C.c_double)
    nul = C.cast(None, dp)

    def flat(w):
        return None if w is None else np.ascontiguousarray(np.asarray(w, dtype=np.float64).reshape(-1, order="F"))
    wdf, wpf = flat(wd), flat(wp)
    J = np.zeros(3)
    dc = np.zeros(nM * nM * 3) if grads else None
    dQ = np.zeros(L) if grads else None
    dT = np.zeros(L) if grads else None
    ptr = lambda a: a.ctypes.data_as(dp) if a is not None else nul
    lib().orc_heat_adjoint(nx, ny, nz, nM, M.ctypes.data_as(C.POINTER(C.c_uint8)), ptr(cd), ptr(Qd), ptr(A), ptr(E),
                           int(bool(hp["lightsOn"])), int(hp["heatBoundaryType"]), int(hp["steps"]), float(hp["dt"]),
                           ptr(T), ptr(wdf), ptr(wpf), ptr(J), ptr(dc), ptr(dQ), ptr(dT))
    if not grads:
        return J
    shp = (nx, ny, nz)
    return J, dc.reshape(nM, nM, 3, order="F"), dQ.reshape(shp, order="F"), dT.reshape(shp, order="F")
