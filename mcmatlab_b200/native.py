"""ctypes binding to the in-tree sm_100a library libmcb200.so (include/mcb200.h).

There is no CPU fallback: if the library or a CUDA device is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import threading

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmcb200.so")

_lock = threading.RLock()
_lib = None
_ctx = {}

STATUS = {0: "MCB_OK", 1: "MCB_EINVAL", 2: "MCB_ENOMEM", 3: "MCB_ECUDA", 4: "MCB_ECANCELLED", 5: "MCB_ETIMEOUT",
          6: "MCB_ELAUNCH"}

EXPORTS = ("mcb_ctx_create", "mcb_ctx_destroy", "mcb_last_error", "mcb_cancel_flag", "mcb_mc_run", "mcb_mc_run_batch",
           "mcb_mc_grad", "mcb_heat_forward_static", "mcb_heat_adjoint", "mcb_probe_atomics",
           "mcb_interface_normals", "mcb_downsample_params",
           "mcb_heat_forward", "mcb_heat_state_create", "mcb_heat_state_step", "mcb_heat_state_read",
           "mcb_heat_state_destroy", "mcb_last_kernel_ms", "mcb_mc_tally_count", "mcb_mc_normalize",
           "mcb_mc_size_class", "mcb_mc_autotune")


class MCBError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


def lib():
    """Loads libmcb200.so (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FileNotFoundError("%s is missing: build it with `python -m mcmatlab_b200.build`" % LIB_PATH)
            L = C.CDLL(LIB_PATH)
            L.mcb_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
            L.mcb_ctx_destroy.argtypes = [C.c_void_p]
            L.mcb_last_error.argtypes = [C.c_void_p]
            L.mcb_last_error.restype = C.c_char_p
            L.mcb_cancel_flag.argtypes = [C.c_void_p]
            L.mcb_cancel_flag.restype = C.POINTER(C.c_int)
            L.mcb_mc_run.argtypes = [C.c_void_p, C.POINTER(abi.mcb_mc_model), C.POINTER(abi.mcb_mc_result)]
            L.mcb_mc_run_batch.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.POINTER(abi.mcb_mc_model)),
                                           C.POINTER(C.POINTER(abi.mcb_mc_result))]
            L.mcb_mc_grad.argtypes = [C.c_void_p, C.POINTER(abi.mcb_mc_model), C.POINTER(abi.mcb_mc_objectives),
                                      C.POINTER(abi.mcb_mc_result), C.POINTER(abi.mcb_mc_grad_result)]
            L.mcb_heat_forward.argtypes = [C.c_void_p, C.POINTER(abi.mcb_heat_params), C.POINTER(C.c_float),
                                           C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_float)]
            L.mcb_heat_forward_static.argtypes = [C.c_void_p, C.POINTER(abi.mcb_heat_params), C.POINTER(C.c_float),
                                                  C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_float)]
            L.mcb_heat_adjoint.argtypes = [C.c_void_p, C.POINTER(abi.mcb_heat_params), C.POINTER(C.c_float),
                                           C.POINTER(abi.mcb_heat_objective), C.c_int32, C.POINTER(abi.mcb_heat_grad)]
            L.mcb_heat_state_create.argtypes = [C.c_void_p, C.POINTER(abi.mcb_heat_params), C.POINTER(C.c_float),
                                                C.POINTER(C.c_float), C.POINTER(C.c_void_p)]
            L.mcb_heat_state_step.argtypes = [C.c_void_p, C.POINTER(abi.mcb_heat_params), C.POINTER(C.c_double),
                                              C.POINTER(C.c_float)]
            L.mcb_heat_state_read.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float)]
            L.mcb_heat_state_destroy.argtypes = [C.c_void_p]
            L.mcb_probe_atomics.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_double)]
            L.mcb_interface_normals.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_uint8),
                                                C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_double, C.c_double,
                                                C.c_double, C.c_double, C.POINTER(C.c_float)]
            L.mcb_downsample_params.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_int64, C.c_int32,
                                                C.POINTER(C.c_float), C.POINTER(C.c_uint8)]
            L.mcb_mc_tally_count.argtypes = [C.POINTER(abi.mcb_mc_model)]
            L.mcb_mc_tally_count.restype = C.c_int64
            L.mcb_mc_normalize.argtypes = [C.c_void_p, C.POINTER(abi.mcb_mc_model), C.POINTER(C.c_double),
                                           C.POINTER(abi.mcb_mc_result)]
            L.mcb_mc_size_class.argtypes = [C.POINTER(abi.mcb_mc_model), C.c_int32, C.c_int32]
            L.mcb_mc_size_class.restype = C.c_int32
            L.mcb_mc_autotune.argtypes = [C.c_void_p, C.POINTER(abi.mcb_mc_model), C.c_double, C.c_int32,
                                          C.POINTER(abi.mcb_mc_launch), C.POINTER(C.c_double)]
            L.mcb_last_kernel_ms.argtypes = [C.c_void_p]
            L.mcb_last_kernel_ms.restype = C.c_double
            _lib = L
        return _lib


def context(device=0):
    L = lib()
    with _lock:
        if device not in _ctx:
            p = C.c_void_p()
            st = L.mcb_ctx_create(int(device), C.byref(p))
            if st != 0:
                raise MCBError(st, "could not create a context on CUDA device %d" % device)
            _ctx[device] = p
        return _ctx[device]


def release(device=0):
    """Destroys the device's context, which frees its work buffers (a later call creates a new one).
    Close every HeatState of the device first: a state keeps a pointer to its context."""
    with _lock:
        p = _ctx.pop(device, None)
    if p is not None:
        lib().mcb_ctx_destroy(p)


def _check(st, ctx):
    if st != 0:
        raise MCBError(st, lib().mcb_last_error(ctx).decode())


def mc_run(mc_in, device=0, example_cap=100000, tallies=False):
    """Runs one model (MEX-level inputs from mexargs.prepare_mc); returns outputs in MATLAB shapes.
    With tallies=True the output also holds "tallies": the run's FP64 tallies before
    normalisation (mcb_mc_result.tallies), which add up over runs on disjoint packet ranges."""
    ctx = context(device)
    mb = abi.McModelBuffers(mc_in)
    nt = int(lib().mcb_mc_tally_count(C.byref(mb.model))) if tallies else 0
    rb = abi.McResultBuffers(mc_in, example_cap if mc_in["nExamplePaths"] else 0, nt)
    _check(lib().mcb_mc_run(ctx, C.byref(mb.model), C.byref(rb.result)), ctx)
    return rb.outputs()


def mc_autotune(mc_in, calibration_packets=2e5, gradient=False, device=0):
    """Tunes the transport kernel's warp-grouping parameters for mc_in's size class on this GPU
    (mcb_mc_autotune); later runs of the class in this process use the choice. Returns
    dict(refillMin, scatterMin, sizeClass, table [16 x 3]: refillMin, scatterMin, kernel ms)."""
    ctx = context(device)
    mb = abi.McModelBuffers(mc_in)
    ch = abi.mcb_mc_launch()
    table = np.zeros(48)
    _check(lib().mcb_mc_autotune(ctx, C.byref(mb.model), float(calibration_packets), int(bool(gradient)), C.byref(ch),
                                 table.ctypes.data_as(C.POINTER(C.c_double))), ctx)
    return {"refillMin": ch.refillMin, "scatterMin": ch.scatterMin,
            "sizeClass": int(lib().mcb_mc_size_class(C.byref(mb.model), int(bool(gradient)), 0)),
            "table": table.reshape(16, 3)}


def mc_normalize(mc_in, tallies, device=0):
    """Normalised outputs (MATLAB shapes, nPhotons, nPhotonsCollected) of given FP64 tallies of
    model mc_in, e.g. the sum of the "tallies" of runs on disjoint packet ranges: the outputs of
    one run over the union of their packets (mcb_mc_normalize)."""
    ctx = context(device)
    mb = abi.McModelBuffers(mc_in)
    t = np.ascontiguousarray(np.asarray(tallies, dtype=np.float64))
    if t.size != int(lib().mcb_mc_tally_count(C.byref(mb.model))):
        raise ValueError("tallies have %d entries, the model needs %d" % (t.size, lib().mcb_mc_tally_count(C.byref(mb.model))))
    rb = abi.McResultBuffers(mc_in)
    _check(lib().mcb_mc_normalize(ctx, C.byref(mb.model), t.ctypes.data_as(C.POINTER(C.c_double)), C.byref(rb.result)), ctx)
    return rb.outputs()


def mc_grad(mc_in, nRadialBins=32, radialBinWidth=0.01, box=None, device=0):
    """Perturbation-MC run: forward outputs plus R (radial reflectance), F (box mean fluence rate)
    and their derivatives with respect to every medium's mua and mus."""
    ctx = context(device)
    mb = abi.McModelBuffers(mc_in)
    rb = abi.McResultBuffers(mc_in)
    gb = abi.GradBuffers(int(np.asarray(mc_in["mua"]).shape[0]), nRadialBins, radialBinWidth, box)
    _check(lib().mcb_mc_grad(ctx, C.byref(mb.model), C.byref(gb.obj), C.byref(rb.result), C.byref(gb.res)), ctx)
    return rb.outputs(), gb.outputs()


def mc_run_batch(mc_ins, device=0):
    """Runs several models in one persistent launch; returns a list of output dicts."""
    ctx = context(device)
    mbs = [abi.McModelBuffers(x) for x in mc_ins]
    rbs = [abi.McResultBuffers(x) for x in mc_ins]
    n = len(mc_ins)
    mp = (C.POINTER(abi.mcb_mc_model) * n)(*[C.pointer(m.model) for m in mbs])
    rp = (C.POINTER(abi.mcb_mc_result) * n)(*[C.pointer(r.result) for r in rbs])
    _check(lib().mcb_mc_run_batch(ctx, n, mp, rp), ctx)
    return [r.outputs() for r in rbs]


def heat_forward(T, Omega, hp, nx, ny, nz, device=0):
    """finiteElementHeatPropagator equivalent. Omega None = no damage.
    Returns (T, Omega or None, sensorTemps [nS, nt+1] or empty, maxMediaTemps [1, nM])."""
    ctx = context(device)
    hb = abi.HeatParamBuffers(nx, ny, nz, hp)
    Tb = np.ascontiguousarray(np.asarray(T, dtype=np.float32).reshape(-1, order="F")).copy()
    Ob = None if Omega is None else np.ascontiguousarray(np.asarray(Omega, dtype=np.float32).reshape(-1, order="F")).copy()
    nt = int(hb.params.steps)
    sens = np.zeros(hb.nS * (nt + 1)) if hb.nS else np.zeros(1)
    mx = np.zeros(hb.nM, dtype=np.float32)
    fp = C.POINTER(C.c_float)
    _check(lib().mcb_heat_forward(ctx, C.byref(hb.params), Tb.ctypes.data_as(fp),
                                  Ob.ctypes.data_as(fp) if Ob is not None else C.cast(None, fp),
                                  sens.ctypes.data_as(C.POINTER(C.c_double)), mx.ctypes.data_as(fp)), ctx)
    shp = (nx, ny, nz)
    return (Tb.reshape(shp, order="F"), None if Ob is None else Ob.reshape(shp, order="F"),
            sens.reshape(hb.nS, nt + 1, order="F") if hb.nS else np.zeros((0, 0)), mx.reshape(1, -1))


def heat_forward_static(T, Omega, hp, nx, ny, nz, device=0):
    """heat_forward through mcb_heat_forward_static (no allocation; 32 MiB static scratch)."""
    ctx = context(device)
    hb = abi.HeatParamBuffers(nx, ny, nz, hp)
    Tb = np.ascontiguousarray(np.asarray(T, dtype=np.float32).reshape(-1, order="F")).copy()
    Ob = None if Omega is None else np.ascontiguousarray(np.asarray(Omega, dtype=np.float32).reshape(-1, order="F")).copy()
    nt = int(hb.params.steps)
    sens = np.zeros(hb.nS * (nt + 1)) if hb.nS else np.zeros(1)
    mx = np.zeros(hb.nM, dtype=np.float32)
    fp = C.POINTER(C.c_float)
    _check(lib().mcb_heat_forward_static(ctx, C.byref(hb.params), Tb.ctypes.data_as(fp),
                                         Ob.ctypes.data_as(fp) if Ob is not None else C.cast(None, fp),
                                         sens.ctypes.data_as(C.POINTER(C.c_double)), mx.ctypes.data_as(fp)), ctx)
    shp = (nx, ny, nz)
    return (Tb.reshape(shp, order="F"), None if Ob is None else Ob.reshape(shp, order="F"),
            sens.reshape(hb.nS, nt + 1, order="F") if hb.nS else np.zeros((0, 0)), mx.reshape(1, -1))


def heat_adjoint(T0, hp, nx, ny, nz, damageWeight=None, peakWeight=None, nCheckpoints=0, device=0):
    """Objective J = sum damageWeight * damage gained + sum peakWeight * max_n T^n over hp['steps'] steps
    from T0, and its gradients (mcb_heat_adjoint). Returns a dict with J, J_damage, J_peak,
    dJ_dc [nM, nM, 3], dJ_dQ and dJ_dT0 (grid shaped), forwardMs, adjointMs."""
    ctx = context(device)
    hb = abi.HeatParamBuffers(nx, ny, nz, hp)
    fp = C.POINTER(C.c_float)
    col = lambda a: None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1, order="F"))
    Tb, wd, wp = col(T0), col(damageWeight), col(peakWeight)
    obj = abi.mcb_heat_objective()
    obj.damageWeight = wd.ctypes.data_as(fp) if wd is not None else C.cast(None, fp)
    obj.peakWeight = wp.ctypes.data_as(fp) if wp is not None else C.cast(None, fp)
    nM = hb.nM
    L = nx * ny * nz
    dc = np.zeros(nM * nM * 3)
    dQ = np.zeros(L, dtype=np.float32)
    dT = np.zeros(L, dtype=np.float32)
    g = abi.mcb_heat_grad()
    g.dJ_dc = dc.ctypes.data_as(C.POINTER(C.c_double))
    g.dJ_dQ = dQ.ctypes.data_as(fp)
    g.dJ_dT0 = dT.ctypes.data_as(fp)
    _check(lib().mcb_heat_adjoint(ctx, C.byref(hb.params), Tb.ctypes.data_as(fp), C.byref(obj), int(nCheckpoints),
                                  C.byref(g)), ctx)
    shp = (nx, ny, nz)
    return dict(J=g.J, J_damage=g.J_damage, J_peak=g.J_peak, dJ_dc=dc.reshape(nM, nM, 3, order="F"),
                dJ_dQ=dQ.reshape(shp, order="F"), dJ_dT0=dT.reshape(shp, order="F"),
                forwardMs=g.forwardMs, adjointMs=g.adjointMs)


def interface_normals(M1, n_per_submedium, dx, dy, dz, smoothingLengthScale=0.0, device=0):
    """prep.interface_normals on the device (mcb_interface_normals): (theta, phi) float32 [2, L]."""
    ctx = context(device)
    M = np.ascontiguousarray(np.asarray(M1, dtype=np.uint8).reshape(-1, order="F"))
    nrows = np.asarray(n_per_submedium, dtype=np.float64)
    if nrows.ndim == 1:
        nrows = nrows[:, None]
    uniq, inv = np.unique(nrows, axis=0, return_inverse=True)
    cls = np.ascontiguousarray(np.asarray(inv, dtype=np.int32).reshape(-1))
    nx, ny, nz = np.shape(M1)
    out = np.empty(2 * M.size, dtype=np.float32)
    _check(lib().mcb_interface_normals(ctx, nx, ny, nz, M.ctypes.data_as(C.POINTER(C.c_uint8)), cls.size,
                                       cls.ctypes.data_as(C.POINTER(C.c_int32)), int(uniq.shape[0]), float(dx),
                                       float(dy), float(dz), float(smoothingLengthScale),
                                       out.ctypes.data_as(C.POINTER(C.c_float))), ctx)
    return out.reshape(2, M.size, order="F")


def downsample_params(paramVals, nBins, device=0):
    """Sub-media binning on the device (mcb_downsample_params; MATLAB's getDownsampledParamVals):
    paramVals [3, n] float32 (mua, mus, g per voxel) -> (downsampled [3, nBins] float32,
    binidx [n] uint8, 1-based)."""
    ctx = context(device)
    par = np.asfortranarray(np.asarray(paramVals, dtype=np.float32))
    if par.ndim != 2 or par.shape[0] != 3:
        raise ValueError("paramVals must be [3, n]")
    n = par.shape[1]
    out = np.zeros((3, int(nBins)), dtype=np.float32, order="F")
    idx = np.zeros(n, dtype=np.uint8)
    _check(lib().mcb_downsample_params(ctx, par.ctypes.data_as(C.POINTER(C.c_float)), n, int(nBins),
                                       out.ctypes.data_as(C.POINTER(C.c_float)), idx.ctypes.data_as(C.POINTER(C.c_uint8))),
           ctx)
    return out, idx


def probe_atomics(slots=1 << 20, device=0):
    """FP64 atomicAdd operations per second to scattered slots of a `slots`-double buffer."""
    ctx = context(device)
    r = C.c_double()
    _check(lib().mcb_probe_atomics(ctx, int(slots), C.byref(r)), ctx)
    return r.value


def last_kernel_ms(device=0):
    """Device time (CUDA events on the library's stream) of the last transport/stepping loop."""
    return lib().mcb_last_kernel_ms(context(device))


class HeatState:
    """Device-resident heat stepper state (mcb_heat_state_*): grids stay in HBM between step() calls."""

    def __init__(self, T, Omega, hp, nx, ny, nz, device=0):
        self.ctx = context(device)
        self.shape = (nx, ny, nz)
        self.hb = abi.HeatParamBuffers(nx, ny, nz, hp)
        self.damage = Omega is not None
        Tb = np.ascontiguousarray(np.asarray(T, dtype=np.float32).reshape(-1, order="F"))
        Ob = None if Omega is None else np.ascontiguousarray(np.asarray(Omega, dtype=np.float32).reshape(-1, order="F"))
        fp = C.POINTER(C.c_float)
        p = C.c_void_p()
        _check(lib().mcb_heat_state_create(self.ctx, C.byref(self.hb.params), Tb.ctypes.data_as(fp),
                                           Ob.ctypes.data_as(fp) if Ob is not None else C.cast(None, fp), C.byref(p)),
               self.ctx)
        self.ptr = p

    def step(self, hp):
        hb = abi.HeatParamBuffers(*self.shape, hp)
        nt = int(hb.params.steps)
        sens = np.zeros(max(hb.nS * (nt + 1), 1))
        mx = np.zeros(hb.nM, dtype=np.float32)
        _check(lib().mcb_heat_state_step(self.ptr, C.byref(hb.params), sens.ctypes.data_as(C.POINTER(C.c_double)),
                                         mx.ctypes.data_as(C.POINTER(C.c_float))), self.ctx)
        return (sens[:hb.nS * (nt + 1)].reshape(hb.nS, nt + 1, order="F") if hb.nS else np.zeros((0, 0))), mx.reshape(1, -1)

    def read(self):
        n = int(np.prod(self.shape))
        T = np.zeros(n, dtype=np.float32)
        O = np.zeros(n, dtype=np.float32) if self.damage else None
        fp = C.POINTER(C.c_float)
        _check(lib().mcb_heat_state_read(self.ptr, T.ctypes.data_as(fp), O.ctypes.data_as(fp) if O is not None else
                                         C.cast(None, fp)), self.ctx)
        return T.reshape(self.shape, order="F"), (None if O is None else O.reshape(self.shape, order="F"))

    def close(self):
        if self.ptr:
            lib().mcb_heat_state_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
