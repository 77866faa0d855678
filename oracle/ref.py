"""Drives the reference's own MEX code, compiled from source into oracle/_ref.

TEST INFRASTRUCTURE ONLY (the checker): imported by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg, never by the product path.

`RefMC.run(tree, seed, nthreads)` calls mexFunction of +MCmatlab/src/MCmatlab.c:317
on a property tree built by mcmatlab_b200.mexargs.mex_model_tree. With
`seed` given, the clock the reference seeds dSFMT from (MCmatlab.c:241) is pinned to
`seed` microseconds and the OpenMP team is pinned to one thread, which makes the run
reproducible (stream = dsfmt_init_gen_rand(seed + 0)). With seed=None the reference
runs exactly as built, on `nthreads` (or all) cores: that is the timed CPU baseline.

`RefHeat.run(T, Omega, params)` calls mexFunction of
+MCmatlab/src/finiteElementHeatPropagator.c:688 and returns
(T, Omega, sensorTemps, maxMediaTemps).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_CLS = {  # numpy dtype -> mxClassID (oracle/mxshim/mex.h)
    np.dtype(np.float64): 6, np.dtype(np.float32): 7, np.dtype(np.uint8): 9,
    np.dtype(np.int32): 12, np.dtype(np.uint32): 13, np.dtype(np.int64): 14,
}
_LOGICAL = 3
_NP = {6: np.float64, 7: np.float32, 9: np.uint8, 3: np.uint8, 12: np.int32, 13: np.uint32, 14: np.int64}


def build(refsrc=None):
    """Builds oracle/_ref with the committed Makefile (needs the reference sources)."""
    args = ["make", "-C", HERE, "oracle"]
    if refsrc:
        args += ["ref", "REFSRC=%s" % refsrc]
    subprocess.run(args, check=True, capture_output=True)


class MxShim:
    def __init__(self):
        path = os.path.join(REF_DIR, "libmxshim.so")
        if not os.path.exists(path):
            raise FileNotFoundError("oracle/_ref/libmxshim.so is missing; run `make -C oracle`")
        self.lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
        L = self.lib
        P = C.c_void_p
        L.mxCreateNumericArray.restype = P
        L.mxCreateNumericArray.argtypes = [C.c_size_t, C.POINTER(C.c_size_t), C.c_int, C.c_int]
        L.mxshim_new_bag.restype = P
        L.mxshim_set.argtypes = [P, C.c_char_p, P]
        L.mxshim_get.restype = P
        L.mxshim_get.argtypes = [P, C.c_char_p]
        L.mxGetData.restype = P
        L.mxGetData.argtypes = [P]
        L.mxGetDimensions.restype = C.POINTER(C.c_size_t)
        L.mxGetDimensions.argtypes = [P]
        L.mxGetNumberOfDimensions.restype = C.c_size_t
        L.mxGetNumberOfDimensions.argtypes = [P]
        L.mxGetClassID.restype = C.c_int
        L.mxGetClassID.argtypes = [P]
        L.mxshim_is_bag.argtypes = [P]
        L.mxDestroyArray.argtypes = [P]
        L.mxshim_call.argtypes = [P, C.c_int, C.POINTER(P), C.c_int, C.POINTER(P)]
        L.mxshim_last_error.restype = C.c_char_p
        self.fixed_us = C.c_longlong.in_dll(L, "mxshim_fixed_us")
        self.nprocs = C.c_int.in_dll(L, "mxshim_nprocs")

    def array(self, a, logical=False):
        if isinstance(a, (bool, np.bool_)):
            a, logical = np.array([[1 if a else 0]], dtype=np.uint8), True
        elif isinstance(a, (int, float, np.integer, np.floating)) and not isinstance(a, np.ndarray):
            a = np.array([[float(a)]], dtype=np.float64)
        a = np.asarray(a)
        if a.dtype == np.bool_:
            a, logical = a.astype(np.uint8), True
        if a.ndim < 2:
            a = a.reshape(1, -1) if a.size else a.reshape(0, 0)
        cls = _LOGICAL if logical else _CLS[a.dtype]
        dims = (C.c_size_t * a.ndim)(*a.shape)
        p = self.lib.mxCreateNumericArray(a.ndim, dims, cls, 0)
        if a.size:
            buf = np.asfortranarray(a)
            C.memmove(self.lib.mxGetData(p), buf.ctypes.data, buf.nbytes)
        return p

    def tree(self, d):
        bag = self.lib.mxshim_new_bag()
        for k, v in d.items():
            self.lib.mxshim_set(bag, k.encode(), self.tree(v) if isinstance(v, dict) else self.array(v))
        return bag

    def to_numpy(self, p):
        if not p or self.lib.mxshim_is_bag(p):
            return None
        cls = self.lib.mxGetClassID(p)
        nd = self.lib.mxGetNumberOfDimensions(p)
        dp = self.lib.mxGetDimensions(p)
        dims = tuple(dp[i] for i in range(nd))
        n = int(np.prod(dims))
        dt = np.dtype(_NP[cls])
        out = np.empty(n, dtype=dt)
        if n:
            C.memmove(out.ctypes.data, self.lib.mxGetData(p), n * dt.itemsize)
        return out.reshape(dims, order="F")

    def get(self, p, *path):
        for name in path:
            p = self.lib.mxshim_get(p, name.encode())
            if not p:
                return None
        return p

    def call(self, fn, nlhs, prhs):
        plhs = (C.c_void_p * max(nlhs, 1))()
        arr = (C.c_void_p * len(prhs))(*prhs)
        rc = self.lib.mxshim_call(C.cast(fn, C.c_void_p), nlhs, plhs, len(prhs), arr)
        if rc:
            raise RuntimeError(self.lib.mxshim_last_error().decode())
        return [plhs[i] for i in range(nlhs)]


_SHIM = None


def shim():
    global _SHIM
    if _SHIM is None:
        _SHIM = MxShim()
    return _SHIM


class RefMC:
    """The reference MC MEX (MCmatlab.c) on the host cores. With libname="libmex_mc_cuda.so"
    the same harness drives this library's MEX gateway (mcmatlab_b200/mex/MCmatlab_CUDA.c)."""
    OUTPUTS = ("NFR", "farField", "NI_xpos", "NI_xneg", "NI_ypos", "NI_yneg", "NI_zpos", "NI_zneg",
               "nPhotons", "nPhotonsCollected", "nThreads", "simulationTime", "examplePaths")

    def __init__(self, libname="libref_mc.so"):
        self.sh = shim()
        self.lib = C.CDLL(os.path.join(REF_DIR, libname))
        self.fn = self.lib.mexFunction

    def run(self, tree, seed=None, nthreads=None, simType=None):
        """Runs the MEX on a property tree (mexargs.mex_model_tree). simType 2 (fluorescence) makes
        the MEX read and write the tree's FMC node (MCmatlab.c:322-323, :463); by default it
        follows the tree (FMC when that node is filled)."""
        sh = self.sh
        if simType is None:
            simType = 2 if tree.get("FMC") else 1
        key = "FMC" if simType == 2 else "MC"
        t = dict(tree)
        t[key] = dict(tree[key])
        # outputs the MEX overwrites are created up front, as MATLAB's object would hold them
        for k in self.OUTPUTS:
            t[key].setdefault(k, np.nan)
        t[key]["LC"] = dict(tree[key]["LC"])
        t[key]["LC"].setdefault("image", np.nan)
        if seed is not None:
            t[key]["useAllCPUs"] = True
            sh.fixed_us.value = int(seed)
            sh.nprocs.value = 1
        else:
            sh.fixed_us.value = -1
            sh.nprocs.value = int(nthreads) if nthreads else 0
            if nthreads:
                t[key]["useAllCPUs"] = True
        root = sh.tree(t)
        simtype = sh.array(float(simType))
        try:
            (out,) = sh.call(self.fn, 1, [root, simtype])
        finally:
            sh.fixed_us.value = -1
            sh.nprocs.value = 0
        MC = sh.get(out, key)
        res = {}
        for k in self.OUTPUTS:
            res[k] = sh.to_numpy(sh.get(MC, k))
        res["image"] = sh.to_numpy(sh.get(MC, "LC", "image"))
        sh.lib.mxDestroyArray(out)
        sh.lib.mxDestroyArray(root)
        sh.lib.mxDestroyArray(simtype)
        return res


class RefDownsample:
    """The reference's sub-media binning MEX (getDownsampledParamVals.c) on the host:
    (paramVals [3 x n] single, nBins) -> (downsampled [3 x nBins] single, binidx [1 x n] uint8).
    With libname="libmex_ds_cuda.so" the same harness drives this library's gateway
    (mcmatlab_b200/mex/getDownsampledParamVals_CUDA.c)."""

    def __init__(self, libname="libref_downsample.so"):
        self.sh = shim()
        self.lib = C.CDLL(os.path.join(REF_DIR, libname))
        self.fn = self.lib.mexFunction

    def run(self, paramVals, nBins):
        sh = self.sh
        a = sh.array(np.asfortranarray(np.asarray(paramVals, dtype=np.float32)))
        b = sh.array(float(nBins))
        try:
            d, idx = sh.call(self.fn, 2, [a, b])
            out = sh.to_numpy(d), sh.to_numpy(idx).reshape(-1)
        finally:
            sh.lib.mxDestroyArray(a)
            sh.lib.mxDestroyArray(b)
        sh.lib.mxDestroyArray(d)
        sh.lib.mxDestroyArray(idx)
        return out


class RefHeat:
    """The reference heat MEX (finiteElementHeatPropagator.c) on the host cores. With
    libname="libmex_heat_cuda.so" it drives this library's heat MEX gateway instead."""

    def __init__(self, libname="libref_heat.so"):
        self.sh = shim()
        self.lib = C.CDLL(os.path.join(REF_DIR, libname))
        self.fn = self.lib.mexFunction

    def run(self, T, Omega, params, nthreads=None):
        sh = self.sh
        p = dict(params)
        if nthreads:
            p["useAllCPUs"] = True
            sh.nprocs.value = int(nthreads)
        Tm = sh.array(np.asfortranarray(np.asarray(T, dtype=np.float32)))
        Om = sh.array(np.asarray(Omega, dtype=np.float32) if np.ndim(Omega) else np.array([[Omega]], dtype=np.float32))
        Pm = sh.tree(p)
        try:
            outs = sh.call(self.fn, 4, [Tm, Om, Pm])
        finally:
            sh.nprocs.value = 0
        res = tuple(sh.to_numpy(o) for o in outs)
        for o in outs:
            sh.lib.mxDestroyArray(o)
        for o in (Tm, Om, Pm):
            sh.lib.mxDestroyArray(o)
        return res
