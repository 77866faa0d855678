"""Host-side input preparation for the two hot paths.

The reference prepares the MEX inputs in MATLAB. MATLAB is not part of this
library's runtime, so the preparation steps that feed the kernels are restated
here in numpy, each citing the MATLAB function it follows:

* geometry evaluation           +MCmatlab/@geometry/geometry.m:44-66, :130-138
* optical media properties      +MCmatlab/@model/private/getOpticalMediaProperties.m:1-258
* Sobel interface normals       +MCmatlab/@model/private/imgradientxyz.m:38-59 and
                                getOpticalMediaProperties.m:222-244, with the smoothn
                                smoothing of the gradients (:230-231; smooth_gradients)
* thermal media properties      +MCmatlab/@model/private/getThermalMediaProperties.m
* dT/dt arrays, dt limit        +MCmatlab/@model/simulateHeatDistribution.m:469-514
* temperature sensor weights    +MCmatlab/@model/simulateHeatDistribution.m:543-609

All arrays use MATLAB's column-major voxel order (x fastest): a grid array is a
numpy array of shape (nx, ny, nz) in Fortran order, flattened with order="F".
"""
from __future__ import annotations

import inspect
import math

import numpy as np

CDFSIZE = 201  # +MCmatlab/src/MCmatlab.c:171 (one more than the 200 theta bins below)


def _nargs(f):
    """Number of required positional parameters (MATLAB's nargin of a function handle)."""
    try:
        return sum(1 for p in inspect.signature(f).parameters.values()
                   if p.default is inspect.Parameter.empty and p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD))
    except (TypeError, ValueError):
        return 1


def eval_optical(f, wavelength):
    """Evaluates a medium property given as a number, f(wavelength) or f(wavelength, FR, T, FD).

    The reference wraps numbers and one-argument functions into four-argument
    functions (+MCmatlab/@mediumProperties/mediumProperties.m:30-52) and evaluates
    them at (wavelength, 0, 0, 0) for media without FR/T/FD dependence
    (getOpticalMediaProperties.m:72-92).
    """
    if callable(f):
        n = _nargs(f)
        return f(wavelength) if n == 1 else f(wavelength, 0.0, 0.0, 0.0)
    return f


def elementwise(f, *args):
    """f applied to array arguments: called once on the arrays, as the reference requires of
    FR/T/FD-dependent property functions (element-wise arithmetic, getOpticalMediaProperties.m:
    67-83); a function written for scalars is applied element by element instead."""
    try:
        return f(*args)
    except (TypeError, ValueError):
        return np.vectorize(f, otypes=[np.float64])(*args)


def eval_thermal(f, T=37.0, FD=0.0):
    """Thermal property given as a number or f(T, FD) (mediumProperties.m:180-207)."""
    if callable(f):
        return f(T, FD)
    return f


def geometry_axes(nx, ny, nz, Lx, Ly, Lz):
    """Voxel-centre coordinates; x and y are centred on 0, z starts at 0 (geometry.m:121-138)."""
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    y = (np.arange(ny) - (ny - 1) / 2) * dy
    z = (np.arange(nz) + 0.5) * dz
    return x, y, z


def evaluate_geometry(G):
    """Runs geomFunc on single-precision ndgrid coordinates (geometry.m:44-66)."""
    x, y, z = geometry_axes(G.nx, G.ny, G.nz, G.Lx, G.Ly, G.Lz)
    X, Y, Z = np.meshgrid(x.astype(np.float32), y.astype(np.float32), z.astype(np.float32), indexing="ij")
    M = np.asarray(G.geomFunc(X, Y, Z, G.geomFuncParams))
    if M.shape != (G.nx, G.ny, G.nz):
        raise ValueError("Error: The M returned by the geometry function must be nx by ny by nz in size.")
    if np.any(M <= 0):
        raise ValueError("Error: The M returned by the geometry function must only contain positive numbers.")
    if np.any(np.mod(M, 1)):
        raise ValueError("Error: The M returned by the geometry function must only contain integers.")
    if np.any(M > 255):
        raise ValueError("Error: The M returned by the geometry function must not contain numbers over 255.")
    return np.asfortranarray(M.astype(np.uint8))


def _replicate_pad(I):
    return np.pad(I, 1, mode="edge")


def sobel_gradients(I):
    """3D Sobel gradient with replicated borders (imgradientxyz.m 'sobel', correlation).

    Returns (Gx, Gy, Gz) as derivatives along the first (x), second (y) and third (z)
    array dimension. imgradientxyz names its outputs the other way round for the
    first two (its 'Gx' differentiates along columns), which getOpticalMediaProperties.m:229
    undoes by unpacking them as [Gy_Sobel, Gx_Sobel, Gz_Sobel].

    The kernels are central differences [-1 0 1] along the derivative axis times the
    transverse weights [[1 3 1],[3 6 3],[1 3 1]] = [1 3 1] x [1 3 1] - 3 delta, evaluated
    with separable 1-D correlations.
    """
    from scipy.ndimage import correlate1d
    I = np.asarray(I, dtype=np.float64)
    s = np.array([1.0, 3.0, 1.0])
    d = np.array([-1.0, 0.0, 1.0])
    out = []
    for ax in range(3):
        o1, o2 = [a for a in range(3) if a != ax]
        D = correlate1d(I, d, axis=ax, mode="nearest")
        T = correlate1d(correlate1d(D, s, axis=o1, mode="nearest"), s, axis=o2, mode="nearest")
        out.append(T - 3.0 * D)
    return out[0], out[1], out[2]


def smooth_gradients(fields, s, spacing):
    """The smoothing MCmatlab applies to the Sobel gradients (smoothn.m with a given smoothness s,
    no weights, no robust iterations): penalised least squares with a second-difference
    penalty, solved in the DCT-II basis (Garcia, Comput. Stat. Data Anal. 54, 2010):
        z = IDCT(Gamma * DCT(y)),  Gamma = 1 / (1 + s * Lambda^2),
        Lambda = sum_i (2 - 2 cos(pi k_i / n_i)) / h_i^2,  h = spacing / max(spacing).
    Every field is smoothed with the same s."""
    from scipy.fft import dctn, idctn
    shape = np.shape(fields[0])
    h = np.asarray(spacing, dtype=np.float64)
    h = h / h.max()
    lam = np.zeros(shape)
    for ax, n in enumerate(shape):
        k = np.arange(n).reshape([n if a == ax else 1 for a in range(len(shape))])
        lam = lam + (2.0 - 2.0 * np.cos(np.pi * k / n)) / h[ax] ** 2
    gamma = 1.0 / (1.0 + s * lam ** 2)
    return [idctn(gamma * dctn(np.asarray(f, dtype=np.float64), type=2, norm="ortho"), type=2, norm="ortho")
            for f in fields]


def interface_normals(M1, n_per_submedium, dx, dy, dz, smoothingLengthScale=0.0):
    """(theta, phi) of the interface normal per voxel, float32 [2, L] (getOpticalMediaProperties.m:222-240).

    M1 is the 1-based sub-medium grid; n_per_submedium is the [nSM, nL] refractive
    index table. Voxels are grouped by unique refractive-index rows; for each group the
    Sobel gradient of the group's indicator gives the normal inside that group, smoothed
    with s = max(1, round(smoothingLengthScale / max(dx, dy, dz))) when the length scale is
    positive (:230-231).
    """
    nrows = np.asarray(n_per_submedium, dtype=np.float64)
    if nrows.ndim == 1:
        nrows = nrows[:, None]
    uniq, inv = np.unique(nrows, axis=0, return_inverse=True)
    inv = np.asarray(inv).reshape(-1)
    ri_class = inv[M1.astype(np.int64) - 1]
    Gx = np.full(M1.shape, np.nan)
    Gy = np.full(M1.shape, np.nan)
    Gz = np.full(M1.shape, np.nan)
    for k in range(uniq.shape[0]):
        mask = ri_class == k
        gx, gy, gz = sobel_gradients(mask)
        gx, gy, gz = gx / dx, gy / dy, gz / dz
        if smoothingLengthScale > 0:
            s = max(1, int(np.round(smoothingLengthScale / max(dx, dy, dz))))
            gx, gy, gz = smooth_gradients([gx, gy, gz], s, [dx, dy, dz])
        Gx[mask] = gx[mask]
        Gy[mask] = gy[mask]
        Gz[mask] = gz[mask]
    # cart2sph: phi = atan2(y, x), elevation = atan2(z, hypot(x, y)); theta = pi/2 - elevation
    phi = np.arctan2(Gy, Gx)
    elev = np.arctan2(Gz, np.hypot(Gx, Gy))
    theta = np.pi / 2 - elev
    out = np.empty((2, M1.size), dtype=np.float32, order="F")  # MATLAB order: (theta, phi) per voxel
    out[0] = theta.reshape(-1, order="F")
    out[1] = phi.reshape(-1, order="F")
    return out


def custom_phase_cdf(phase_func, wavelength):
    """201-entry CDF of a custom phase function over 200 theta bins (getOpticalMediaProperties.m:94-102)."""
    n_thetas = CDFSIZE - 1
    thetas = np.pi / n_thetas * (np.arange(1, n_thetas + 1) - 0.5)
    pdf = np.array([math.sin(t) * float(phase_func(wavelength, t)) for t in thetas])
    if not np.all(np.isfinite(pdf)) or np.any(pdf < 0):
        raise ValueError("Error: The custom phase function did not return real, finite, non-negative numbers.")
    return np.concatenate([[0.0], np.cumsum(pdf) / np.sum(pdf)])


_TEST_WAVELENGTHS = np.linspace(100e-9, 10000e-9, 10)  # geometry.m:71 (as written there)


def _test_grid():
    FRs = np.concatenate([[0.0], np.logspace(-20, 20, 9)])
    Ts = np.linspace(-100, 300, 10)
    FDs = np.linspace(0, 1, 10)
    return np.meshgrid(FRs, Ts, FDs, indexing="ij")


def _varies(vals, axis):
    """any(~isequaln(max(v,[],axis), min(v,[],axis))) with MATLAB's NaN-ignoring max/min."""
    with np.errstate(all="ignore"):
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            hi = np.nanmax(vals, axis=axis)
            lo = np.nanmin(vals, axis=axis)
    return not np.array_equal(hi, lo, equal_nan=True)


def dependence_flags(media):
    """FRdependent, optTdependent, optFDdependent [nM, 5] (mua, mus, g, QY, ES) of the given media
    (geometry.m:64-101): each property is sampled over wavelengths x (FR, T, FD) test grids and
    flagged when it changes along the FR, T or FD axis."""
    FR, T, FD = _test_grid()
    nM = len(media)
    flags = np.zeros((3, nM, 5), dtype=bool)
    for iM, med in enumerate(media):
        for iL, L in enumerate(_TEST_WAVELENGTHS):
            for col, f in enumerate((med.mua, med.mus, med.g, med.QY, med.ES)):
                if not callable(f) or _nargs(f) == 1:
                    continue  # constant in FR, T and FD
                vals = np.broadcast_to(np.asarray(elementwise(f, L, FR, T, FD), dtype=np.float64), FR.shape)
                for ax in range(3):
                    flags[ax, iM, col] |= _varies(vals, ax)
    return flags[0], flags[1], flags[2]


def _eval_dep(f, wavelength, dependent, FRs, Ts, FDs):
    """A medium property at one wavelength: over the medium's voxels when it depends on FR, T or
    FD, else at (wavelength, 0, 0, 0) (getOpticalMediaProperties.m:64-84). The wavelength is a
    Python float, so single-precision voxel arrays stay single as in MATLAB's mixed arithmetic."""
    if not callable(f):
        return f
    if _nargs(f) == 1:
        return f(wavelength)
    return elementwise(f, wavelength, FRs, Ts, FDs) if dependent else f(wavelength, 0.0, 0.0, 0.0)


def optical_media_properties(mediaList, M_raw, wavelengths, matchedInterfaces, dx, dy, dz, DC, smoothingLengthScale=0.0,
                             normals=None, FR=0.0, T=0.0, FD=0.0, downsample=None):
    """Per-sub-medium optical tables and the sub-medium grid (getOpticalMediaProperties.m:1-244).

    Media whose mua, mus or g depend on fluence rate, temperature or damage are evaluated per
    voxel and split into nBins sub-media by the sub-media binning (getDownsampledParamVals; the
    `downsample` callable, native.downsample_params on the device) on the first wavelength; later
    wavelengths take the mean per bin (:147-197). FR, T and FD are grids (or scalars) of the
    model's fluence rate, temperature and fractional damage.
    Returns a dict with mua, mus, g, n, CDFidx ([nSM, nL] float64), M (uint8, 1-based),
    CDFs ([201, nCDF] float64), interfaceNormals (float32 [2, L] or None) and the
    sub-media index range of the deposition criteria (1-based, may be inf).
    """
    wavelengths = np.atleast_1d(np.asarray(wavelengths, dtype=np.float64))
    M_raw = np.asarray(M_raw)
    unique_media, M_trim = np.unique(M_raw, return_inverse=True)
    M_trim = M_trim.reshape(M_raw.shape) + 1
    trimmed = [mediaList[int(m) - 1] for m in unique_media]
    names_trim = [m.name for m in trimmed]
    if len(set(names_trim)) != len(names_trim):
        raise ValueError("Error: Two media have the same name.")
    nM = len(trimmed)
    nL = wavelengths.size
    nSMtotal = sum(int(getattr(m, "nBins", 1)) for m in trimmed)
    if nSMtotal > 256:
        raise ValueError("Error: The total number of (sub-)media may not exceed 256")
    FRd, Td, FDd = dependence_flags(trimmed)
    Mflat = M_trim.reshape(-1, order="F")
    shape = M_raw.shape
    FRf = np.broadcast_to(np.asarray(FR, dtype=np.float32), shape).reshape(-1, order="F")
    Tf = np.broadcast_to(np.asarray(T, dtype=np.float32), shape).reshape(-1, order="F")
    FDf = np.broadcast_to(np.asarray(FD, dtype=np.float32), shape).reshape(-1, order="F")
    mua = np.full((nSMtotal, nL), np.nan)
    mus = np.full((nSMtotal, nL), np.nan)
    g = np.full((nSMtotal, nL), np.nan)
    n = np.full((nSMtotal, nL), np.nan)
    CDFidx = np.full((nSMtotal, nL), np.nan)
    names = [None] * nSMtotal
    Msub = np.zeros(Mflat.size, dtype=np.int64)
    cdfs = []
    minSub, maxSub = np.inf, np.inf
    iSM = 0  # 0-based first sub-medium of the current medium
    for iM, med in enumerate(trimmed):
        idx = np.nonzero(Mflat == iM + 1)[0]
        dep = [FRd[iM, c] or Td[iM, c] or FDd[iM, c] for c in range(3)]
        FRs, Ts, FDs = FRf[idx], Tf[idx], FDf[idx]
        nSM = int(getattr(med, "nBins", 1))
        binidx = None
        for iL, L in enumerate(wavelengths):
            vals = []
            for c, (f, what) in enumerate(((med.mua, "mua"), (med.mus, "mus"), (med.g, "g"))):
                try:
                    v = _eval_dep(f, float(L), dep[c], FRs, Ts, FDs)
                except Exception as e:
                    raise ValueError("Error: The %s function of medium %s is throwing an error: %s" % (what, med.name, e))
                v = np.float32(math.nan) if v is None else v
                vals.append(np.asarray(v, dtype=np.float32))
            muav, musv, gv = vals
            if np.any(~np.isfinite(muav)):
                raise ValueError("The mua function of medium %s returns NaN or Inf values." % med.name)
            if np.any(~np.isfinite(musv)):
                raise ValueError("The mus function of medium %s returns NaN or Inf values." % med.name)
            if np.any(~np.isfinite(gv)) and not np.all(~np.isfinite(gv)):
                raise ValueError("The g function of medium %s returns NaN or Inf values in some, but not all voxels." % med.name)
            useg = not np.all(~np.isfinite(gv))
            if useg:
                cidx = math.nan
            else:
                cdf = custom_phase_cdf(med.customPhaseFunc, L)
                cidx = None
                for k, c in enumerate(cdfs):
                    if np.array_equal(c, cdf):
                        cidx = k
                        break
                if cidx is None:
                    cdfs.append(cdf)
                    cidx = len(cdfs) - 1
            nval = float(eval_optical(med.n, L))
            if DC.minMediumIdxToConsider == unique_media[iM]:
                minSub = iSM + 1
            if DC.maxMediumIdxToConsider == unique_media[iM]:
                maxSub = iSM + nSM
            rows = slice(iSM, iSM + nSM)
            if muav.ndim == 0 and musv.ndim == 0 and gv.ndim == 0:
                if iL == 0:
                    names[rows] = [med.name] * nSM
                    Msub[idx] = iSM + 1
                mua[rows, iL] = float(muav)
                mus[rows, iL] = float(musv)
                if useg:
                    g[rows, iL] = float(gv)
                n[rows, iL] = nval
                CDFidx[rows, iL] = cidx
            elif iL == 0:
                # one binning, from the first wavelength (getOpticalMediaProperties.m:148-165)
                if downsample is None:
                    raise ValueError("medium %s depends on FR, T or FD: splitting it needs the sub-media binning "
                                     "(pass downsample=native.downsample_params)" % med.name)
                par = np.zeros((3, idx.size), dtype=np.float32)
                par[0] = muav
                par[1] = musv
                par[2] = gv if useg else 0.0
                reps, lab = downsample(np.asfortranarray(par), nSM)
                reps = np.asarray(reps, dtype=np.float32)
                order = np.lexsort((reps[2], reps[1], reps[0]))  # sortrows of the representatives
                rank = np.empty(nSM, dtype=np.int64)
                rank[order] = np.arange(nSM)
                binidx = rank[np.asarray(lab, dtype=np.int64) - 1] + 1
                Msub[idx] = iSM + binidx
                reps = reps[:, order]
                names[rows] = [med.name] * nSM
                mua[rows, 0] = reps[0].astype(np.float64)
                mus[rows, 0] = reps[1].astype(np.float64)
                if useg:
                    g[rows, 0] = reps[2].astype(np.float64)
                n[rows, 0] = nval
                CDFidx[rows, 0] = cidx
            else:
                # later wavelengths: the mean of the new values in each bin (:167-196); a medium
                # that took one value on the first wavelength has all its voxels in its first bin
                if binidx is None:
                    binidx = np.ones(idx.size, dtype=np.int64)
                present = np.zeros(nSM, dtype=bool)
                present[np.unique(Msub[idx]) - 1 - iSM] = True
                for k in range(nSM):
                    if present[k]:
                        sel = binidx == k + 1
                        mua[iSM + k, iL] = float(muav) if muav.ndim == 0 else float(np.mean(muav[sel].astype(np.float64)))
                        mus[iSM + k, iL] = float(musv) if musv.ndim == 0 else float(np.mean(musv[sel].astype(np.float64)))
                        g[iSM + k, iL] = float(gv) if gv.ndim == 0 else float(np.mean(gv[sel].astype(np.float64)))
                    else:
                        mua[iSM + k, iL] = mua[iSM, iL]
                        mus[iSM + k, iL] = mus[iSM, iL]
                        g[iSM + k, iL] = g[iSM, iL]
                    n[iSM + k, iL] = nval
                    CDFidx[iSM + k, iL] = cidx
        iSM += nSM
    if matchedInterfaces:
        n[:] = 1.0
    if np.any(~np.isfinite(mua)) or np.any(mua <= 0):
        raise ValueError("Error: A medium has invalid mua. Must be finite, real and positive.")
    if np.any(~np.isfinite(mus)) or np.any(mus <= 0):
        raise ValueError("Error: A medium has invalid mus. Must be finite, real and positive.")
    if not np.all(np.isnan(g) | (np.isfinite(g) & (np.abs(g) <= 1))):
        raise ValueError("Error: A medium has invalid g. Must be finite, real and between -1 and 1, or NaN.")
    if np.any(np.isnan(n)) or np.any(n < 1):
        raise ValueError("Error: A medium has invalid n. Must not be NaN, must be real and at least 1.")
    M = np.asfortranarray(Msub.reshape(shape, order="F").astype(np.uint8))
    # `normals` may supply another implementation of interface_normals (the device one)
    normals = None if matchedInterfaces else (normals or interface_normals)(M, n, dx, dy, dz, smoothingLengthScale)
    CDFs = np.stack(cdfs, axis=1) if cdfs else np.zeros((0, 0))
    return dict(mua=mua, mus=mus, g=g, n=n, CDFidx=CDFidx, M=M, CDFs=CDFs,
                interfaceNormals=normals, minSubmediaIdx=minSub, maxSubmediaIdx=maxSub,
                names=names)


def _eval_yield(f, wavelength, FR, T, FD):
    """QY or ES of one medium at one wavelength over that medium's voxels: a number, f(wavelength)
    or f(wavelength, FR, T, FD) with FR, T, FD the voxels' arrays (element-wise, as the
    reference requires of four-argument functions, runMonteCarlo.m:135-137)."""
    if callable(f):
        return f(wavelength) if _nargs(f) == 1 else elementwise(f, wavelength, FR, T, FD)
    return f


def fluorescence_source(mediaList, M_raw, NA, Ls_E, Ls_F, FR, T, FD):
    """Fluorescence source distribution [nx, ny, nz, nL_F] float32 (runMonteCarlo.m:119-166).

    NA is the excitation run's normalised absorption [nx, ny, nz, nL_E]; FR, T and FD are the
    fluence rate, temperature and fractional damage grids the yields may depend on. Per voxel
    the emitted photon count is sum over excitation wavelengths of NA * QY * lambda_E (absorbed
    power / photon energy, up to a constant), spread over the fluorescence wavelengths by the
    voxel's emission spectrum normalised to unit sum, divided by lambda_F (power per photon).
    Media are indexed by the raw geometry (1-based positions in mediaList), as the reference
    loops over all media of the list.
    """
    Ls_E = np.atleast_1d(np.asarray(Ls_E, dtype=np.float64))
    Ls_F = np.atleast_1d(np.asarray(Ls_F, dtype=np.float64))
    shape = np.shape(M_raw)
    NA4 = np.asarray(NA, dtype=np.float64)
    if NA4.ndim == 3:
        NA4 = NA4[..., None]
    nLE, nLF = Ls_E.size, Ls_F.size
    if NA4.shape != tuple(shape) + (nLE,):
        raise ValueError("Error: normalizedAbsorption must be of size [nx, ny, nz, nLambda_excitation]")
    Mflat = np.asarray(M_raw).reshape(-1, order="F")
    NAf = NA4.reshape(-1, nLE, order="F")
    FRf = np.broadcast_to(np.asarray(FR, dtype=np.float32), shape).reshape(-1, order="F")
    Tf = np.broadcast_to(np.asarray(T, dtype=np.float32), shape).reshape(-1, order="F")
    FDf = np.broadcast_to(np.asarray(FD, dtype=np.float32), shape).reshape(-1, order="F")
    Fphotons = np.zeros(Mflat.size)
    emSp = np.full((Mflat.size, nLF), np.nan)
    for iM, med in enumerate(mediaList):
        idx = np.nonzero(Mflat == iM + 1)[0]
        if idx.size == 0:
            continue
        acc = np.zeros(idx.size)
        for iLE in range(nLE):
            try:
                qy = _eval_yield(med.QY, float(Ls_E[iLE]), FRf[idx], Tf[idx], FDf[idx])
            except Exception as e:
                raise ValueError("Error: The QY function of medium %s is throwing an error: %s" % (med.name, e))
            acc = acc + NAf[idx, iLE] * np.asarray(qy, dtype=np.float64) * Ls_E[iLE]
        Fphotons[idx] = acc
        for iLF in range(nLF):
            try:
                es = _eval_yield(med.ES, float(Ls_F[iLF]), FRf[idx], Tf[idx], FDf[idx])
            except Exception as e:
                raise ValueError("Error: The ES function of medium %s is throwing an error: %s" % (med.name, e))
            emSp[idx, iLF] = np.asarray(es, dtype=np.float64)
    if np.any(~np.isfinite(Fphotons)) or np.any(Fphotons < 0):
        raise ValueError("Error: A quantum yield function is returning values that are not finite, real and non-negative.")
    if np.any(~np.isfinite(emSp)) or np.any(emSp < 0):
        raise ValueError("Error: An emission spectrum function is returning values that are not finite, real and non-negative.")
    with np.errstate(invalid="ignore", divide="ignore"):
        emSp = emSp / emSp.sum(axis=1, keepdims=True)
        S = Fphotons[:, None] * emSp / Ls_F[None, :]
    S = S.astype(np.float32)  # FMC.sourceDistribution is a single-precision property
    if not np.nanmax(S, initial=0.0) > 0:
        raise ValueError("Error: No fluorescence emitters")
    return np.asfortranarray(S.reshape(tuple(shape) + (nLF,), order="F"))


def thermal_dependence_flags(media):
    """thmTdependent, thmFDdependent [nM, 2] (VHC, TC) as geometry.m:95-100 computes them: each
    property is evaluated on the (FR, T, FD) test grids and flagged when it changes along the
    grids' first axis (thmTdependent) or second axis (thmFDdependent). As written there, the first
    axis is the fluence-rate axis, so a temperature-dependent property shows up in thmFDdependent
    and thmTdependent stays false; the recalculation test uses their union (:520, :534)."""
    FR, T, FD = _test_grid()
    nM = len(media)
    thmT = np.zeros((nM, 2), dtype=bool)
    thmFD = np.zeros((nM, 2), dtype=bool)
    for iM, med in enumerate(media):
        for col, f in enumerate((med.VHC, med.TC)):
            if not callable(f):
                continue
            vals = np.broadcast_to(np.asarray(elementwise(f, T, FD), dtype=np.float64), FR.shape)
            thmT[iM, col] = _varies(vals, 0)
            thmFD[iM, col] = _varies(vals, 1)
    return thmT, thmFD


def thermal_media_properties(mediaList, M_raw, T=37.0, FD=0.0, downsample=None):
    """VHC, TC, A, E per sub-medium and the sub-medium grid (getThermalMediaProperties.m:27-96).

    VHC and TC are evaluated per voxel at the voxel's temperature and fractional damage; every
    medium is then split into nBins sub-media by the sub-media binning of the (VHC, TC, 1) triples
    (the `downsample` callable, native.downsample_params on the device; only needed when a
    medium's values differ between voxels, otherwise every voxel keeps the common value), with
    the representatives sorted as MATLAB's sortrows orders them.
    """
    M_raw = np.asarray(M_raw)
    unique_media, M_trim = np.unique(M_raw, return_inverse=True)
    M_trim = M_trim.reshape(M_raw.shape) + 1
    trimmed = [mediaList[int(m) - 1] for m in unique_media]
    names_trim = [m.name for m in trimmed]
    if len(set(names_trim)) != len(names_trim):
        raise ValueError("Error: Two media have the same name.")
    nSMtotal = sum(int(getattr(m, "nBins", 1)) for m in trimmed)
    if nSMtotal > 256:
        raise ValueError("Error: The total number of (sub-)media may not exceed 256")
    shape = M_raw.shape
    Mflat = M_trim.reshape(-1, order="F")
    Tf = np.broadcast_to(np.asarray(T, dtype=np.float32), shape).reshape(-1, order="F")
    FDf = np.broadcast_to(np.asarray(FD, dtype=np.float32), shape).reshape(-1, order="F")
    VHC = np.full(nSMtotal, np.nan)
    TC = np.full(nSMtotal, np.nan)
    A = np.full(nSMtotal, np.nan)
    E = np.full(nSMtotal, np.nan)
    names = [None] * nSMtotal
    Msub = np.zeros(Mflat.size, dtype=np.int64)
    iSM = 0
    for iM, med in enumerate(trimmed):
        idx = np.nonzero(Mflat == iM + 1)[0]
        par = np.ones((3, idx.size), dtype=np.float32)
        for row, (f, what) in enumerate(((med.VHC, "VHC"), (med.TC, "TC"))):
            try:
                v = elementwise(f, Tf[idx], FDf[idx]) if callable(f) else f
            except Exception as e:
                raise ValueError("Error: The %s function of medium %s is throwing an error: %s" % (what, med.name, e))
            par[row] = np.asarray(v, dtype=np.float32)
            if np.any(~np.isfinite(par[row])) or np.any(par[row] <= 0):
                raise ValueError("The %s function of medium %s returns values that are not finite and positive." % (what, med.name))
        nSM = int(getattr(med, "nBins", 1))
        if np.all(par == par[:, :1]):
            reps = np.repeat(par[:, :1], nSM, axis=1)  # the binning of a single value
            lab = np.ones(idx.size, dtype=np.int64)
        else:
            if downsample is None:
                raise ValueError("medium %s has voxel-dependent thermal properties: splitting it needs the sub-media "
                                 "binning (pass downsample=native.downsample_params)" % med.name)
            reps, lab = downsample(np.asfortranarray(par), nSM)
            reps = np.asarray(reps, dtype=np.float32)
        order = np.lexsort((reps[2], reps[1], reps[0]))
        rank = np.empty(nSM, dtype=np.int64)
        rank[order] = np.arange(nSM)
        Msub[idx] = iSM + rank[np.asarray(lab, dtype=np.int64) - 1] + 1
        reps = reps[:, order]
        names[iSM:iSM + nSM] = [med.name] * nSM
        VHC[iSM:iSM + nSM] = reps[0].astype(np.float64)
        TC[iSM:iSM + nSM] = reps[1].astype(np.float64)
        A[iSM:iSM + nSM] = float(med.A)
        E[iSM:iSM + nSM] = float(med.E)
        iSM += nSM
    return dict(VHC=VHC, TC=TC, A=A, E=E, M=np.asfortranarray(Msub.reshape(shape, order="F").astype(np.uint8)),
                names=names, nBins=[int(getattr(m, "nBins", 1)) for m in trimmed])


def calc_dTdt_arrays(VHC, TC, dx, dy, dz, NA_sum, P, M1):
    """dTdtperdeltaT [nM, nM, 3] and dTdt_abs [L] in single precision (simulateHeatDistribution.m:469-494).

    TC_eff(i, j) = 2 TC_i TC_j / (TC_i + TC_j); c(i, j, d) = TC_eff(i, j) / VHC_i / d_d^2;
    dTdt_abs = NA * P / VHC(M). NA_sum is the normalised absorption summed over wavelengths.
    """
    VHC = np.asarray(VHC, dtype=np.float32)
    TC = np.asarray(TC, dtype=np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        TC_eff = (2 * np.outer(TC, TC) / (TC[None, :] + TC[:, None])).astype(np.float32)
    TC_eff[np.isnan(TC_eff)] = 0
    rowv = VHC[:, None]
    c = np.empty((len(VHC), len(VHC), 3), dtype=np.float32)
    # MATLAB evaluates single-double mixtures in single precision
    c[:, :, 0] = (TC_eff / rowv) / np.float32(dx ** 2)
    c[:, :, 1] = (TC_eff / rowv) / np.float32(dy ** 2)
    c[:, :, 2] = (TC_eff / rowv) / np.float32(dz ** 2)
    NAP = (np.asarray(NA_sum, dtype=np.float64) * P).astype(np.float32)
    dTdt_abs = NAP / VHC[M1.astype(np.int64) - 1]
    return np.asfortranarray(c), np.asfortranarray(dTdt_abs)


def calc_dtmax(M1, TC, VHC, dx, dy, dz):
    """Smallest explicit-stability time step over all voxels (simulateHeatDistribution.m:496-514)."""
    TCv = np.asarray(TC, dtype=np.float32)[M1.astype(np.int64) - 1]
    VHCv = np.asarray(VHC, dtype=np.float32)[M1.astype(np.int64) - 1]
    nx, ny, nz = M1.shape
    ex = np.zeros((nx + 1, ny, nz), np.float32)
    ey = np.zeros((nx, ny + 1, nz), np.float32)
    ez = np.zeros((nx, ny, nz + 1), np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        ex[1:-1] = 2 * TCv[:-1] * TCv[1:] / (TCv[:-1] + TCv[1:])
        ey[:, 1:-1] = 2 * TCv[:, :-1] * TCv[:, 1:] / (TCv[:, :-1] + TCv[:, 1:])
        ez[:, :, 1:-1] = 2 * TCv[:, :, :-1] * TCv[:, :, 1:] / (TCv[:, :, :-1] + TCv[:, :, 1:])
    for e in (ex, ey, ez):
        e[np.isnan(e)] = 0
    fx, fy, fz = np.float32(dx ** 2), np.float32(dy ** 2), np.float32(dz ** 2)
    denom = (ex[:-1] / fx + ex[1:] / fx + ey[:, :-1] / fy + ey[:, 1:] / fy
             + ez[:, :, :-1] / fz + ez[:, :, 1:] / fz)
    with np.errstate(divide="ignore"):
        ind = VHCv / denom
    return float(np.min(ind))


def convert_temp_sensor_pos(positions, x, y, z):
    """Corner voxel (0-based linear index) and interpolation weights of each sensor (simulateHeatDistribution.m:543-609)."""
    positions = np.atleast_2d(np.asarray(positions, dtype=np.float64))
    nS = positions.shape[0] if positions.size else 0
    nx, ny, nz = len(x), len(y), len(z)
    li = np.zeros(nS)
    w = np.zeros((nS, 3))
    axes = [(x, nx), (y, ny), (z, nz)]
    for i in range(nS):
        idx = []
        for d, (ax, n) in enumerate(axes):
            step = ax[1] - ax[0]
            rel = positions[i, d] - ax[0]
            if rel < 0:
                k, wt = 0, 0.0
            elif rel < ax[-1] - ax[0]:
                k, wt = int(math.floor(rel / step)), math.fmod(rel / step, 1.0)
            else:
                k, wt = n - 2, 1.0
            idx.append(k)
            w[i, d] = wt
        li[i] = idx[0] + idx[1] * nx + idx[2] * nx * ny
    return li, w


def heat_schedule(durationOn, durationOff, durationEnd, nUpdates, dtmax):
    """Updates, steps per update and dt per phase (simulateHeatDistribution.m:80-110)."""
    tot = durationOn + durationOff
    out = {}
    if durationOn != 0:
        nU = max(1, round(nUpdates * durationOn / tot))
        nT = math.ceil(durationOn / nU / dtmax)
        out["on"] = (nU, nT, durationOn / nU / nT)
    else:
        out["on"] = (0, 1, 1.0)
    if durationOff != 0:
        nU = max(1, nUpdates - out["on"][0])
        nT = math.ceil(durationOff / nU / dtmax)
        out["off"] = (nU, nT, durationOff / nU / nT)
    else:
        out["off"] = (0, 1, 1.0)
    if durationEnd != 0:
        nU = max(1, round(nUpdates * durationEnd / tot))
        nT = math.ceil(durationEnd / nU / dtmax)
        out["end"] = (nU, nT, durationEnd / nU / nT)
    else:
        out["end"] = (0, 1, 1.0)
    return out
