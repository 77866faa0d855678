"""Synthetic, seeded workload definitions used by the tests and the benchmark.

No public dataset is involved; each workload is generated from its description:

* standard_tissue_cube(n)  — cube of side 0.1 cm with n^3 voxels: air above z = 0.01 cm,
  an epidermis-like layer to z = 0.016 cm, dermis below, and a y-aligned vessel of
  radius 0.01 cm centred at x = 0 (centred coordinates), z = 0.04 cm. Pencil beam at
  the centre, all cuboid faces escaping, refractive index mismatches on.
* heat_on_cube(...)        — thermal properties for the same geometry (tissue VHC 3.9,
  TC 0.0037; air VHC 0.0012, TC 0.00026), damage (E = 4.48e5, A = 7.6e66) in the vessel.
* batched_sweep(...)       — seeded instances of layered media + one cylinder with
  randomised grids, wavelengths and optical properties.
* perturbation_cube(...)   — 8 seeded tissue media (layers + ellipsoids) under an air layer.
* heat_adjoint_case(...)   — 4 seeded thermal media, a Gaussian heat-source blob, a damage
  target ellipsoid and a sparing region (adjoint objectives).
"""
from __future__ import annotations

import math

import numpy as np

from . import model as mm


def _tissue_media(params):
    air = mm.mediumProperties(name="air", mua=1e-8, mus=1e-8, g=1.0, n=1.0, VHC=0.0012, TC=0.00026)
    epi = mm.mediumProperties(name="epidermis", mua=10.0, mus=150.0, g=0.9, n=1.3, VHC=3.9, TC=0.0037)
    der = mm.mediumProperties(name="dermis", mua=1.0, mus=100.0, g=0.9, n=1.3, VHC=3.9, TC=0.0037)
    ves = mm.mediumProperties(name="blood vessel", mua=200.0, mus=100.0, g=0.9, n=1.3, VHC=3.9, TC=0.0037,
                              E=4.48e5, A=7.6e66)
    return [air, epi, der, ves]


def _tissue_geom(X, Y, Z, params):
    M = np.full(X.shape, 3.0)
    M[Z < 0.016] = 2
    M[Z < 0.01] = 1
    M[(X - 0.0) ** 2 + (Z - 0.04) ** 2 < 0.01 ** 2] = 4
    return M


def standard_tissue_cube(n=100, nPhotons=1e6, seed=1, matched=False):
    m = mm.model()
    m.G.nx = m.G.ny = m.G.nz = n
    m.G.Lx = m.G.Ly = m.G.Lz = 0.1
    m.G.mediaPropertiesFunc = _tissue_media
    m.G.geomFunc = _tissue_geom
    m.MC.nPhotonsRequested = nPhotons
    m.MC.seed = seed
    m.MC.matchedInterfaces = matched
    m.MC.boundaryType = 1
    m.MC.wavelength = 532.0
    m.MC.lightSource.sourceType = 0
    m.MC.silentMode = True
    m.G.updateGeometry()
    return m


def heat_on_cube(m, durationOn=0.5, durationOff=0.5, nUpdates=10, dtFactor=0.9):
    m.HS.T = 37.0
    m.HS.durationOn = durationOn
    m.HS.durationOff = durationOff
    m.HS.nUpdates = nUpdates
    m.HS.heatBoundaryType = 0
    m.HS.dtFactor = dtFactor
    m.HS.silentMode = True
    return m


def _layered_media_factory(rng, wavelengths):
    """Three layers plus one cylinder; per-medium mua log-uniform(0.1, 300)/cm per wavelength,
    mus = a (lambda/500 nm)^-b, g in [0.7, 0.95], n in {1.0, 1.37, 1.4}."""
    nmed = 4
    mua_tab = {float(w): np.exp(rng.uniform(np.log(0.1), np.log(300.0), nmed)) for w in wavelengths}
    a = rng.uniform(50.0, 300.0, nmed)
    b = rng.uniform(0.5, 2.0, nmed)
    g = rng.uniform(0.7, 0.95, nmed)
    nvals = np.array([1.0, 1.37, 1.4])
    n = nvals[rng.integers(0, 3, nmed)]
    n[0] = 1.0  # top layer index-matched to the outside so packets can escape through it

    def media(params):
        out = []
        for k in range(nmed):
            out.append(mm.mediumProperties(
                name="medium%d" % k,
                mua=(lambda wl, k=k: mua_tab[float(wl)][k]),
                mus=(lambda wl, k=k: a[k] * (wl / 500.0) ** (-b[k])),
                g=float(g[k]), n=float(n[k])))
        return out
    return media


def batched_sweep(n_instances=64, seed=7, min_grid=(64, 64, 64), max_grid=(200, 200, 150),
                  photons=(1e5, 1e7), scale=1.0):
    """Seeded instances for a batched launch (grids, wavelengths, media, photon counts, Gaussian beams).

    Half the instances add time tagging (64 bins to 1 ns on a fibre light collector) and cyclic
    x/y boundaries. `scale` multiplies photon counts (tests use small values).
    """
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_instances):
        nx = int(rng.integers(min_grid[0], max_grid[0] + 1))
        ny = int(rng.integers(min_grid[1], max_grid[1] + 1))
        nz = int(rng.integers(min_grid[2], max_grid[2] + 1))
        wl = float(rng.uniform(450.0, 900.0))
        m = mm.model()
        m.G.nx, m.G.ny, m.G.nz = nx, ny, nz
        m.G.Lx = m.G.Ly = 0.2
        m.G.Lz = 0.15
        m.G.mediaPropertiesFunc = _layered_media_factory(rng, [wl])
        t1, t2 = sorted(rng.uniform(0.01, 0.08, 2))
        cz = float(rng.uniform(0.05, 0.12))
        r = float(rng.uniform(0.005, 0.02))

        def geom(X, Y, Z, p, t1=t1, t2=t2, cz=cz, r=r):
            M = np.full(X.shape, 3.0)
            M[Z < t2] = 2
            M[Z < t1] = 1
            M[X ** 2 + (Z - cz) ** 2 < r ** 2] = 4
            return M
        m.G.geomFunc = geom
        m.MC.wavelength = wl
        m.MC.matchedInterfaces = False
        m.MC.nPhotonsRequested = float(max(1000, round(math.exp(rng.uniform(math.log(photons[0]), math.log(photons[1]))) * scale)))
        m.MC.seed = 1000 + i
        m.MC.silentMode = True
        m.MC.lightSource.sourceType = 4
        m.MC.lightSource.FPID.radialDistr = 1
        m.MC.lightSource.FPID.radialWidth = float(rng.uniform(0.005, 0.02))
        m.MC.lightSource.AID.radialDistr = 1
        m.MC.lightSource.AID.radialWidth = 0.0
        if i % 2 == 1:
            m.MC.boundaryType = 3
            m.MC.useLightCollector = True
            lc = m.MC.lightCollector
            lc.x, lc.y, lc.z = 0.0, 0.0, -0.05
            lc.theta, lc.phi = 0.0, math.pi / 2
            lc.f = math.inf
            lc.diam = 0.1
            lc.NA = 0.5
            lc.res = 1
            lc.tStart, lc.tEnd, lc.nTimeBins = 0.0, 1e-9, 64
        else:
            m.MC.boundaryType = 1
        m.G.updateGeometry()
        out.append(m)
    return out


def perturbation_cube(n=256, nPhotons=1e8, seed=11, media_seed=5, L=0.5):
    """Perturbation-MC workload: an n^3 cube of side L cm with 8 tissue media (6 z-layers and 2
    ellipsoidal inclusions, seeded mua in [0.1, 50] /cm, mus in [20, 400] /cm, g = 0.9, n = 1.4)
    under a one-voxel air layer (mua = mus = 1e-8, n = 1) so that light can escape through the
    top face (MCmatlab counts an escape only where the refractive index is 1). Pencil beam at
    the centre, all faces escaping."""
    rng = np.random.default_rng(media_seed)
    mua = np.exp(rng.uniform(np.log(0.1), np.log(50.0), 8))
    mus = np.exp(rng.uniform(np.log(20.0), np.log(400.0), 8))
    bounds = np.sort(rng.uniform(0.05, 0.95, 5)) * L
    ell = [(rng.uniform(-0.25, 0.25) * L, rng.uniform(-0.25, 0.25) * L, rng.uniform(0.2, 0.7) * L,
            rng.uniform(0.05, 0.15) * L, rng.uniform(0.05, 0.15) * L, rng.uniform(0.03, 0.1) * L) for _ in range(2)]
    dz = L / n

    def media(params):
        out = [mm.mediumProperties(name="air", mua=1e-8, mus=1e-8, g=1.0, n=1.0)]
        for k in range(8):
            out.append(mm.mediumProperties(name="tissue%d" % k, mua=float(mua[k]), mus=float(mus[k]), g=0.9, n=1.4))
        return out

    def geom(X, Y, Z, p):
        M = np.full(X.shape, 7.0)  # deepest layer; media indices are 1-based (1 = air, 2..9 = tissue0..7)
        for k in range(5):
            M[Z < bounds[4 - k]] = 6 - k
        for q, (cx, cy, cz, ax, ay, az) in enumerate(ell):
            M[((X - cx) / ax) ** 2 + ((Y - cy) / ay) ** 2 + ((Z - cz) / az) ** 2 < 1] = 8 + q
        M[Z < dz] = 1
        return M

    m = mm.model()
    m.G.nx = m.G.ny = m.G.nz = n
    m.G.Lx = m.G.Ly = m.G.Lz = L
    m.G.mediaPropertiesFunc = media
    m.G.geomFunc = geom
    m.MC.nPhotonsRequested = nPhotons
    m.MC.seed = seed
    m.MC.matchedInterfaces = False
    m.MC.boundaryType = 1
    m.MC.wavelength = 700.0
    m.MC.silentMode = True
    m.G.updateGeometry()
    return m


def heat_adjoint_case(shape=(300, 300, 200), size=(1.0, 1.0, 0.6), nt=2000, seed=21, peak=50.0, dtFactor=0.9,
                      heatBoundaryType=0, T0=37.0):
    """Heat-adjoint workload: a grid of `shape` voxels over `size` cm with 4 media (a bulk, a top
    layer, a deep layer and an ellipsoidal target), seeded TC in [0.002, 0.006] W/cm/K and VHC in
    [3.0, 4.2] J/cm^3/K, a Gaussian heat-source blob of `peak` W/cm^3 centred on the target, and
    Arrhenius damage (E = 4.48e5 J/mol, A = 7.6e66 /s) in the target medium. Objectives: damage
    summed over the target ellipsoid (weight 1 per voxel) and the mean peak temperature over a
    sparing region (a slab above the target; weight 1/count). dt = dtFactor x the explicit limit.

    Returns dict(T0, hp (heatSimParameters), wd, wp, n, TC, VHC, S (W/cm^3), M1 (1-based), d)."""
    from . import mexargs, prep
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    Lx, Ly, Lz = size
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
    x = (np.arange(nx) + 0.5) * dx - Lx / 2
    y = (np.arange(ny) + 0.5) * dy - Ly / 2
    z = (np.arange(nz) + 0.5) * dz
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    TC = rng.uniform(0.002, 0.006, 4)
    VHC = rng.uniform(3.0, 4.2, 4)
    zt, zd = rng.uniform(0.1, 0.2) * Lz, rng.uniform(0.7, 0.85) * Lz
    c0 = np.array([rng.uniform(-0.1, 0.1) * Lx, rng.uniform(-0.1, 0.1) * Ly, rng.uniform(0.4, 0.55) * Lz])
    ax = np.array([rng.uniform(0.08, 0.15) * Lx, rng.uniform(0.08, 0.15) * Ly, rng.uniform(0.08, 0.15) * Lz])
    M1 = np.ones(shape, dtype=np.uint8)
    M1[Z < zt] = 2
    M1[Z > zd] = 3
    inT = ((X - c0[0]) / ax[0]) ** 2 + ((Y - c0[1]) / ax[1]) ** 2 + ((Z - c0[2]) / ax[2]) ** 2 < 1
    M1[inT] = 4
    w = 1.5 * ax
    S = peak * np.exp(-((X - c0[0]) ** 2 / w[0] ** 2 + (Y - c0[1]) ** 2 / w[1] ** 2 + (Z - c0[2]) ** 2 / w[2] ** 2))
    c, Q = prep.calc_dTdt_arrays(VHC, TC, dx, dy, dz, S, 1.0, M1)
    dtmax = prep.calc_dtmax(M1, TC, VHC, dx, dy, dz)
    A = np.array([0.0, 0.0, 0.0, 7.6e66])
    E = np.array([0.0, 0.0, 0.0, 4.48e5])
    hp = mexargs.heat_mex_params(M1, A, E, c, Q, True, heatBoundaryType, None, None, True, nt, dtFactor * dtmax)
    wd = inT.astype(np.float32)
    spare = (Z > zt) & (Z < c0[2] - ax[2]) & (np.abs(X - c0[0]) < ax[0]) & (np.abs(Y - c0[1]) < ax[1]) & ~inT
    wp = np.where(spare, 1.0 / max(int(spare.sum()), 1), 0.0).astype(np.float32)
    T0a = np.full(shape, T0, dtype=np.float32, order="F")
    return dict(T0=T0a, hp=hp, wd=np.asfortranarray(wd), wp=np.asfortranarray(wp), n=shape, TC=TC, VHC=VHC,
                S=S, M1=M1, d=(dx, dy, dz))
