"""Summary statistics and a batch z-test for comparing Monte Carlo outputs.

Two MC implementations agree when, for K independent batches of each, every summary
statistic's mean differs by less than `zmax` combined standard errors. The statistics
are linear in the tallies (integrated absorbed power per medium, escape fraction per
face, depth and radial profiles), so each is an unbiased estimator with a finite
variance and the batch means are close to normal.
"""
from __future__ import annotations

import numpy as np


def summaries(out, mc_in, zbins=8, rbins=6):
    """Vector of summary statistics from one run's normalised outputs (MATLAB shapes)."""
    s = {}
    dx, dy, dz = mc_in["dx"], mc_in["dy"], mc_in["dz"]
    V = dx * dy * dz
    M = np.asarray(mc_in["M"]).astype(np.int64) - 1
    mua = np.asarray(mc_in["mua"])
    nL = mua.shape[1]
    if "NFR" in out and out["NFR"] is not None and np.size(out["NFR"]) > 1:
        NFR = np.asarray(out["NFR"], dtype=np.float64)
        if NFR.ndim == 3:
            NFR = NFR[..., None]
        for iL in range(nL):
            absorbed = NFR[..., iL] * mua[:, iL][M] * V  # power absorbed per voxel / incident power
            for m in range(mua.shape[0]):
                s["abs_m%d_l%d" % (m, iL)] = absorbed[M == m].sum()
            nz = absorbed.shape[2]
            edges = np.linspace(0, nz, zbins + 1).astype(int)
            for b in range(zbins):
                s["absz%d_l%d" % (b, iL)] = absorbed[:, :, edges[b]:edges[b + 1]].sum()
            # fluence in a central column (log-scale quantity would be biased; keep linear)
            cx, cy = NFR.shape[0] // 2, NFR.shape[1] // 2
            col = NFR[max(cx - 2, 0):cx + 2, max(cy - 2, 0):cy + 2, :, iL].mean(axis=(0, 1))
            for b in range(zbins):
                s["colz%d_l%d" % (b, iL)] = col[edges[b]:edges[b + 1]].mean() * 1e-3
    faces = {"NI_xpos": dy * dz, "NI_xneg": dy * dz, "NI_ypos": dx * dz, "NI_yneg": dx * dz,
             "NI_zpos": dx * dy, "NI_zneg": dx * dy}
    for k, area in faces.items():
        a = out.get(k)
        if a is None or np.size(a) <= 1:
            continue
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 2:
            a = a[..., None]
        for iL in range(a.shape[2]):
            s["%s_l%d" % (k, iL)] = a[..., iL].sum() * area
        if k == "NI_zneg":
            # radial reflectance profile about the centre
            n0, n1 = a.shape[0], a.shape[1]
            X, Y = np.meshgrid(np.arange(n0) - (n0 - 1) / 2, np.arange(n1) - (n1 - 1) / 2, indexing="ij")
            r = np.hypot(X, Y)
            edges = np.linspace(0, r.max() + 1e-9, rbins + 1)
            for b in range(rbins):
                msk = (r >= edges[b]) & (r < edges[b + 1])
                s["Rr%d" % b] = a[..., 0][msk].sum() * area
    for k in ("image", "farField"):
        a = out.get(k)
        if a is None or np.size(a) <= 1 or (np.ndim(a) and not np.any(np.isfinite(a))):
            continue
        a = np.asarray(a, dtype=np.float64)
        s[k + "_sum"] = a.sum()
        if k == "image" and a.ndim >= 3 and a.shape[2] > 1:
            tb = a.sum(axis=(0, 1))[..., 0] if a.ndim == 4 else a.sum(axis=(0, 1))
            tb = np.asarray(tb).ravel()
            edges = np.linspace(0, tb.size, 5).astype(int)
            for b in range(4):
                s["img_t%d" % b] = tb[edges[b]:edges[b + 1]].sum()
        if k == "farField":
            th = a.sum(axis=1)
            th = th[..., 0] if th.ndim > 1 else th
            edges = np.linspace(0, th.size, 5).astype(int)
            for b in range(4):
                s["ff_th%d" % b] = th[edges[b]:edges[b + 1]].sum()
    if "nPhotonsCollected" in out and out["nPhotonsCollected"] is not None:
        npc = float(np.asarray(out["nPhotonsCollected"]).ravel()[0])
        nph = float(np.asarray(out["nPhotons"]).ravel()[0])
        if npc > 0:
            s["collected_frac"] = npc / nph
    return s


def ztest(batches_a, batches_b, zmax=4.5, rel_floor=0.0):
    """Compares per-key batch means. Returns (ok, report, worst_z)."""
    keys = sorted(set(batches_a[0]) & set(batches_b[0]))
    worst = 0.0
    lines = []
    ok = True
    for k in keys:
        a = np.array([b[k] for b in batches_a], dtype=np.float64)
        b = np.array([x[k] for x in batches_b], dtype=np.float64)
        ma, mb = a.mean(), b.mean()
        se = np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)
        se = max(se, rel_floor * max(abs(ma), abs(mb)), 1e-300)
        if ma == mb:
            z = 0.0
        else:
            z = abs(ma - mb) / se
        worst = max(worst, z)
        lines.append("%-16s %.6g %.6g z=%.2f" % (k, ma, mb, z))
        if z > zmax:
            ok = False
    return ok, "\n".join(lines), worst


def welch_z(ma, va, na, mb, vb, nb):
    """Normal-equivalent z of the Welch t statistic for the difference of two batch means.

    ma, mb: batch means; va, vb: batch variances (ddof 1); na, nb: batch counts. The Welch t
    (unequal variances, Welch-Satterthwaite degrees of freedom) is mapped through its own
    tail probability to the standard normal quantile with the same tail, so that under equal
    means z is N(0, 1) for normal batch values whatever the batch counts: |z| > 3 then has the
    normal 0.27% rate and mean(z^2) has expectation 1."""
    from scipy import stats
    ma, va, mb, vb = (np.asarray(x, dtype=np.float64) for x in (ma, va, mb, vb))
    sa, sb = va / na, vb / nb
    se2 = sa + sb
    z = np.zeros(np.broadcast(ma, mb).shape)
    ok = se2 > 0
    t = np.where(ok, (ma - mb) / np.sqrt(np.where(ok, se2, 1.0)), 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        dof = se2 ** 2 / (sa ** 2 / (na - 1) + sb ** 2 / (nb - 1))
    dof = np.where(ok & np.isfinite(dof), dof, 1e6)
    p = stats.t.sf(np.abs(t), dof)
    z = np.sign(t) * stats.norm.isf(np.clip(p, 1e-300, 0.5))
    return np.where(ok, z, np.where(ma == mb, 0.0, np.inf))


def voxel_chi2(ma, va, na, mb, vb, nb):
    """Voxel-wise agreement of two batch-mean fields: (chi^2 / dof of the Welch z values,
    fraction of voxels beyond 3 sigma, the z values)."""
    z = welch_z(ma, va, na, mb, vb, nb)
    return float(np.mean(z ** 2)), float(np.mean(np.abs(z) > 3.0)), z
