"""Shared perturbation-MC test case: the 8-medium layered cube (configs.perturbation_cube) at a
test size, its objectives (radial reflectance bins on the top face, mean fluence rate in a box
under the beam) and the flattening of a gradient result into summary statistics."""
from __future__ import annotations

import numpy as np

from mcmatlab_b200 import configs, mexargs

# media whose derivatives carry signal in the small case (1-based 2, 3: the top two tissue layers)
MEDIA = (1, 2)


def case(n=24, nPhotons=2e4, seed=1):
    mc_in = mexargs.prepare_mc(configs.perturbation_cube(n=n, nPhotons=nPhotons, seed=seed))
    box = [n // 4, 3 * n // 4, n // 4, 3 * n // 4, 1, n // 2]
    obj = dict(nRadialBins=8, radialBinWidth=0.25 / 8, box=box)
    return mc_in, obj


def summary(g, nbins=4):
    s = {"F": g["F"]}
    for j in MEDIA:
        s["dF_dmua%d" % j] = g["dF_dmua"][j]
        s["dF_dmus%d" % j] = g["dF_dmus"][j]
        for b in range(nbins):
            s["dR%d_dmua%d" % (b, j)] = g["dR_dmua"][b, j]
            s["dR%d_dmus%d" % (b, j)] = g["dR_dmus"][b, j]
    for b in range(nbins):
        s["R%d" % b] = g["R"][b]
    return s


def perturbed(mc_in, name, j, factor):
    out = dict(mc_in)
    a = np.array(mc_in[name], dtype=np.float64).copy()
    a[j, :] *= factor
    out[name] = a
    return out


def fd_differences(run, mc_in, obj, h=0.02):
    """Per-seed differences (analytic - central finite difference with common random numbers)
    of the box fluence and the first reflectance bin, for mua and mus of MEDIA."""
    _, g = run(mc_in, obj)
    d = {}
    for j in MEDIA:
        for name in ("mua", "mus"):
            _, gp = run(perturbed(mc_in, name, j, 1 + h), obj)
            _, gm = run(perturbed(mc_in, name, j, 1 - h), obj)
            step = 2 * h * float(np.asarray(mc_in[name])[j, 0])
            d["F_%s%d" % (name, j)] = g["dF_d" + name][j] - (gp["F"] - gm["F"]) / step
            d["R0_%s%d" % (name, j)] = g["dR_d" + name][0, j] - (gp["R"][0] - gm["R"][0]) / step
    return d


def zero_mean_test(diffs, zmax=4.5):
    """Every key's mean over the per-seed differences is zero within zmax standard errors."""
    bad = []
    for k in diffs[0]:
        v = np.array([d[k] for d in diffs])
        se = v.std(ddof=1) / np.sqrt(v.size)
        if se == 0:
            if np.any(v != 0):
                bad.append((k, float(v.mean()), 0.0))
            continue
        z = abs(v.mean()) / se
        if z > zmax:
            bad.append((k, float(v.mean()), float(se)))
    return bad
