"""The FP64 oracle pinned at the transport benchmark's configuration (100^3 standard-tissue cube,
pencil beam, 1e6 packets per run) against the 32 reference batches of tests/golden/mc_c0_ref.npz,
with the statistics of tests/test_gpu_mc_c0.py; and the Welch-to-normal mapping those tests use,
checked on synthetic normal batches."""
import os

import numpy as np

import mcstats
from mcmatlab_b200 import configs, mexargs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mc_c0_ref.npz")
K_ORC = 16
AGGREGATES = ["abs_m%d_l0" % m for m in range(4)] + ["NI_%s_l0" % f for f in ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")]


def test_welch_z_is_standard_normal_under_equal_means():
    rng = np.random.default_rng(5)
    n = 200000
    mu = rng.uniform(1, 10, n)
    sa, sb = mu * rng.uniform(0.05, 0.2, n), mu * rng.uniform(0.05, 0.2, n)
    a = mu + sa * rng.standard_normal((64, n))
    b = mu + sb * rng.standard_normal((32, n))
    chi2, frac3, z = mcstats.voxel_chi2(a.mean(0), a.var(0, ddof=1), 64, b.mean(0), b.var(0, ddof=1), 32)
    assert abs(chi2 - 1) < 0.01 and abs(frac3 - 0.0027) < 0.0005 and abs(np.mean(z)) < 0.01
    # a shift of one combined standard error moves chi^2 / dof by about 1
    se = np.sqrt(sa ** 2 / 64 + sb ** 2 / 32)
    chi2s, _, _ = mcstats.voxel_chi2(a.mean(0) + se, a.var(0, ddof=1), 64, b.mean(0), b.var(0, ddof=1), 32)
    assert chi2s > 1.8


def test_golden_c0_fixture_layout():
    g = np.load(GOLD)
    mask = np.unpackbits(g["mask"])[:100 ** 3].astype(bool)
    assert int(g["K"]) == 32 and mask.sum() == g["nfr_mean"].size == g["nfr_sd"].size
    assert g["summaries"].shape == (32, len(g["keys"]))
    assert np.all(g["nfr_sd"] < float(g["cv_max"]) * g["nfr_mean"])


def test_oracle_matches_reference_at_c0(oracle_lib):
    from oracle import orc
    g = np.load(GOLD)
    keys = list(g["keys"])
    Kr = int(g["K"])
    mc_in = mexargs.prepare_mc(configs.standard_tissue_cube(n=100, nPhotons=1e6, seed=1))
    mask = np.unpackbits(g["mask"])[:100 ** 3].astype(bool)
    vals, summ = [], []
    for k in range(K_ORC):
        mc_in["seed"] = 1 + k
        out = orc.oracle_mc(mc_in, 0)
        summ.append(mcstats.summaries(out, mc_in))
        v = np.asarray(out["NFR"], dtype=np.float64)
        vals.append((v[..., 0] if v.ndim == 4 else v).ravel(order="F")[mask])
    X = np.array(vals)
    lines = []
    for k in AGGREGATES:
        r = g["summaries"][:, keys.index(k)]
        a = np.array([s[k] for s in summ])
        z = float(mcstats.welch_z(a.mean(), a.var(ddof=1), K_ORC, r.mean(), r.var(ddof=1), Kr))
        lines.append("%-12s oracle %.6g ref %.6g z=%+.2f" % (k, a.mean(), r.mean(), z))
        assert abs(z) < 3.0, "\n".join(lines)
    chi2, frac3, _ = mcstats.voxel_chi2(X.mean(0), X.var(0, ddof=1), K_ORC, g["nfr_mean"], g["nfr_sd"].astype(np.float64) ** 2, Kr)
    print("\n".join(lines), "\noracle C0 voxel-wise chi2/dof %.4f, beyond 3 sigma %.3f%%" % (chi2, 100 * frac3))
    assert abs(chi2 - 1) < 0.1 and frac3 < 0.006
