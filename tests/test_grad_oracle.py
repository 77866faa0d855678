"""Perturbation-MC estimator in the FP64 oracle: its value outputs restate MCmatlab's normalised
tallies of the same run, and its derivatives agree with central finite differences taken with
common random numbers (the Philox stream is keyed by seed and packet index, so the perturbed runs
reuse the same random numbers)."""
import numpy as np

import gradcase


def _run(mc_in, obj):
    from oracle import orc
    return orc.oracle_mc_grad(mc_in, nthreads=0, **obj)


def test_oracle_grad_values_restate_forward_tallies(oracle_lib):
    mc_in, obj = gradcase.case(n=20, nPhotons=1e4)
    n = mc_in["nx"]
    obj = dict(obj, nRadialBins=64, radialBinWidth=0.5 * np.sqrt(0.5) / 60)
    out, g = _run(mc_in, obj)
    b = obj["box"]
    F = np.asarray(out["NFR"], dtype=np.float64)[b[0]:b[1], b[2]:b[3], b[4]:b[5]].mean()
    assert abs(g["F"] - F) <= 1e-6 * abs(F)
    w = obj["radialBinWidth"]
    area = np.pi * w * w * (2 * np.arange(64) + 1)
    Rtot = float((g["R"] * area).sum())
    NI = float(np.asarray(out["NI_zneg"], dtype=np.float64).sum()) * mc_in["dx"] * mc_in["dy"]
    assert abs(Rtot - NI) <= 1e-6 * NI
    assert n == 20


def test_oracle_grad_matches_crn_finite_differences(oracle_lib):
    diffs = []
    for seed in range(1, 6):
        mc_in, obj = gradcase.case(n=16, nPhotons=8e3, seed=seed)
        mc_in["seed"] = seed
        diffs.append(gradcase.fd_differences(_run, mc_in, obj))
    bad = gradcase.zero_mean_test(diffs)
    assert not bad, bad
