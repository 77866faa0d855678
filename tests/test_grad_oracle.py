"""Perturbation-MC estimator in the FP64 oracle: its value outputs restate MCmatlab's normalised
tallies of the same run, and its derivatives agree with central finite differences taken with
common random numbers (the Philox stream is keyed by seed and packet index, so the perturbed runs
reuse the same random numbers)."""
import numpy as np
import pytest

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


def test_oracle_grad_matches_reference_differences(oracle_lib, ref_available):
    """dF/dmua of the box fluence against central differences (1% step) of the reference's own MC
    (MCmatlab.c compiled from source, pinned seed, one thread). The reference's stream follows
    a mua change except through roulette, so its differences are nearly common-random-number
    ones; the per-seed differences (oracle estimate - reference difference) have zero mean."""
    if not ref_available:
        pytest.skip("reference build not present")
    from oracle import ref
    from mcmatlab_b200 import mexargs
    rm = ref.RefMC()
    diffs = []
    for seed in range(1, 7):
        mc_in, obj = gradcase.case(n=16, nPhotons=1.5e4, seed=seed)
        b = obj["box"]
        _, g = _run(mc_in, obj)

        def F(m):
            out = rm.run(mexargs.mex_model_tree(m), seed=seed)
            return float(np.asarray(out["NFR"], np.float64)[b[0]:b[1], b[2]:b[3], b[4]:b[5]].mean())
        d = {}
        for j in gradcase.MEDIA:
            step = 0.02 * float(np.asarray(mc_in["mua"])[j, 0])
            fd = (F(gradcase.perturbed(mc_in, "mua", j, 1.01)) - F(gradcase.perturbed(mc_in, "mua", j, 0.99))) / step
            d["F_mua%d" % j] = g["dF_dmua"][j] - fd
        diffs.append(d)
    bad = gradcase.zero_mean_test(diffs)
    assert not bad, bad
