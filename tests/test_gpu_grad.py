"""Perturbation-MC gradients on the GPU (mcb_mc_grad through the C ABI): against the FP64 oracle
running the same estimator on the same Philox streams, against central finite differences with
common random numbers, and the value outputs against the forward tallies of the same call."""
import numpy as np
import pytest

import gradcase
import mcstats

pytestmark = pytest.mark.gpu


def _gpu(mc_in, obj):
    from mcmatlab_b200 import native
    return native.mc_grad(mc_in, **obj)


def test_gpu_grad_values_restate_forward_tallies():
    mc_in, obj = gradcase.case(n=48, nPhotons=2e5)
    obj = dict(obj, nRadialBins=64, radialBinWidth=0.5 * np.sqrt(0.5) / 60)
    out, g = _gpu(mc_in, obj)
    b = obj["box"]
    F = np.asarray(out["NFR"], dtype=np.float64)[b[0]:b[1], b[2]:b[3], b[4]:b[5]].mean()
    assert abs(g["F"] - F) <= 1e-4 * abs(F)
    w = obj["radialBinWidth"]
    Rtot = float((g["R"] * np.pi * w * w * (2 * np.arange(64) + 1)).sum())
    NI = float(np.asarray(out["NI_zneg"], dtype=np.float64).sum()) * mc_in["dx"] * mc_in["dy"]
    assert abs(Rtot - NI) <= 1e-5 * NI


def test_gpu_grad_matches_oracle_same_streams(oracle_lib):
    from oracle import orc
    ga, gb = [], []
    for seed in range(1, 9):
        mc_in, obj = gradcase.case(n=24, nPhotons=2e4, seed=seed)
        ga.append(gradcase.summary(orc.oracle_mc_grad(mc_in, nthreads=0, **obj)[1]))
        gb.append(gradcase.summary(_gpu(mc_in, obj)[1]))
    ok, rep, worst = mcstats.ztest(ga, gb)
    assert ok, rep


def test_gpu_grad_matches_crn_finite_differences():
    diffs = []
    for seed in range(1, 9):
        mc_in, obj = gradcase.case(n=32, nPhotons=2e5, seed=seed)
        diffs.append(gradcase.fd_differences(_gpu, mc_in, obj))
    bad = gradcase.zero_mean_test(diffs)
    assert not bad, bad


def test_gpu_grad_forward_outputs_match_plain_run():
    """The gradient kernel's forward tallies are the plain kernel's (same streams, same steps)."""
    from mcmatlab_b200 import native
    mc_in, obj = gradcase.case(n=32, nPhotons=5e4)
    a = native.mc_run(mc_in)
    b, _ = _gpu(mc_in, obj)
    assert a["nPhotons"] == b["nPhotons"]
    np.testing.assert_allclose(b["NFR"], a["NFR"], rtol=1e-4, atol=1e-6 * float(np.max(a["NFR"])))


@pytest.mark.parametrize("bad", ["two_wavelengths", "too_many_media", "bins", "time_limit"])
def test_gpu_grad_rejects_unsupported_inputs(bad):
    from mcmatlab_b200 import native
    mc_in, obj = gradcase.case(n=16, nPhotons=1e3)
    if bad == "two_wavelengths":
        for k in ("mua", "mus", "g", "n", "CDFidx"):
            mc_in[k] = np.repeat(np.asarray(mc_in[k]), 2, axis=1)
        mc_in["spectrum"] = np.array([0.5, 0.5])
    elif bad == "too_many_media":
        for k in ("mua", "mus", "g", "n", "CDFidx"):
            mc_in[k] = np.repeat(np.asarray(mc_in[k]), 2, axis=0)
    elif bad == "bins":
        obj["nRadialBins"] = 65
    else:
        mc_in["nPhotonsRequested"] = float("nan")
        mc_in["simulationTimeRequested"] = 0.01
    with pytest.raises(native.MCBError):
        _gpu(mc_in, obj)
