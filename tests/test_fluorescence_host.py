"""Fluorescence MC host side (runMonteCarlo.m:119-166 and the simType 2 checks at :263-274):
the source built from the excitation results, the FMC property tree the MEX reads, and the
reference MEX run as simType 2 against the oracle on the same inputs."""
import math

import numpy as np
import pytest

import mccases
import mcstats
from mcmatlab_b200 import mexargs, prep
from mcmatlab_b200 import model as mm


def _media():
    return [mm.mediumProperties(name="a", mua=1.0, mus=10.0, g=0.9),
            mm.mediumProperties(name="b", mua=2.0, mus=10.0, g=0.9, QY=0.3, ES=lambda wl: 1.0 / wl),
            mm.mediumProperties(name="c", mua=3.0, mus=10.0, g=0.9,
                                QY=lambda wl, FR, T, FD: 0.05 * T / 37.0 + 0.01 * FR - 0.02 * FD,
                                ES=lambda wl, FR, T, FD: (wl / 500.0) ** 2 * (1 + 0 * T)),
            mm.mediumProperties(name="unused", mua=1.0, mus=1.0, g=0.0, QY=1.0)]


def test_source_matches_voxel_by_voxel_restatement():
    rng = np.random.default_rng(3)
    shape = (5, 4, 3)
    M = rng.integers(1, 4, size=shape).astype(np.float64)
    Ls_E = np.array([450.0, 480.0])
    Ls_F = np.array([520.0, 600.0, 700.0])
    NA = rng.uniform(0, 2, size=shape + (2,)).astype(np.float32).astype(np.float64)
    FR = rng.uniform(0, 3, size=shape).astype(np.float32)
    T = rng.uniform(30, 60, size=shape).astype(np.float32)
    FD = rng.uniform(0, 0.5, size=shape).astype(np.float32)
    media = _media()
    S = prep.fluorescence_source(media, M, NA, Ls_E, Ls_F, FR, T, FD)
    assert S.shape == shape + (3,) and S.dtype == np.float32 and S.flags["F_CONTIGUOUS"]
    for v in np.ndindex(shape):
        med = media[int(M[v]) - 1]

        def ev(f, wl):
            if not callable(f):
                return float(f)
            try:
                return float(f(wl))
            except TypeError:
                return float(f(wl, FR[v], T[v], FD[v]))
        fph = sum(NA[v + (e,)] * ev(med.QY, Ls_E[e]) * Ls_E[e] for e in range(2))
        es = np.array([ev(med.ES, w) for w in Ls_F])
        want = fph * es / es.sum() / Ls_F
        np.testing.assert_allclose(S[v], want.astype(np.float32), rtol=2e-6, atol=0)
    # emitted photons per voxel = sum_F S * lambda_F (the spectrum splits them, 1/lambda_F scales power)
    assert np.all(S[M == 1] == 0)


def test_source_errors():
    shape = (3, 3, 3)
    M = np.ones(shape)
    NA = np.ones(shape + (1,))
    with pytest.raises(ValueError, match="No fluorescence emitters"):
        prep.fluorescence_source(_media(), M, NA, [450.0], [600.0], 0.0, 37.0, 0.0)
    bad = [mm.mediumProperties(name="x", mua=1.0, mus=1.0, g=0.0, QY=-1.0)]
    with pytest.raises(ValueError, match="quantum yield"):
        prep.fluorescence_source(bad, M, NA, [450.0], [600.0], 0.0, 37.0, 0.0)
    with pytest.raises(ValueError, match="normalizedAbsorption"):
        prep.fluorescence_source(_media(), M, np.ones(shape + (2,)), [450.0], [600.0], 0.0, 37.0, 0.0)


def test_prepare_fluorescence_reads_fmc_and_checks_the_excitation():
    m = mccases.fluorescence_excited()
    mc_in = mexargs.prepare_mc(m, 2)
    assert mc_in["simType"] == 2
    np.testing.assert_array_equal(mc_in["wavelength"], [550.0, 650.0])
    sd = mc_in["sourceDistribution"]
    assert sd.shape == (24, 24, 24, 2)
    assert m.FMC.sourceDistribution is not None and np.array_equal(m.FMC.sourceDistribution, sd)
    # the fluorescence source keeps its scale (MCmatlab.c:626-629 takes each wavelength's power
    # from its integral); only the excitation source is normalised (runMonteCarlo.m:65)
    top = np.asarray(mc_in["M"]) == 1
    assert float(sd.sum()) > 0 and np.all(sd[top] == 0)
    tree = mexargs.mex_model_tree(mc_in)
    assert tree["FMC"] and not tree["MC"]
    assert tree["FMC"]["sourceDistribution"] is sd
    m2 = mccases.fluorescence_excited()
    m2.MC.normalizedFluenceRate = 0
    with pytest.raises(ValueError, match="normalizedFluenceRate"):
        mexargs.prepare_mc(m2, 2)
    m3 = mccases.fluorescence_excited()
    m3.MC.depositionCriteria.minScatterings = 1
    with pytest.raises(ValueError, match="restrictive deposition criteria"):
        mexargs.prepare_mc(m3, 2)


def test_reference_fluorescence_run_matches_oracle(ref_available, oracle_lib):
    """The reference MEX run as simType 2 (it reads the FMC node) against the FP64 oracle on the
    same fluorescence inputs; 8 batches each."""
    if not ref_available:
        pytest.skip("reference build absent")
    from oracle import orc, ref
    mc_in = mexargs.prepare_mc(mccases.fluorescence_excited(), 2)
    tree = mexargs.mex_model_tree(mc_in)
    R = ref.RefMC()
    a = [mcstats.summaries(R.run(tree, seed=301 + s), mc_in) for s in range(8)]
    b = []
    for s in range(8):
        mc_in["seed"] = 31 + s
        b.append(mcstats.summaries(orc.oracle_mc(mc_in, 0), mc_in))
    ok, rep, _ = mcstats.ztest(a, b)
    assert ok, rep
    assert not math.isnan(a[0]["abs_m1_l0"])
