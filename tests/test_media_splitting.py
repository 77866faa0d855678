"""Fluence-rate / temperature / damage dependent media (getOpticalMediaProperties.m:57-203 with
geometry.m:64-101): dependence flags, splitting into nBins sub-media through the sub-media binning
(here the oracle's restatement, pinned to the reference build), means per bin for later
wavelengths, and the fluence-rate iterations' photon schedule."""
import numpy as np
import pytest

from mcmatlab_b200 import prep
from mcmatlab_b200 import model as mm
from mcmatlab_b200.model import depositionCriteria


def _oracle_ds(oracle_lib):
    from oracle import orc
    return orc.oracle_downsample


def _media():
    return [mm.mediumProperties(name="plain", mua=1.0, mus=50.0, g=0.9, n=1.0, nBins=3),
            mm.mediumProperties(name="absorber", mua=lambda wl, FR, T, FD: 10.0 / (1.0 + FR / 100.0) * (500.0 / wl),
                                mus=lambda wl, FR, T, FD: 80.0 + 0.1 * T, g=0.8, n=1.0, nBins=6)]


def test_dependence_flags():
    FRd, Td, FDd = prep.dependence_flags(_media())
    assert not FRd[0].any() and not Td[0].any() and not FDd[0].any()
    assert FRd[1, 0] and not Td[1, 0] and not FDd[1, 0]   # mua: fluence rate only
    assert Td[1, 1] and not FRd[1, 1] and not FDd[1, 1]   # mus: temperature only
    assert not FRd[1, 2] and not Td[1, 2]                 # g constant


def test_split_media_bins_and_tables(oracle_lib):
    ds = _oracle_ds(oracle_lib)
    rng = np.random.default_rng(2)
    shape = (10, 8, 6)
    M_raw = np.ones(shape)
    M_raw[:, :, 2:] = 2
    FR = rng.uniform(0, 400, shape).astype(np.float32)
    T = rng.uniform(30, 50, shape).astype(np.float32)
    wl = np.array([500.0, 600.0])
    mp = prep.optical_media_properties(_media(), M_raw, wl, True, 0.1, 0.1, 0.1, depositionCriteria(),
                                       FR=FR, T=T, FD=0.0, downsample=ds)
    M = mp["M"]
    assert mp["mua"].shape == (9, 2)
    # the plain medium: three identical rows, every voxel in the first
    assert np.all(M[M_raw == 1] == 1)
    np.testing.assert_array_equal(mp["mua"][:3], 1.0)
    # the absorber: voxels in sub-media 4..9, rows sorted by (mua, mus), binned on wavelength 1
    sub = M[M_raw == 2].astype(int)
    assert sub.min() >= 4 and sub.max() <= 9
    mua1 = mp["mua"][3:, 0]
    assert np.all(np.diff(mua1) >= 0)
    idx = np.nonzero((M_raw == 2).reshape(-1, order="F"))[0]
    FRv = FR.reshape(-1, order="F")[idx]
    Tv = T.reshape(-1, order="F")[idx]
    par = np.stack([10.0 / (1.0 + FRv / 100.0) * (500.0 / 500.0), 80.0 + 0.1 * Tv,
                    np.full(idx.size, 0.8, np.float32)]).astype(np.float32)
    reps, lab = ds(par, 6)
    order = np.lexsort((reps[2], reps[1], reps[0]))
    np.testing.assert_array_equal(mp["mua"][3:, 0], reps[0, order].astype(np.float64))
    np.testing.assert_array_equal(mp["mus"][3:, 0], reps[1, order].astype(np.float64))
    # wavelength 2: the mean of the new values over each bin
    mua2 = (10.0 / (1.0 + FRv / 100.0) * (500.0 / 600.0)).astype(np.float32)
    Mv = M.reshape(-1, order="F")[idx].astype(int)
    for k in range(6):
        sel = Mv == 4 + k
        if sel.any():
            assert mp["mua"][3 + k, 1] == pytest.approx(float(np.mean(mua2[sel].astype(np.float64))), rel=1e-12)


def test_split_needs_the_binning():
    shape = (4, 4, 4)
    M_raw = np.full(shape, 2.0)
    with pytest.raises(ValueError, match="sub-media binning"):
        prep.optical_media_properties(_media(), M_raw, [500.0], True, 0.1, 0.1, 0.1, depositionCriteria(),
                                      FR=np.ones(shape, np.float32), T=37.0)
    too_many = [mm.mediumProperties(name="a%d" % i, mua=1.0, mus=1.0, g=0.0, nBins=200) for i in range(2)]
    with pytest.raises(ValueError, match="256"):
        prep.optical_media_properties(too_many, np.array([[[1, 2]]], dtype=float), [500.0], True, 0.1, 0.1, 0.1,
                                      depositionCriteria())


def test_thermal_splitting_and_flags(oracle_lib):
    ds = _oracle_ds(oracle_lib)
    media = [mm.mediumProperties(name="fixed", VHC=3.9, TC=0.0037, nBins=2),
             mm.mediumProperties(name="soft", VHC=lambda T, FD: 3.9 * (1 + 0.002 * (T - 37.0)), TC=0.0037, nBins=5,
                                 A=1e10, E=1e5)]
    thmT, thmFD = prep.thermal_dependence_flags(media)
    # geometry.m tests the first grid axis (fluence rate) for T and the second (temperature) for FD
    assert not thmT.any() and thmFD[1, 0] and not thmFD[1, 1] and not thmFD[0].any()
    rng = np.random.default_rng(4)
    shape = (6, 6, 6)
    M_raw = np.ones(shape)
    M_raw[:, :, 3:] = 2
    T = rng.uniform(37, 80, shape).astype(np.float32)
    th = prep.thermal_media_properties(media, M_raw, T, 0.0, downsample=ds)
    assert th["VHC"].shape == (7,) and np.all(th["VHC"][:2] == np.float32(3.9))
    assert np.all(th["M"][M_raw == 1] == 1)
    sub = th["M"][M_raw == 2].astype(int)
    assert sub.min() >= 3 and sub.max() <= 7 and np.all(np.diff(th["VHC"][2:]) >= 0)
    np.testing.assert_array_equal(th["A"], [0, 0, 1e10, 1e10, 1e10, 1e10, 1e10])
    idx = np.nonzero((M_raw == 2).reshape(-1, order="F"))[0]
    Tv = T.reshape(-1, order="F")[idx]
    par = np.stack([3.9 * (1 + 0.002 * (Tv - 37.0)), np.full(idx.size, 0.0037, np.float32),
                    np.ones(idx.size, np.float32)]).astype(np.float32)
    reps, lab = ds(par, 5)
    order = np.lexsort((reps[2], reps[1], reps[0]))
    np.testing.assert_array_equal(th["VHC"][2:], reps[0, order].astype(np.float64))
    with pytest.raises(ValueError, match="sub-media binning"):
        prep.thermal_media_properties(media, M_raw, T, 0.0)


def test_scalar_property_functions_apply_elementwise(oracle_lib):
    """A property function written for scalars (math module, `if`) is applied voxel by voxel."""
    import math
    ds = _oracle_ds(oracle_lib)
    med = [mm.mediumProperties(name="s", mua=lambda wl, FR, T, FD: 1.0 + 9.0 * math.exp(-FR / 50.0),
                               mus=10.0, g=0.9, n=1.0, nBins=4,
                               VHC=lambda T, FD: 3.9 + (0.5 if T > 50 else 0.0), TC=0.0037)]
    FRd, _, _ = prep.dependence_flags(med)
    assert FRd[0, 0]
    shape = (5, 5, 5)
    FR = np.linspace(0, 300, 125, dtype=np.float32).reshape(shape)
    mp = prep.optical_media_properties(med, np.ones(shape), [500.0], True, 0.1, 0.1, 0.1, depositionCriteria(),
                                       FR=FR, T=37.0, downsample=ds)
    assert np.unique(mp["M"]).size == 4 and mp["mua"][:, 0].max() <= 10.0
    T = np.where(np.arange(125).reshape(shape) % 2 == 0, 40.0, 60.0).astype(np.float32)
    th = prep.thermal_media_properties(med, np.ones(shape), T, 0.0, downsample=ds)
    assert set(np.round(th["VHC"], 3)) == {3.9, 4.4}


def test_max_media_temps_fold_per_unsplit_medium(oracle_lib):
    """maxMediaTemps keeps one entry per unsplit medium: the stepper's per-sub-medium maxima are
    folded over each medium's nBins sub-media (simulateHeatDistribution.m:268-272), and the first
    run starts from the maxima over the raw medium index (:38-47)."""
    from mcmatlab_b200 import heatsim
    rng = np.random.default_rng(4)
    shape = (6, 5, 4)
    M_raw = np.ones(shape)
    M_raw[:, :, 2:] = 2
    T = rng.uniform(30, 50, shape).astype(np.float32)
    th_media = [mm.mediumProperties(name="a", VHC=3.9, TC=0.0037, nBins=3),
                mm.mediumProperties(name="b", VHC=lambda T, FD: 3.0 + 0.01 * T, TC=0.005, nBins=4)]
    th = prep.thermal_media_properties(th_media, M_raw, T, 0.0, downsample=_oracle_ds(oracle_lib))
    assert th["nBins"] == [3, 4] and len(th["VHC"]) == 7
    maxT = heatsim.initial_max_media_temps(T, M_raw, len(th["nBins"]))
    assert maxT.shape == (2,)
    assert maxT[0] == T[M_raw == 1].max() and maxT[1] == T[M_raw == 2].max()
    new = np.array([10.0, 60.0, 20.0, 1.0, 2.0, 70.0, 3.0], dtype=np.float32)
    heatsim.fold_max_media_temps(maxT, new, th["nBins"])
    assert maxT[0] == 60.0 and maxT[1] == 70.0
    low = np.zeros(7, dtype=np.float32)
    heatsim.fold_max_media_temps(maxT, low, th["nBins"])
    assert maxT[0] == 60.0 and maxT[1] == 70.0
