"""Pins the CPU oracle to the reference: known-answer vectors, golden reference outputs
and, where the reference build is present, live reference runs."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import heatcases
import mccases
import mcstats
from mcmatlab_b200 import abi, mexargs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
K = 8


def test_struct_layout_matches_header(oracle_lib):
    assert oracle_lib.orc_sizeof_mc_model() == C.sizeof(abi.mcb_mc_model)
    assert oracle_lib.orc_sizeof_mc_result() == C.sizeof(abi.mcb_mc_result)
    assert oracle_lib.orc_sizeof_heat_params() == C.sizeof(abi.mcb_heat_params)


def test_philox_known_answers(oracle_lib):
    # Philox-4x32-10 known-answer vectors published with Random123 (Salmon et al., SC'11)
    from oracle import orc
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_lambert_wm1(oracle_lib):
    from scipy.special import lambertw
    xs = -np.exp(-1.0) * np.concatenate([np.linspace(1e-9, 0.9999, 2001), [1e-12, 0.99999999]])
    for x in xs:
        assert abs(oracle_lib.orc_lambert_wm1(float(x)) - lambertw(x, -1).real) <= 1e-8 * abs(lambertw(x, -1).real)
    assert abs(oracle_lib.orc_lambert_wm1(-np.exp(-1.0)) + 1.0) < 1e-6  # branch point


@pytest.mark.parametrize("name", sorted(mccases.CASES))
def test_mc_oracle_matches_reference_golden(name, oracle_lib):
    """Oracle batches vs the committed reference batches: every summary within 4.5 combined SE.
    The packets the free-step limit ended (the reference has no such limit) carried less than
    1e-6 of the launched weight."""
    from oracle import orc
    with open(os.path.join(GOLD, "mc_ref_summaries.json")) as f:
        golden = json.load(f)[name]
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    ob = []
    for s in range(K):
        mc_in["seed"] = 1 + s
        out = orc.oracle_mc(mc_in, 0)
        assert out["freeStepCutWeight"] <= 1e-6 * out["nPhotons"], (out["freeStepCuts"], out["freeStepCutWeight"])
        ob.append(mcstats.summaries(out, mc_in))
    ok, rep, worst = mcstats.ztest(golden, ob)
    assert ok, rep


@pytest.mark.parametrize("name", sorted(mccases.FLUO_CASES))
def test_fluorescence_oracle_matches_reference_golden(name, oracle_lib):
    """Fluorescence runs (the reference MEX as simType 2): oracle batches vs the committed ones."""
    from oracle import orc
    with open(os.path.join(GOLD, "mc_ref_summaries.json")) as f:
        golden = json.load(f)[name]
    mc_in = mexargs.prepare_mc(mccases.FLUO_CASES[name](), 2)
    ob = [mcstats.summaries(orc.oracle_mc(dict(mc_in, seed=1 + s), 0), mc_in) for s in range(K)]
    ok, rep, worst = mcstats.ztest(golden, ob)
    assert ok, rep


def test_mc_oracle_deterministic(oracle_lib):
    from oracle import orc
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    a = orc.oracle_mc(mc_in, 1)
    b = orc.oracle_mc(mc_in, 1)
    assert np.array_equal(a["NFR"], b["NFR"]) and a["propagationSteps"] == b["propagationSteps"]
    c = orc.oracle_mc(mc_in, 4)
    assert c["propagationSteps"] == a["propagationSteps"]
    np.testing.assert_allclose(c["NFR"], a["NFR"], rtol=1e-5, atol=1e-6 * float(a["NFR"].max()))


def test_mc_golden_fixture_matches_live_reference(ref_available):
    """The committed reference batches agree with fresh reference runs (other seeds)."""
    if not ref_available:
        pytest.skip("reference build not present")
    from oracle import ref
    with open(os.path.join(GOLD, "mc_ref_summaries.json")) as f:
        golden = json.load(f)
    R = ref.RefMC()
    for name in ("c0_small", "xy_custom_fiber_cyclic"):
        mc_in = mexargs.prepare_mc(mccases.CASES[name]())
        tree = mexargs.mex_model_tree(mc_in)
        live = [mcstats.summaries(R.run(tree, seed=501 + s), mc_in) for s in range(K)]
        ok, rep, _ = mcstats.ztest(golden[name], live)
        assert ok, rep


@pytest.mark.parametrize("name", sorted(heatcases.CASES))
def test_heat_oracle_vs_reference_fp32(name, oracle_lib):
    """FP64 oracle vs the reference's FP32 stepper (golden). The gap is the reference's own
    FP32 rounding: bounded by 1e-6 relative per step (about 4 float ulps at 37 degC per step)."""
    from oracle import orc
    gold = np.load(os.path.join(GOLD, "heat_ref.npz"))
    case = heatcases.CASES[name]()
    nx, ny, nz = case["n"]
    nt = int(case["hp"]["steps"])
    T, Om, S, Mx = orc.oracle_heat(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    Tr = gold[name + "_T"]
    rel = np.max(np.abs(T - Tr) / np.abs(T))
    assert rel <= 1e-6 * nt + 1e-6, rel
    np.testing.assert_allclose(gold[name + "_sensorTemps"], S, rtol=1e-6 * nt + 1e-6)
    np.testing.assert_allclose(gold[name + "_maxMediaTemps"].ravel(), Mx, rtol=1e-6 * nt + 1e-6)
    if case["Omega0"] is not None:
        Or = gold[name + "_Omega"]
        # dOmega/Omega ~ E/(R T^2) dT amplifies the FP32 temperature error (~0.6/K near 37 degC)
        # and each FP32 accumulation step rounds Omega by up to half an ulp
        scale = np.max(np.abs(Om - case["Omega0"]))
        tol = 1e-3 * scale + (nt + 1) * np.finfo(np.float32).eps * np.abs(Om) + 1e-30
        assert np.all(np.abs(Om - Or) <= tol)


def test_heat_oracle_conserves_energy_insulated(oracle_lib):
    """No source, insulated faces: sum(VHC * T) is conserved; uniform T stays uniform."""
    from oracle import orc
    case = heatcases.insulated_on()
    hp = dict(case["hp"])
    hp["lightsOn"] = False
    nx, ny, nz = case["n"]
    from mcmatlab_b200 import configs, prep
    m = configs.standard_tissue_cube(n=nx, nPhotons=1)
    th = prep.thermal_media_properties(m.G.mediaPropertiesFunc([]), m.G.M_raw)
    vhc = th["VHC"][th["M"].astype(int) - 1]
    T, _, _, _ = orc.oracle_heat(case["T0"], None, hp, nx, ny, nz)
    e0 = np.sum(vhc * case["T0"].astype(np.float64))
    assert abs(np.sum(vhc * T) - e0) <= 1e-9 * abs(e0)
    U = np.full((nx, ny, nz), 41.5, np.float32)
    T, _, _, _ = orc.oracle_heat(U, None, hp, nx, ny, nz)
    assert np.max(np.abs(T - 41.5)) < 1e-10
