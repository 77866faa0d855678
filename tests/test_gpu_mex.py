"""The MEX gateways (mcmatlab_b200/mex/*.c), driven through the mx shim exactly as the
reference MEX is, against the reference's golden outputs."""
import json
import os
import subprocess

import numpy as np
import pytest

import heatcases
import mccases
import mcstats
from mcmatlab_b200 import mexargs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def gateways():
    from mcmatlab_b200 import build
    build.build()
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "mexgw"], check=True, capture_output=True)
    from oracle import ref
    return ref.RefMC("libmex_mc_cuda.so"), ref.RefHeat("libmex_heat_cuda.so")


@pytest.mark.parametrize("name", ["c0_small", "radial_lens_ff", "xy_custom_fiber_cyclic", "broadband"])
def test_mc_gateway_matches_reference(name, gateways):
    gw, _ = gateways
    with open(os.path.join(GOLD, "mc_ref_summaries.json")) as f:
        golden = json.load(f)[name]
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    batches = []
    for s in range(8):
        tree = mexargs.mex_model_tree(dict(mc_in, seed=11 + s))
        out = gw.run(tree)
        batches.append(mcstats.summaries(out, mc_in))
    ok, rep, _ = mcstats.ztest(golden, batches)
    assert ok, rep


def test_binning_gateway_matches_reference_build(gateways):
    """getDownsampledParamVals through the gateway (device binning) against the reference MEX's
    own outputs: bit for bit."""
    import dscases
    from oracle import ref
    gw = ref.RefDownsample("libmex_ds_cuda.so")
    cases = dscases.cases(count=24, seed=3)
    if ref_build_present():
        R = ref.RefDownsample()
        for par, nb in cases:
            a, b = R.run(par, nb), gw.run(par, nb)
            np.testing.assert_array_equal(b[0], a[0])
            np.testing.assert_array_equal(b[1], a[1])
    else:
        from oracle import orc
        for par, nb in cases:
            a, b = orc.oracle_downsample(par, nb), gw.run(par, nb)
            np.testing.assert_array_equal(b[0], a[0])
            np.testing.assert_array_equal(b[1].reshape(-1), a[1])


def ref_build_present():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_downsample.so"))


def test_heat_gateway_matches_reference(gateways):
    _, gw = gateways
    gold = np.load(os.path.join(GOLD, "heat_ref.npz"))
    case = heatcases.insulated_on()
    T, Om, S, Mx = gw.run(case["T0"], case["Omega0"], case["hp"])
    nt = int(case["hp"]["steps"])
    assert np.max(np.abs(T - gold["insulated_on_T"]) / gold["insulated_on_T"]) <= 1e-6 * nt + 2e-6
    np.testing.assert_allclose(S, gold["insulated_on_sensorTemps"], rtol=1e-6 * nt + 2e-6)
    np.testing.assert_allclose(Mx.ravel(), gold["insulated_on_maxMediaTemps"].ravel(), rtol=1e-6 * nt + 2e-6)
    assert S.shape == (3, nt + 1) and Mx.shape == (1, 4)


def test_mc_gateway_ctrl_c_returns_partial_results(gateways):
    """With MATLAB's interrupt flag raised, the gateway stops the run and returns the packets
    that ran, normalised over them, without an error (the reference's Ctrl+C behaviour)."""
    import ctypes as C
    gw, _ = gateways
    flag = C.c_int.in_dll(gw.sh.lib, "mxshim_interrupt")
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    tree = mexargs.mex_model_tree(dict(mc_in, nPhotonsRequested=2e9, seed=3))
    flag.value = 1
    try:
        out = gw.run(tree)
    finally:
        flag.value = 0
    n = float(np.asarray(out["nPhotons"]).ravel()[0])
    assert 0 < n < 2e9
    assert np.all(np.isfinite(out["NFR"])) and float(np.max(out["NFR"])) > 0
    # the next call runs to completion
    out = gw.run(mexargs.mex_model_tree(dict(mc_in, seed=4)))
    assert float(np.asarray(out["nPhotons"]).ravel()[0]) == mc_in["nPhotonsRequested"]
