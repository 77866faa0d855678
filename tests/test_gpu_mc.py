"""GPU transport parity: the CUDA kernel through the C ABI against the reference's own
batches (golden) and against the FP64 CPU oracle on the same Philox streams."""
import json
import os

import numpy as np
import pytest

import mccases
import mcstats
from mcmatlab_b200 import mexargs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
K = 8


def gpu_batches(mc_in, K=K, first_seed=1):
    from mcmatlab_b200 import native
    out = []
    for s in range(K):
        mc_in["seed"] = first_seed + s
        out.append(mcstats.summaries(native.mc_run(mc_in), mc_in))
    return out


@pytest.mark.parametrize("name", sorted(mccases.CASES))
def test_gpu_matches_reference_golden(name):
    with open(os.path.join(GOLD, "mc_ref_summaries.json")) as f:
        golden = json.load(f)[name]
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    ok, rep, worst = mcstats.ztest(golden, gpu_batches(mc_in))
    assert ok, rep


@pytest.mark.parametrize("name", ["c0_small", "radial_lens_ff", "xy_custom_fiber_cyclic", "dc_end_of_life"])
def test_gpu_matches_oracle_same_streams(name, oracle_lib):
    from oracle import orc
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    ob = []
    for s in range(K):
        mc_in["seed"] = 1 + s
        ob.append(mcstats.summaries(orc.oracle_mc(mc_in, 0), mc_in))
    ok, rep, worst = mcstats.ztest(ob, gpu_batches(mc_in))
    assert ok, rep


def test_gpu_deterministic_counters():
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    a = native.mc_run(mc_in)
    b = native.mc_run(mc_in)
    assert a["propagationSteps"] == b["propagationSteps"] and a["nPhotons"] == b["nPhotons"]
    np.testing.assert_allclose(a["NFR"], b["NFR"], rtol=1e-9, atol=1e-12 * float(np.max(a["NFR"])))


def test_gpu_energy_balance_c0():
    """Absorbed + escaped weight = launched weight up to roulette noise (standard tissue cube)."""
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    mc_in["nPhotonsRequested"] = 2e5
    o = native.mc_run(mc_in)
    s = mcstats.summaries(o, mc_in)
    absorbed = sum(v for k, v in s.items() if k.startswith("abs_m"))
    escaped = sum(v for k, v in s.items() if k.startswith("NI_"))
    assert abs(absorbed + escaped - 1.0) < 0.01, (absorbed, escaped)


def test_gpu_requested_collected_and_timed_modes():
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.xy_custom_fiber_cyclic())
    mc_in["requestCollectedPhotons"] = True
    mc_in["nPhotonsRequested"] = 500.0
    o = native.mc_run(mc_in)
    assert o["nPhotonsCollected"] >= 500 and o["nPhotons"] > o["nPhotonsCollected"]
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    mc_in["nPhotonsRequested"] = float("nan")
    mc_in["simulationTimeRequested"] = 0.5 / 60  # half a second
    o = native.mc_run(mc_in)
    assert o["nPhotons"] > 1000 and 0.3 / 60 < o["simulationTime"] < 5.0 / 60


def test_gpu_example_paths():
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    mc_in["nExamplePaths"] = 5
    o = native.mc_run(mc_in)
    P = o["examplePaths"]
    assert P.shape[0] == 4 and P.shape[1] > 10
    starts = np.sum(np.isnan(P[0, :-1]) & np.isnan(P[0, 1:]))
    assert starts == 5


def split_paths(P):
    """Example-path columns -> list of paths (each [4, n], NaN columns kept), split at the two
    NaN columns that open every path (MCmatlablib.c:479-504)."""
    nan = np.isnan(P[0])
    starts = [k for k in range(P.shape[1] - 1) if nan[k] and nan[k + 1] and (k == 0 or not nan[k - 1])]
    return [P[:, a:b] for a, b in zip(starts, starts[1:] + [P.shape[1]])]


def paths_agree(a, b, rtol=1e-4, atol=1e-5):
    if a.shape != b.shape or not np.array_equal(np.isnan(a), np.isnan(b)):
        return False
    f = ~np.isnan(a)
    return bool(np.all(np.abs(a[f] - b[f]) <= atol + rtol * np.abs(b[f])))


@pytest.mark.parametrize("name", ["c0_small", "xy_custom_fiber_cyclic", "dc_end_of_life", "iso_point_bt0"])
def test_gpu_example_paths_match_oracle_replay(name, oracle_lib):
    """Example paths (packets 0, 1, 2, ... replayed and recorded as the reference's master thread
    records its packets, MCmatlablib.c:465-514, MCmatlab.c:270-278) against the FP64 oracle's
    replay of the same Philox streams: vertex by vertex (positions to 1e-5 cm + 1e-4 relative,
    weights to 1e-4 relative), with the NaN separators of cyclic wraps and the deletion of paths
    whose end-of-life criteria fail. FP32 rounding may send a rare packet the other way at a
    decision; at least 9 of the 10 paths must agree in full."""
    from mcmatlab_b200 import native
    from oracle import orc
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    mc_in["nExamplePaths"] = 10
    g = split_paths(native.mc_run(mc_in)["examplePaths"])
    o = split_paths(orc.oracle_mc(mc_in, 0)["examplePaths"])
    assert len(o) == 10 and len(g) == 10
    same = [paths_agree(x, y) for x, y in zip(g, o)]
    print(name, "paths agreeing with the oracle:", sum(same), "of", len(same), [x.shape[1] for x in g])
    assert sum(same) >= 9, same


@pytest.mark.parametrize("name", sorted(mccases.CASES))
def test_gpu_free_step_cut_weight_is_negligible(name):
    """The transport ends a packet after 2e4 sub-steps without scattering (the reference has no
    such limit). On every golden case the weight those packets still carried is below 1e-6 of
    the launched weight, far below the cases' statistical errors."""
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    o = native.mc_run(mc_in)
    assert o["freeStepCuts"] >= 0 and o["freeStepCutWeight"] >= 0
    assert o["freeStepCutWeight"] <= 1e-6 * o["nPhotons"], (o["freeStepCuts"], o["freeStepCutWeight"], o["nPhotons"])


def test_gpu_tallies_normalise_to_the_run_outputs():
    """mcb_mc_normalize on a run's own FP64 tallies reproduces its outputs bit for bit."""
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.radial_lens_ff())
    o = native.mc_run(mc_in, tallies=True)
    n = native.mc_normalize(mc_in, o["tallies"])
    assert n["nPhotons"] == o["nPhotons"] and n["nPhotonsCollected"] == o["nPhotonsCollected"]
    for k in ("NFR", "image", "farField", "NI_zneg", "NI_xpos"):
        if k in o:
            assert np.array_equal(n[k], o[k]), k


@pytest.mark.parametrize("name", ["c0_small", "radial_lens_ff", "broadband"])
def test_gpu_resume_from_tallies_equals_one_long_run(name):
    """MC checkpoint/resume: a run of N packets continued by a run of the next N packets of the
    same streams (packetOffset = N per wavelength), merged from their FP64 tallies, equals one run of 2N packets
    up to FP64 summation order (the outputs are single precision)."""
    from mcmatlab_b200 import combine, native
    mc_in = mexargs.prepare_mc(mccases.CASES[name]())
    N = float(mc_in["nPhotonsRequested"])
    nL = np.asarray(mc_in["mua"]).shape[1]
    assert N % nL == 0
    a = native.mc_run(mc_in, tallies=True)
    # packet indices count per wavelength (each wavelength has its own streams)
    b = native.mc_run(dict(mc_in, packetOffset=int(N) // nL), tallies=True)
    m = combine.merge_tallies(mc_in, [a, b])
    full = native.mc_run(dict(mc_in, nPhotonsRequested=2 * N))
    assert m["nPhotons"] == full["nPhotons"] == a["nPhotons"] + b["nPhotons"]
    for k in ("NFR", "image", "farField", "NI_zneg", "NI_zpos", "NI_xpos"):
        if k in full and np.size(full[k]) > 1:
            x, y = np.asarray(m[k], np.float64), np.asarray(full[k], np.float64)
            np.testing.assert_allclose(x, y, rtol=2e-6, atol=2e-6 * float(np.max(np.abs(y))), err_msg=k)
