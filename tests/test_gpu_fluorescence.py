"""Fluorescence MC on the GPU (simType 2: the run reads model.FMC and a source built from the
excitation results): against the reference MEX run as simType 2 (golden batches), against the
FP64 oracle on the same Philox streams, through the MEX gateway, and end to end through
runMonteCarlo(model) followed by runMonteCarlo(model, 'fluorescence')."""
import json
import os
import subprocess

import numpy as np
import pytest

import mccases
import mcstats
from mcmatlab_b200 import mexargs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
K = 8


def _gpu_batches(mc_in, first_seed=1):
    from mcmatlab_b200 import native
    out = []
    for s in range(K):
        out.append(mcstats.summaries(native.mc_run(dict(mc_in, seed=first_seed + s)), mc_in))
    return out


def test_gpu_fluorescence_matches_reference_golden():
    with open(os.path.join(GOLD, "mc_ref_summaries.json")) as f:
        golden = json.load(f)["fluorescence"]
    mc_in = mexargs.prepare_mc(mccases.fluorescence_excited(), 2)
    ok, rep, _ = mcstats.ztest(golden, _gpu_batches(mc_in))
    assert ok, rep


def test_gpu_fluorescence_matches_oracle_same_streams(oracle_lib):
    from oracle import orc
    mc_in = mexargs.prepare_mc(mccases.fluorescence_excited(), 2)
    ob = [mcstats.summaries(orc.oracle_mc(dict(mc_in, seed=1 + s), 0), mc_in) for s in range(K)]
    ok, rep, _ = mcstats.ztest(ob, _gpu_batches(mc_in))
    assert ok, rep


def test_mex_gateway_fluorescence_matches_reference():
    from mcmatlab_b200 import build
    build.build()
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "mexgw"], check=True, capture_output=True)
    from oracle import ref
    gw = ref.RefMC("libmex_mc_cuda.so")
    with open(os.path.join(GOLD, "mc_ref_summaries.json")) as f:
        golden = json.load(f)["fluorescence"]
    mc_in = mexargs.prepare_mc(mccases.fluorescence_excited(), 2)
    batches = [mcstats.summaries(gw.run(mexargs.mex_model_tree(dict(mc_in, seed=21 + s))), mc_in) for s in range(K)]
    ok, rep, _ = mcstats.ztest(golden, batches)
    assert ok, rep


def test_run_monte_carlo_then_fluorescence_end_to_end():
    """Excitation transport, then the fluorescence step from its results: outputs land in
    model.FMC, and per fluorescence wavelength absorbed + escaped equals P^2, P the source's
    integral, up to roulette noise: the reference normalises a distributed-source run by
    nPhotons / P (MCmatlab.c:752 passes P as the power fraction) and divides once more by P
    (MCmatlablib.c:1195-1198)."""
    m = mccases.fluorescence_excited(nph=1e5)
    m.MC.normalizedFluenceRate = 0
    m.MC.nPhotonsRequested = 1e5
    m.MC.lightSource.sourceType = 0
    m.runMonteCarlo()
    assert np.asarray(m.MC.NFR).shape == (24, 24, 24)
    m.runMonteCarlo("fluorescence")
    F = m.FMC
    NFR = np.asarray(F.NFR)
    assert NFR.shape == (24, 24, 24, 2) and np.all(np.isfinite(NFR)) and NFR.max() > 0
    assert np.asarray(F.farField).shape == (8, 8, 2)
    assert F.nPhotons == 1e5
    S = np.asarray(F.sourceDistribution, dtype=np.float64)
    dV = m.G.dx * m.G.dy * m.G.dz
    mc_in = {"dx": m.G.dx, "dy": m.G.dy, "dz": m.G.dz, "M": F.M, "mua": F.mediaProperties["mua"]}
    out = {"NFR": NFR}
    for face in ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg"):
        out["NI_" + face] = np.asarray(getattr(F, "normalizedIrradiance_" + face))
    s = mcstats.summaries(out, mc_in)
    for iL in range(2):
        P = S[..., iL].sum() * dV
        absorbed = sum(v for k, v in s.items() if k.startswith("abs_m") and k.endswith("_l%d" % iL))
        escaped = sum(v for k, v in s.items() if k.startswith("NI_") and k.endswith("_l%d" % iL))
        assert abs((absorbed + escaped) / P ** 2 - 1.0) < 0.02, (iL, absorbed, escaped, P)
