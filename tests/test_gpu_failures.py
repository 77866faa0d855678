"""Failure paths of the C ABI on the device, made on the host (no GPU fault is provoked): the
cancel flag the transport polls (MCmatlab.c:293-298 polls utIsInterruptPending the same way),
set before and during a run, and rejected inputs. Every failure returns a status and a
message, and the context stays usable afterwards."""
import threading
import time

import numpy as np
import pytest

import heatcases
import mccases
from mcmatlab_b200 import mexargs

pytestmark = pytest.mark.gpu


def _flag():
    from mcmatlab_b200 import native
    return native.lib().mcb_cancel_flag(native.context())


def test_cancel_before_run_then_context_reusable():
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    flag = _flag()
    flag[0] = 1
    try:
        with pytest.raises(native.MCBError) as e:
            native.mc_run(dict(mc_in, nPhotonsRequested=1e7))
        assert e.value.status == 4  # MCB_ECANCELLED
    finally:
        flag[0] = 0
    out = native.mc_run(mc_in)
    assert out["nPhotons"] == mc_in["nPhotonsRequested"]


def test_cancel_during_run():
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    native.mc_run(dict(mc_in, nPhotonsRequested=1e5))
    flag = _flag()
    timer = threading.Timer(0.3, lambda: flag.__setitem__(0, 1))
    t0 = time.perf_counter()
    timer.start()
    try:
        with pytest.raises(native.MCBError) as e:
            native.mc_run(dict(mc_in, nPhotonsRequested=2e9))  # tens of seconds uncancelled
        assert e.value.status == 4
    finally:
        timer.cancel()
        flag[0] = 0
    assert time.perf_counter() - t0 < 20.0
    assert native.mc_run(mc_in)["nPhotons"] == mc_in["nPhotonsRequested"]


@pytest.mark.parametrize("bad", ["medium_index", "mus", "boundary", "photons"])
def test_transport_rejects_bad_inputs(bad):
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    if bad == "medium_index":
        M = np.array(mc_in["M"], copy=True)
        M.flat[5] = 200
        mc_in["M"] = M
    elif bad == "mus":
        mus = np.array(mc_in["mus"], dtype=float, copy=True)
        mus[1, 0] = -1.0
        mc_in["mus"] = mus
    elif bad == "boundary":
        mc_in["boundaryType"] = 7
    else:
        mc_in["nPhotonsRequested"] = 0.0
    with pytest.raises(native.MCBError) as e:
        native.mc_run(mc_in)
    assert e.value.status == 1 and str(e.value)
    assert native.mc_run(mexargs.prepare_mc(mccases.c0_small()))["nPhotons"] > 0


@pytest.mark.parametrize("bad", ["steps", "sensor", "media"])
def test_heat_rejects_bad_inputs(bad):
    from mcmatlab_b200 import native
    case = heatcases.CASES["insulated_on"]()
    hp = dict(case["hp"])
    nx, ny, nz = case["n"]
    if bad == "steps":
        hp["steps"] = -1.0
    elif bad == "sensor":
        hp["tempSensorCornerIdxs"] = np.array([[float(nx * ny * nz)]])
        hp["tempSensorInterpWeights"] = np.zeros((1, 3))
    else:
        M = np.array(hp["M"], copy=True)
        M.flat[0] = 250  # beyond the media tables
        hp["M"] = M
    with pytest.raises(native.MCBError) as e:
        native.heat_forward(case["T0"], case["Omega0"], hp, nx, ny, nz)
    assert e.value.status == 1
    T, _, _, _ = native.heat_forward(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    assert np.all(np.isfinite(T))
