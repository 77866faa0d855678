"""GPU heat stepper parity: against the FP64 CPU oracle (relative tolerance stated per
output) and against the reference's FP32 stepper (golden outputs)."""
import os

import numpy as np
import pytest

import heatcases

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Tolerances vs the FP64 oracle (north star: heat and damage fields within 1e-5 relative)
TOL_T = 1e-5
TOL_SENS = 1e-5
TOL_OMEGA_INC = 1e-4  # relative to the damage accumulated in the call (Arrhenius amplifies T error ~0.6/K)


@pytest.mark.parametrize("name", sorted(heatcases.CASES))
def test_gpu_heat_vs_fp64_oracle(name, oracle_lib):
    from mcmatlab_b200 import native
    from oracle import orc
    case = heatcases.CASES[name]()
    nx, ny, nz = case["n"]
    To, Oo, So, Mo = orc.oracle_heat(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    Tg, Og, Sg, Mg = native.heat_forward(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    assert np.max(np.abs(Tg - To) / np.abs(To)) <= TOL_T
    if So is not None:
        assert np.max(np.abs(Sg - So) / np.abs(So)) <= TOL_SENS
    np.testing.assert_allclose(Mg.ravel(), Mo, rtol=TOL_T)
    if Oo is not None:
        inc = np.max(np.abs(Oo - case["Omega0"]))
        assert np.max(np.abs(Og - Oo)) <= TOL_OMEGA_INC * inc + 2 * np.finfo(np.float32).eps * np.max(np.abs(Oo))


@pytest.mark.parametrize("name", sorted(heatcases.CASES))
def test_gpu_heat_vs_reference_fp32(name):
    """Difference to the reference FP32 build stays within the reference's own FP32 drift."""
    from mcmatlab_b200 import native
    gold = np.load(os.path.join(GOLD, "heat_ref.npz"))
    case = heatcases.CASES[name]()
    nx, ny, nz = case["n"]
    nt = int(case["hp"]["steps"])
    Tg, Og, Sg, Mg = native.heat_forward(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    Tr = gold[name + "_T"]
    assert np.max(np.abs(Tg - Tr) / np.abs(Tr)) <= 1e-6 * nt + 2e-6
    np.testing.assert_allclose(Mg.ravel(), gold[name + "_maxMediaTemps"].ravel(), rtol=1e-6 * nt + 2e-6)


def test_gpu_heat_uniform_and_conservation(oracle_lib):
    from mcmatlab_b200 import configs, native, prep
    case = heatcases.insulated_on()
    hp = dict(case["hp"])
    hp["lightsOn"] = False
    hp["steps"] = 200.0
    nx, ny, nz = case["n"]
    U = np.full((nx, ny, nz), 41.5, np.float32)
    T, _, _, _ = native.heat_forward(U, None, hp, nx, ny, nz)
    assert np.max(np.abs(T - 41.5)) == 0.0
    m = configs.standard_tissue_cube(n=nx, nPhotons=1)
    th = prep.thermal_media_properties(m.G.mediaPropertiesFunc([]), m.G.M_raw)
    vhc = th["VHC"][th["M"].astype(int) - 1]
    T, _, _, _ = native.heat_forward(case["T0"], None, hp, nx, ny, nz)
    e0 = np.sum(vhc * case["T0"].astype(np.float64))
    assert abs(np.sum(vhc * T.astype(np.float64)) - e0) <= 1e-6 * abs(e0)


def test_gpu_heat_long_run_c1_geometry(oracle_lib):
    """100^3 standard-tissue grid, light on, 300 steps at 0.9x the stability limit."""
    from mcmatlab_b200 import native
    from oracle import orc
    case = heatcases._base(100, 11, 0, True, 300, 0.9, True)
    nx, ny, nz = case["n"]
    To, Oo, So, Mo = orc.oracle_heat(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    Tg, Og, Sg, Mg = native.heat_forward(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    errT = np.max(np.abs(Tg - To) / np.abs(To))
    print("100^3 x 300 steps vs FP64 oracle: max relative T error %.3g" % errT)
    assert errT <= TOL_T
    inc = np.max(np.abs(Oo - case["Omega0"]))
    assert np.max(np.abs(Og - Oo)) <= TOL_OMEGA_INC * inc + 2 * np.finfo(np.float32).eps * np.max(np.abs(Oo))
