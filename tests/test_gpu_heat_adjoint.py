"""GPU heat adjoint (mcb_heat_adjoint through the C ABI) against the FP64 oracle adjoint, whose
gradients are pinned to central differences on the CPU; checkpoint-count invariance."""
import numpy as np
import pytest

from mcmatlab_b200 import configs

pytestmark = pytest.mark.gpu

TOL_J = 1e-5     # relative, peak-temperature objective (FP32 stepper vs FP64)
TOL_JD = 1e-4    # relative, damage objective (Arrhenius amplifies the temperature error, as in the forward)
TOL_GRAD = 2e-3  # relative to the largest entry of each gradient


def _case(shape=(12, 10, 8), size=(0.12, 0.1, 0.08), nt=12, hs=0, light=True, peak=2000.0):
    case = configs.heat_adjoint_case(shape=shape, size=size, nt=nt, peak=peak, heatBoundaryType=hs)
    case["hp"]["lightsOn"] = light
    if not light:
        case["T0"] = np.asfortranarray(37.0 + 40.0 * case["S"] / case["S"].max()).astype(np.float32)
    return case


def _check(case, nCheckpoints=0):
    from mcmatlab_b200 import native
    from oracle import orc
    nx, ny, nz = case["n"]
    J, dc, dQ, dT = orc.oracle_heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"])
    g = native.heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"], nCheckpoints)
    assert abs(g["J_damage"] - J[1]) <= TOL_JD * abs(J[1]) + 1e-30
    assert abs(g["J_peak"] - J[2]) <= TOL_J * abs(J[2])
    for name, ref in (("dJ_dc", dc), ("dJ_dQ", dQ), ("dJ_dT0", dT)):
        scale = np.max(np.abs(ref))
        if scale == 0:
            assert np.all(g[name] == 0), name
            continue
        err = np.max(np.abs(g[name] - ref)) / scale
        assert err <= TOL_GRAD, (name, err)
    return g


@pytest.mark.parametrize("hs,light", [(0, True), (1, True), (0, False)])
def test_gpu_adjoint_matches_oracle_small(oracle_lib, hs, light):
    _check(_case(hs=hs, light=light))


def test_gpu_adjoint_matches_oracle_segments(oracle_lib):
    """A 40x36x30 grid over 50 steps with 7 checkpoints (segments of 8 steps, the last one short)."""
    _check(_case(shape=(40, 36, 30), size=(0.4, 0.36, 0.3), nt=50, peak=250.0), nCheckpoints=7)


@pytest.mark.parametrize("shape", [(20, 300, 200), (300, 24, 20), (400, 20, 16)])
def test_gpu_adjoint_line_length_classes(oracle_lib, shape):
    """The transposed solves' launch classes by line length against the FP64 oracle: y lines of 300
    rows (16-row lanes) and z lines of 200 (25 warps per line), x lines of 300 and 400 voxels
    (12 and 16 rows per lane); voxels of 1/300 cm as in the 300x300x200 workload, 8 steps with a
    heat-sinked boundary."""
    size = tuple(n / 300.0 for n in shape)
    _check(_case(shape=shape, size=size, nt=8, hs=1, peak=50.0), nCheckpoints=3)


def test_gpu_adjoint_checkpoint_count_invariance():
    from mcmatlab_b200 import native
    case = _case(shape=(24, 20, 16), size=(0.24, 0.2, 0.16), nt=30, peak=1500.0)
    nx, ny, nz = case["n"]
    # one segment, segments of 6, of 8 (the last one 6), of 2, and every state stored (30)
    runs = [native.heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"], k)
            for k in (1, 5, 4, 29, 30, 0)]
    # the recomputed inner states of the segments reproduce the forward states bit for bit; only
    # the order of the FP64 atomic sums (damage objective, dJ/dc) varies between runs
    for r in runs[1:]:
        assert abs(r["J"] - runs[0]["J"]) <= 1e-12 * abs(runs[0]["J"])
        np.testing.assert_allclose(r["dJ_dc"], runs[0]["dJ_dc"], rtol=1e-12, atol=1e-12 * np.max(np.abs(runs[0]["dJ_dc"])))
        for name in ("dJ_dQ", "dJ_dT0"):
            np.testing.assert_array_equal(r[name], runs[0][name])


def test_gpu_adjoint_matches_oracle_large(oracle_lib):
    """150x120x100 voxels (the 300x300x200 workload's voxel size, a tenth of its voxels) over 60
    steps with the default sqrt(N) checkpoints, against the FP64 oracle adjoint: objective and
    every gradient (the printed errors are the margin under the bounds)."""
    from mcmatlab_b200 import native
    from oracle import orc
    case = configs.heat_adjoint_case(shape=(150, 120, 100), size=(0.5, 0.4, 0.3), nt=60)
    nx, ny, nz = case["n"]
    J, dc, dQ, dT = orc.oracle_heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"])
    g = native.heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"])
    err = {"J_damage": abs(g["J_damage"] - J[1]) / abs(J[1]), "J_peak": abs(g["J_peak"] - J[2]) / abs(J[2])}
    for name, ref in (("dJ_dc", dc), ("dJ_dQ", dQ), ("dJ_dT0", dT)):
        err[name] = float(np.max(np.abs(g[name] - ref)) / np.max(np.abs(ref)))
    print("adjoint 150x120x100 x 60 vs FP64 oracle:", err)
    assert err["J_damage"] <= TOL_JD and err["J_peak"] <= TOL_J
    assert max(err["dJ_dc"], err["dJ_dQ"], err["dJ_dT0"]) <= TOL_GRAD, err
