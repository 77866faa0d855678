"""The streamed heat stepper (TMA-staged passes, coefficients and pivots formed on the fly)
against the FP64 oracle on every line-length class of its X, Y and Z passes, with and without
heat-sinked faces and light, at time steps up to far beyond the explicit limit (where the pivot
warm-up becomes the whole line), on the factored fallback for axes over 512 voxels, and at the
300x300x200 heat-adjoint workload size."""
import numpy as np
import pytest

import heatcases

pytestmark = pytest.mark.gpu

TOL_T = 1e-5          # relative, temperatures, sensors and per-medium maxima vs the FP64 oracle
TOL_OMEGA_INC = 1e-4  # relative to the damage accumulated in the call


def _check(case, oracle_lib):
    from mcmatlab_b200 import native
    from oracle import orc
    nx, ny, nz = case["n"]
    To, Oo, So, Mo = orc.oracle_heat(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    Tg, Og, Sg, Mg = native.heat_forward(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    err = {"T": float(np.max(np.abs(Tg - To) / np.abs(To)))}
    if So is not None:
        err["sensors"] = float(np.max(np.abs(Sg - So) / np.abs(So)))
    Mg = Mg.ravel().astype(np.float64)
    assert np.array_equal(np.isfinite(Mg), np.isfinite(Mo)) and np.all(Mg[~np.isfinite(Mg)] == Mo[~np.isfinite(Mo)])
    fin = np.isfinite(Mo)
    err["maxMediaTemps"] = float(np.max(np.abs(Mg[fin] - Mo[fin]) / np.abs(Mo[fin]))) if fin.any() else 0.0
    if Oo is not None:
        # relative to the damage accumulated in the call; Omega itself is FP32, so its own rounding
        # (2 ulp of the largest value) is allowed on top
        inc = np.max(np.abs(Oo - case["Omega0"]))
        excess = max(np.max(np.abs(Og - Oo)) - 2 * np.finfo(np.float32).eps * np.max(np.abs(Oo)), 0.0)
        err["Omega"] = float(excess / inc) if inc > 0 else float(excess)
    assert err["T"] <= TOL_T, err
    assert err.get("sensors", 0.0) <= TOL_T, err
    assert err["maxMediaTemps"] <= TOL_T, err
    assert err.get("Omega", 0.0) <= TOL_OMEGA_INC, err
    return err


SHAPES = [
    (100, 20, 18), (200, 12, 10), (300, 9, 8), (400, 6, 6), (37, 5, 7),       # X chunk classes 4, 8, 12, 16
    (16, 60, 8), (16, 130, 8), (20, 190, 6), (18, 250, 6), (18, 300, 6), (17, 500, 4),  # Y: 16 lanes, 32 lanes, 2 boxes
    (12, 10, 60), (12, 10, 250), (10, 8, 300), (10, 6, 510),                   # Z
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_streamed_stepper_line_classes(shape, oracle_lib):
    _check(heatcases.shaped(shape, seed=sum(shape)), oracle_lib)


@pytest.mark.parametrize("hs,lights", [(1, True), (1, False), (0, False)])
def test_streamed_stepper_sink_and_light(hs, lights, oracle_lib):
    _check(heatcases.shaped((44, 36, 28), seed=9, heatSinked=hs, lightsOn=lights, nt=20), oracle_lib)


@pytest.mark.parametrize("dtf", [1.5, 15.0, 400.0])
def test_streamed_stepper_large_time_steps(dtf, oracle_lib):
    """MCmatlab's own factors (1.5, 15 with largeTimeSteps) and one far beyond, where no
    contraction bound holds and every lane runs the pivot recurrence from the line start."""
    _check(heatcases.shaped((70, 40, 30), seed=13, nt=8, dt_factor=dtf), oracle_lib)


def test_factored_fallback_for_long_axes(oracle_lib):
    err = _check(heatcases.shaped((530, 16, 12), seed=17, nt=6), oracle_lib)
    assert err["Omega"] >= 0.0


def test_streamed_stepper_state_api_light_toggle(oracle_lib):
    """mcb_heat_state_*: light-on then light-off calls on one resident state equal the FP64
    oracle run the same way."""
    from mcmatlab_b200 import native
    from oracle import orc
    case = heatcases.shaped((60, 50, 40), seed=21, nt=10)
    nx, ny, nz = case["n"]
    off = dict(case["hp"])
    off["lightsOn"] = False
    To, Oo, _, _ = orc.oracle_heat(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    To, Oo, _, _ = orc.oracle_heat(To.astype(np.float32), Oo.astype(np.float32), off, nx, ny, nz)
    st = native.HeatState(case["T0"], case["Omega0"], case["hp"], nx, ny, nz)
    try:
        st.step(case["hp"])
        st.step(off)
        Tg, Og = st.read()
    finally:
        st.close()
    assert np.max(np.abs(Tg - To) / np.abs(To)) <= 2 * TOL_T


def test_streamed_stepper_c4_size(oracle_lib):
    """300x300x200 (the heat-adjoint workload size), light on, damage in the target, 50 steps."""
    case = heatcases.shaped((300, 300, 200), seed=21, nt=50)
    err = _check(case, oracle_lib)
    print("C4-size forward vs FP64 oracle, max relative errors:", err)


def _tri_inv(a, n):
    A = np.diag(np.full(n, 1 + 2 * a))
    A[0, 0] = A[-1, -1] = 1 + a
    A[np.arange(1, n), np.arange(n - 1)] = -a
    A[np.arange(n - 1), np.arange(1, n)] = -a
    return np.linalg.inv(A)


def _lap(T, ax):
    Tm, Tp = np.roll(T, 1, ax), np.roll(T, -1, ax)
    out = (Tm - T) + (Tp - T)
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    lo[ax], hi[ax] = 0, T.shape[ax] - 1
    out[tuple(lo)] = (Tp - T)[tuple(lo)]
    out[tuple(hi)] = (Tm - T)[tuple(hi)]
    return out


def _solve_axis(R, ax, a):
    return np.moveaxis(np.tensordot(_tri_inv(a, R.shape[ax]), np.moveaxis(R, ax, 0), axes=(1, 0)), 0, ax)


@pytest.mark.parametrize("on", [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)])
def test_each_pass_on_a_uniform_medium(on):
    """One DG-ADI step of a single medium with conduction along the selected axes only, against
    the step written out with dense line inverses: isolates the X, Y and Z passes."""
    from mcmatlab_b200 import mexargs, native
    rng = np.random.default_rng(3)
    nx, ny, nz = 40, 36, 30
    T0 = (37 + 2 * rng.random((nx, ny, nz))).astype(np.float32)
    c = np.zeros((1, 1, 3), np.float32)
    c[0, 0, :] = np.array([0.5, 0.4, 0.3]) * np.array(on)
    dt = 0.2
    hp = mexargs.heat_mex_params(np.ones((nx, ny, nz), np.uint8), [0.0], [0.0], c, np.zeros((nx, ny, nz), np.float32),
                                 True, 0, None, None, False, 1, dt)
    Tg, _, _, _ = native.heat_forward(T0, None, hp, nx, ny, nz)
    T = T0.astype(np.float64)
    H = (dt / 2) * c[0, 0, :].astype(np.float64)
    Dx, Dy, Dz = H[0] * _lap(T, 0), H[1] * _lap(T, 1), H[2] * _lap(T, 2)
    A1 = _solve_axis(T + 2 * (Dy + Dz) + Dx, 0, H[0])
    A2 = _solve_axis(A1 - Dy, 1, H[1])
    Tn = _solve_axis(A2 - Dz, 2, H[2])
    assert np.max(np.abs(Tg - Tn) / Tn) <= TOL_T
