"""The FP64 oracle's adjoint of the DG-ADI stepper: its forward objective agrees with the
reference-pinned forward oracle (orc_heat_run), and its gradients with respect to the conduction
table c, the heat source Q and the initial temperature agree with FP64 central differences."""
import numpy as np
import pytest

from mcmatlab_b200 import configs


def _case(hs=0, light=True):
    case = configs.heat_adjoint_case(shape=(12, 10, 8), size=(0.12, 0.1, 0.08), nt=12, peak=2000.0,
                                     heatBoundaryType=hs)
    case["hp"]["lightsOn"] = light
    if not light:  # start hot so that damage and peaks still depend on the parameters
        case["T0"] = np.asfortranarray(37.0 + 40.0 * case["S"] / case["S"].max()).astype(np.float32)
    return case


@pytest.mark.parametrize("hs,light", [(0, True), (1, True), (0, False)])
def test_oracle_adjoint_matches_central_differences(oracle_lib, hs, light):
    from oracle import orc
    case = _case(hs, light)
    nx, ny, nz = case["n"]
    hp, wd, wp = case["hp"], case["wd"], case["wp"]
    J, dc, dQ, dT = orc.oracle_heat_adjoint(case["T0"], hp, nx, ny, nz, wd, wp)
    run = lambda **kw: orc.oracle_heat_adjoint(kw.pop("T0", case["T0"]), hp, nx, ny, nz, wd, wp, grads=False, **kw)[0]
    c = np.asarray(hp["dTdtperdeltaT"], dtype=np.float64)
    for idx in [(0, 0, 0), (3, 3, 2), (0, 3, 1), (3, 0, 1), (1, 1, 2), (0, 1, 2)]:
        h = 1e-5 * c[idx]
        cp, cm = c.copy(), c.copy()
        cp[idx] += h
        cm[idx] -= h
        fd = (run(c=cp) - run(c=cm)) / (2 * h)
        assert abs(fd - dc[idx]) <= 1e-6 * np.max(np.abs(dc)), (idx, fd, dc[idx])
    Q = np.asarray(hp["dTdt_abs"], dtype=np.float64)
    T0 = np.asarray(case["T0"], dtype=np.float64)
    for v in [(6, 5, 4), (3, 2, 2), (1, 8, 6)]:
        h = 1e-3
        Qp, Qm = Q.copy(), Q.copy()
        Qp[v] += h
        Qm[v] -= h
        fd = (run(Q=Qp) - run(Q=Qm)) / (2 * h)
        assert abs(fd - dQ[v]) <= 1e-6 * np.max(np.abs(dQ)) + 1e-12, (v, fd, dQ[v])
        Tp, Tm = T0.copy(), T0.copy()
        Tp[v] += h
        Tm[v] -= h
        fd = (run(T0=Tp) - run(T0=Tm)) / (2 * h)
        assert abs(fd - dT[v]) <= 1e-6 * np.max(np.abs(dT)), (v, fd, dT[v])
    if not light:
        assert np.all(dQ == 0)


def test_oracle_adjoint_forward_restates_forward_oracle(oracle_lib):
    """The damage part of the adjoint's objective is the damage orc_heat_run accumulates."""
    from oracle import orc
    case = _case()
    nx, ny, nz = case["n"]
    J = orc.oracle_heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"], grads=False)
    _, Om, _, _ = orc.oracle_heat(case["T0"], np.zeros(case["n"], np.float32), case["hp"], nx, ny, nz)
    assert J[1] > 0
    assert abs(J[1] - float((case["wd"] * Om).sum())) <= 1e-12 * J[1]
    assert J[0] == J[1] + J[2]


def test_oracle_adjoint_matches_reference_stepper_differences(oracle_lib, ref_available):
    """Central differences of the reference's own FP32 stepper (damage objective) against the
    oracle adjoint: agreement within the FP32 difference noise."""
    if not ref_available:
        pytest.skip("reference build not present")
    from oracle import orc, ref
    case = _case()
    nx, ny, nz = case["n"]
    hp, wd = case["hp"], case["wd"]
    _, dc, dQ, _ = orc.oracle_heat_adjoint(case["T0"], hp, nx, ny, nz, wd, None)
    rh = ref.RefHeat()

    def Jref(c=None, Q=None):
        p = dict(hp)
        if c is not None:
            p["dTdtperdeltaT"] = np.asfortranarray(c.astype(np.float32))
        if Q is not None:
            p["dTdt_abs"] = np.asfortranarray(Q.astype(np.float32))
        _, Om, _, _ = rh.run(case["T0"], np.zeros(case["n"], np.float32), p, nthreads=1)
        return float((wd.astype(np.float64) * Om.astype(np.float64)).sum())

    c = np.asarray(hp["dTdtperdeltaT"], dtype=np.float64)
    h = 2e-2
    for idx in [(0, 0, 2), (3, 3, 0), (3, 0, 1)]:
        cp, cm = c.copy(), c.copy()
        cp[idx] *= 1 + h
        cm[idx] *= 1 - h
        fd = (Jref(c=cp) - Jref(c=cm)) / (2 * h * c[idx])
        assert abs(fd - dc[idx]) <= 2e-2 * np.max(np.abs(dc)), (idx, fd, dc[idx])
    Q = np.asarray(hp["dTdt_abs"], dtype=np.float64)
    v = np.unravel_index(np.argmax(np.abs(dQ)), dQ.shape)
    Qp, Qm = Q.copy(), Q.copy()
    Qp[v] *= 1 + h
    Qm[v] *= 1 - h
    fd = (Jref(Q=Qp) - Jref(Q=Qm)) / (2 * h * Q[v])
    assert abs(fd - dQ[v]) <= 2e-2 * abs(dQ[v]), (fd, dQ[v])
