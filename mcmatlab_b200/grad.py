"""Gradient harness: the derivative entries of libmcb200 as torch.autograd.Functions.

The compute stays in the CUDA library (mcb_heat_adjoint, mcb_mc_grad); torch only carries the
chain rule from the MEX-level tables to physical parameters, e.g. from the conduction table c
and heat source Q to per-medium TC, VHC and the per-voxel source power density:

    TC, VHC, S = (torch tensors, requires_grad=True)
    c, Q = thermal_tables(TC, VHC, S, M1, (dx, dy, dz))
    J = HeatObjective.apply(c, Q, T0, hp, (nx, ny, nz), damageWeight, peakWeight)
    J.backward()          # TC.grad, VHC.grad, S.grad

    R, F = ReflectanceFluence.apply(mua, mus, mc_in, objectives)   # perturbation Monte Carlo

thermal_tables restates calcdTdtArrays (+MCmatlab/@model/simulateHeatDistribution.m:469-494):
TC_eff(i, j) = 2 TC_i TC_j / (TC_i + TC_j), c(i, j, d) = TC_eff(i, j) / VHC_i / d_d^2 and
Q = S / VHC(M), in float64.
"""
from __future__ import annotations

import numpy as np
import torch

from . import native


def thermal_tables(TC, VHC, S, M1, d):
    """c [nM, nM, 3] and Q (grid shaped) as differentiable functions of TC, VHC [nM] and S (grid)."""
    TC = TC.to(torch.float64)
    VHC = VHC.to(torch.float64)
    TCeff = 2 * TC[:, None] * TC[None, :] / (TC[:, None] + TC[None, :])
    base = TCeff / VHC[:, None]
    c = torch.stack([base / float(d[0]) ** 2, base / float(d[1]) ** 2, base / float(d[2]) ** 2], dim=2)
    idx = torch.as_tensor(np.asarray(M1, dtype=np.int64) - 1)
    Q = S.to(torch.float64) / VHC[idx]
    return c, Q


class HeatObjective(torch.autograd.Function):
    """J(c, Q, T0) of mcb_heat_adjoint: damage gained over the weighted voxels plus the weighted
    per-voxel peak temperatures; backward returns dJ/dc, dJ/dQ, dJ/dT0 from the adjoint sweep."""

    @staticmethod
    def forward(ctx, c, Q, T0, hp, n, damageWeight=None, peakWeight=None, nCheckpoints=0):
        hp2 = dict(hp)
        hp2["dTdtperdeltaT"] = np.asfortranarray(c.detach().cpu().numpy().astype(np.float32))
        hp2["dTdt_abs"] = np.asfortranarray(Q.detach().cpu().numpy().astype(np.float32))
        nx, ny, nz = n
        g = native.heat_adjoint(T0.detach().cpu().numpy(), hp2, nx, ny, nz, damageWeight, peakWeight, nCheckpoints)
        ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(g["dJ_dc"])),
                              torch.from_numpy(np.ascontiguousarray(g["dJ_dQ"], dtype=np.float64)),
                              torch.from_numpy(np.ascontiguousarray(g["dJ_dT0"], dtype=np.float64)))
        ctx.dtypes = (c.dtype, Q.dtype, T0.dtype)
        return torch.tensor(g["J"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        dc, dQ, dT = ctx.saved_tensors
        tc, tq, tt = ctx.dtypes
        return (gJ * dc).to(tc), (gJ * dQ).to(tq), (gJ * dT).to(tt), None, None, None, None, None


class ReflectanceFluence(torch.autograd.Function):
    """(R [nRadialBins], F) of mcb_mc_grad as functions of per-medium mua and mus [nM] (one
    wavelength). backward contracts the perturbation-MC derivatives with the incoming gradients."""

    @staticmethod
    def forward(ctx, mua, mus, mc_in, objectives):
        m = dict(mc_in)
        m["mua"] = mua.detach().cpu().numpy().astype(np.float64).reshape(-1, 1)
        m["mus"] = mus.detach().cpu().numpy().astype(np.float64).reshape(-1, 1)
        _, g = native.mc_grad(m, **objectives)
        ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(g["dR_dmua"])),
                              torch.from_numpy(np.ascontiguousarray(g["dR_dmus"])),
                              torch.from_numpy(g["dF_dmua"]), torch.from_numpy(g["dF_dmus"]))
        ctx.dtypes = (mua.dtype, mus.dtype)
        return torch.from_numpy(g["R"]), torch.tensor(g["F"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, gR, gF):
        dRa, dRs, dFa, dFs = ctx.saved_tensors
        ga = gR @ dRa + gF * dFa
        gs = gR @ dRs + gF * dFs
        return ga.to(ctx.dtypes[0]), gs.to(ctx.dtypes[1]), None, None


def recover_optical_properties(mc_in, R_target, fit_media, objectives, mua0=None, mus0=None, max_evals=40,
                               history_size=10, tolerance_change=1e-7, transport=None):
    """Fits per-medium absorption and scattering coefficients to a radial reflectance map.

    mc_in: MEX-level inputs of one wavelength (mexargs.prepare_mc); R_target: the measured
    reflectance [nRadialBins] (same objectives); fit_media: 0-based medium indices to fit (the
    others keep mc_in's values); mua0, mus0: starting values of the fitted media (default mc_in's).

    Minimises the mean over bins with R_target > 0 of ((R_b - R_target_b) / R_target_b)^2 with
    torch.optim.LBFGS (strong Wolfe line search) over log(mua), log(mus), so the coefficients stay
    positive. Every evaluation runs the perturbation-MC transport (ReflectanceFluence) with
    mc_in's seed, so all evaluations share their random numbers (common random numbers): the
    objective is a deterministic function of the parameters and its gradient comes from the same
    packets. `transport` replaces native.mc_grad (same signature) for testing the fit logic.

    Returns dict(mua, mus (full per-medium arrays), loss, evals, history [(loss, mua_fit, mus_fit)])."""
    idx = torch.as_tensor(np.asarray(fit_media, dtype=np.int64))
    base_a = torch.as_tensor(np.asarray(mc_in["mua"], dtype=np.float64)[:, 0])
    base_s = torch.as_tensor(np.asarray(mc_in["mus"], dtype=np.float64)[:, 0])
    a0 = base_a[idx] if mua0 is None else torch.as_tensor(np.asarray(mua0, dtype=np.float64))
    s0 = base_s[idx] if mus0 is None else torch.as_tensor(np.asarray(mus0, dtype=np.float64))
    la = a0.log().clone().requires_grad_(True)
    ls = s0.log().clone().requires_grad_(True)
    Rt = torch.as_tensor(np.asarray(R_target, dtype=np.float64))
    use = Rt > 0
    history = []
    fn = ReflectanceFluence if transport is None else _with_transport(transport)

    def closure():
        opt.zero_grad()
        mua = base_a.clone()
        mus = base_s.clone()
        mua[idx] = la.exp()
        mus[idx] = ls.exp()
        R, _ = fn.apply(mua, mus, mc_in, objectives)
        loss = (((R - Rt) / Rt)[use] ** 2).mean()
        loss.backward()
        history.append((float(loss.detach()), la.detach().exp().numpy().copy(), ls.detach().exp().numpy().copy()))
        return loss

    opt = torch.optim.LBFGS([la, ls], lr=1.0, max_iter=max_evals, max_eval=max_evals, history_size=history_size,
                            tolerance_grad=1e-12, tolerance_change=tolerance_change, line_search_fn="strong_wolfe")
    opt.step(closure)
    best = min(history, key=lambda h: h[0])
    mua = base_a.numpy().copy()
    mus = base_s.numpy().copy()
    mua[idx.numpy()] = best[1]
    mus[idx.numpy()] = best[2]
    return {"mua": mua, "mus": mus, "loss": best[0], "evals": len(history), "history": history}


def _with_transport(transport):
    """ReflectanceFluence with another mc_grad-like transport (tests of the fit logic)."""

    class _F(ReflectanceFluence):
        @staticmethod
        def forward(ctx, mua, mus, mc_in, objectives):
            m = dict(mc_in)
            m["mua"] = mua.detach().cpu().numpy().astype(np.float64).reshape(-1, 1)
            m["mus"] = mus.detach().cpu().numpy().astype(np.float64).reshape(-1, 1)
            _, g = transport(m, **objectives)
            ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(g["dR_dmua"])),
                                  torch.from_numpy(np.ascontiguousarray(g["dR_dmus"])),
                                  torch.from_numpy(np.asarray(g["dF_dmua"])), torch.from_numpy(np.asarray(g["dF_dmus"])))
            ctx.dtypes = (mua.dtype, mus.dtype)
            return torch.from_numpy(np.asarray(g["R"])), torch.tensor(g["F"], dtype=torch.float64)

    return _F
