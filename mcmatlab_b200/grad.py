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
