"""Packet sharding of one MC run over the ranks of a torch.distributed process group.

Packets are independent, so rank r of W runs packets r, r + W, r + 2W, ... of the unsharded
run's random streams (mcb_mc_model.packetOffset / packetStride) and the normalised outputs are
merged once at the end with a single all-reduce (NCCL over NVLink on GPUs, gloo on CPUs).
The merge is the weighted combination MCmatlab itself uses to merge runs
(+MCmatlab/@model/combineModels.m:59-101): every output of wavelength l is normalised by that
wavelength's launched packets, so the merged output is sum_r n_{r,l} out_{r,l} / sum_r n_{r,l}.
For a fixed packet count the shards together launch exactly the packets of the unsharded run,
so the merged result equals it up to floating-point summation order.

Perturbation-MC gradient runs shard the same way: their objective values and derivatives are
means over the launched packets too, so they merge with the same weights, in the same single
all-reduce as the forward outputs.

Heat is not sharded: its line solves couple whole grid axes (replicas only).
"""
from __future__ import annotations

import math

import numpy as np

# outputs merged with per-wavelength weights (last axis = wavelength when nL > 1)
WEIGHTED = ("NFR", "image", "farField", "NI_xpos", "NI_xneg", "NI_ypos", "NI_yneg", "NI_zpos", "NI_zneg")


def shard_count(total, rank, world):
    """Packets of rank `rank` when `total` packets are dealt round-robin over `world` ranks."""
    return (int(total) - rank + world - 1) // world if rank < int(total) else 0


def wavelength_counts(total, nL):
    """Packets per wavelength of a fixed-count run (the split of MCmatlab.c:635): an equal
    share for every wavelength but the last, which takes the remainder."""
    total = int(total)
    per = total // nL
    return [per] * (nL - 1) + [total - per * (nL - 1)]


def shard_model(mc_in, rank, world):
    """The MEX-level inputs of rank `rank`'s shard."""
    if math.isnan(float(mc_in["nPhotonsRequested"])) or mc_in.get("requestCollectedPhotons"):
        raise ValueError("sharding needs a fixed launched-packet count")
    m = dict(mc_in)
    m["nPhotonsRequested"] = float(shard_count(mc_in["nPhotonsRequested"], rank, world))
    m["packetOffset"] = int(mc_in.get("packetOffset", 0)) + rank * int(mc_in.get("packetStride", 1))
    m["packetStride"] = int(mc_in.get("packetStride", 1)) * world
    if rank != 0:
        m["nExamplePaths"] = 0
    return m


def _weights(mc_in, rank, world):
    nL = np.asarray(mc_in["mua"]).shape[1]
    n_r = wavelength_counts(shard_count(mc_in["nPhotonsRequested"], rank, world), nL)
    n = wavelength_counts(mc_in["nPhotonsRequested"], nL)
    return np.array([a / b if b else 0.0 for a, b in zip(n_r, n)]), nL


def merge(out, mc_in, rank, world, allreduce):
    """Combines this rank's outputs with the other ranks' through `allreduce(flat float64 array)
    -> summed array` (one call). Returns the merged output dict (on every rank).

    The layout of the reduced buffer comes from mc_in alone (abi.result_shapes), so every rank
    submits a buffer of the same length and order whatever its own run produced: an output this
    rank lacks (a rank that ran no packets passes out=None) contributes zeros. Non-finite values
    are reduced as they are, so a NaN on any rank stays NaN in the merge, as combineModels gives."""
    return _merge(out, mc_in, rank, world, allreduce)[0]


def _merge(out, mc_in, rank, world, allreduce, tail=None):
    """merge() with an optional flat float64 `tail` (already weighted by this rank) appended to
    the reduced buffer; returns (merged outputs, summed tail or None)."""
    from .abi import result_shapes
    w, nL = _weights(mc_in, rank, world)
    shapes = result_shapes(mc_in)
    keys = [k for k in WEIGHTED if k in shapes]
    out = out if out is not None else {}
    parts = []
    for k in keys:
        shp = shapes[k]
        a = out.get(k)
        if a is None or np.shape(a) != shp:
            parts.append(np.zeros(int(np.prod(shp))))
            continue
        a = np.asarray(a, dtype=np.float64)
        parts.append((a * w).reshape(-1, order="F"))
    counts = np.array([float(out.get("nPhotons", 0.0)), float(out.get("nPhotonsCollected", 0.0)),
                       float(out.get("nThreads", 0.0))])
    total = allreduce(np.concatenate(parts + [counts] + ([] if tail is None else [np.asarray(tail, np.float64)])))
    res = dict(out)
    off = 0
    for k in keys:
        shp = shapes[k]
        n = int(np.prod(shp))
        res[k] = total[off:off + n].reshape(shp, order="F").astype(np.float32)
        off += n
    res["nPhotons"] = total[off]
    res["nPhotonsCollected"] = total[off + 1]
    res["nThreads"] = total[off + 2]
    return res, (None if tail is None else total[off + 3:])


# gradient outputs (mcb_mc_grad_result) in the reduced buffer's order
GRAD_KEYS = ("R", "dR_dmua", "dR_dmus", "F", "dF_dmua", "dF_dmus")


def _grad_shapes(mc_in, nRadialBins):
    nM = int(np.asarray(mc_in["mua"]).shape[0])
    return {"R": (nRadialBins,), "dR_dmua": (nRadialBins, nM), "dR_dmus": (nRadialBins, nM), "F": (),
            "dF_dmua": (nM,), "dF_dmus": (nM,)}


def merge_grad(out, g, mc_in, nRadialBins, rank, world, allreduce):
    """merge() of a gradient run: the forward outputs as merge() does, and the objective values
    and derivatives (means over the launched packets of the single wavelength) weighted by this
    rank's share of the packets, all in one all-reduce. A rank without a run passes g=None."""
    shapes = _grad_shapes(mc_in, nRadialBins)
    w = _weights(mc_in, rank, world)[0][0]
    tail = []
    for k in GRAD_KEYS:
        n = int(np.prod(shapes[k]))
        a = None if g is None else g.get(k)
        tail.append(np.zeros(n) if a is None else w * np.asarray(a, np.float64).reshape(-1, order="F"))
    res, total = _merge(out, mc_in, rank, world, allreduce, np.concatenate(tail))
    gm, off = {}, 0
    for k in GRAD_KEYS:
        shp = shapes[k]
        n = int(np.prod(shp))
        v = total[off:off + n]
        gm[k] = float(v[0]) if shp == () else v.reshape(shp, order="F").copy()
        off += n
    return res, gm


def torch_allreduce(group=None):
    """all-reduce (sum) of a float64 numpy array through torch.distributed: on the rank's GPU for
    NCCL, on the host for gloo."""
    import torch
    import torch.distributed as dist

    def f(a):
        dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()
    return f


def sharded_mc_run(mc_in, run=None, group=None):
    """runMonteCarlo's MEX call on every rank of `group`: each rank runs its shard with `run`
    (default: the CUDA transport, native.mc_run) and all ranks return the merged outputs."""
    import torch.distributed as dist
    if run is None:
        from . import native
        run = native.mc_run
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    return sharded_run(mc_in, rank, world, run, torch_allreduce(group))


def sharded_run(mc_in, rank, world, run, allreduce):
    """One rank's part of a sharded run. Every check that can fail happens before any work and
    gives the same answer on every rank (it depends on mc_in only), so no rank leaves while the
    others wait in the collective. A rank whose shard is empty (fewer packets than ranks) runs
    nothing and contributes zeros."""
    total = float(mc_in["nPhotonsRequested"])
    if not math.isfinite(total) or mc_in.get("requestCollectedPhotons"):
        raise ValueError("sharding needs a fixed launched-packet count")
    if int(total) < 1:
        raise ValueError("nPhotonsRequested must be at least 1")
    out = run(shard_model(mc_in, rank, world)) if shard_count(total, rank, world) > 0 else None
    return merge(out, mc_in, rank, world, allreduce)


def sharded_mc_grad(mc_in, nRadialBins=32, radialBinWidth=0.01, box=None, run=None, group=None):
    """mcb_mc_grad on every rank of `group` (single wavelength): each rank runs its packet shard
    with `run(mc_in, nRadialBins=, radialBinWidth=, box=)` (default: the CUDA path,
    native.mc_grad) and all ranks return the merged (outputs, gradients)."""
    import torch.distributed as dist
    if run is None:
        from . import native
        run = native.mc_grad
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    return sharded_grad_run(mc_in, rank, world, run, torch_allreduce(group), nRadialBins=nRadialBins,
                            radialBinWidth=radialBinWidth, box=box)


def sharded_grad_run(mc_in, rank, world, run, allreduce, nRadialBins=32, radialBinWidth=0.01, box=None):
    """One rank's part of a sharded gradient run; the checks depend on mc_in only (same answer on
    every rank, before any work)."""
    total = float(mc_in["nPhotonsRequested"])
    if not math.isfinite(total) or mc_in.get("requestCollectedPhotons"):
        raise ValueError("sharding needs a fixed launched-packet count")
    if int(total) < 1:
        raise ValueError("nPhotonsRequested must be at least 1")
    if np.asarray(mc_in["mua"]).shape[1] != 1:
        raise ValueError("gradient runs take one wavelength")
    out, g = None, None
    if shard_count(total, rank, world) > 0:
        out, g = run(shard_model(mc_in, rank, world), nRadialBins=nRadialBins, radialBinWidth=radialBinWidth, box=box)
    return merge_grad(out, g, mc_in, nRadialBins, rank, world, allreduce)
