"""MC packet sharding over a process group: shard arithmetic, and on two gloo ranks (CPU, the
oracle as each rank's transport) the merged result equals the unsharded run of the same seed."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

import mccases
from mcmatlab_b200 import mexargs, shard


def test_shard_counts_partition_packets():
    for total in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            counts = [shard.shard_count(total, r, world) for r in range(world)]
            assert sum(counts) == total
            ids = sorted(r + world * k for r in range(world) for k in range(counts[r]))
            assert ids == list(range(total))
    assert shard.wavelength_counts(10, 3) == [3, 3, 4]


def _case():
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    mc_in["nPhotonsRequested"] = 4001.0
    mc_in["seed"] = 5
    return mc_in


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import orc
        out = shard.sharded_mc_run(_case(), run=lambda m: orc.oracle_mc(m, 2))
        if rank == 0:
            q.put({k: out[k] for k in ("NFR", "NI_zneg", "nPhotons")})
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_merge_to_the_unsharded_run(oracle_lib):
    from oracle import orc
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    full = orc.oracle_mc(_case(), 4)
    assert got["nPhotons"] == full["nPhotons"] == 4001
    for k in ("NFR", "NI_zneg"):
        a, b = np.asarray(got[k], np.float64), np.asarray(full[k], np.float64)
        assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(b)), k


def test_shards_run_disjoint_streams(oracle_lib):
    """Two shards of one seed differ from each other, and the unsharded run is their merge."""
    from oracle import orc
    mc_in = _case()
    outs = [orc.oracle_mc(shard.shard_model(mc_in, r, 2), 2) for r in range(2)]
    assert not np.allclose(outs[0]["NFR"], outs[1]["NFR"])
    merged = [None]

    def fake_allreduce(rank):
        def f(a):
            merged[0] = a if merged[0] is None else merged[0] + a
            return merged[0]
        return f
    shard.merge(outs[0], mc_in, 0, 2, fake_allreduce(0))
    res = shard.merge(outs[1], mc_in, 1, 2, fake_allreduce(1))
    full = orc.oracle_mc(mc_in, 4)
    assert np.max(np.abs(res["NFR"] - full["NFR"])) <= 1e-5 * np.max(full["NFR"])


def _rank_few(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import orc
        m = _case()
        m["nPhotonsRequested"] = 2.0
        out = shard.sharded_mc_run(m, run=lambda mm: orc.oracle_mc(mm, 1))
        q.put((rank, float(out["nPhotons"]), np.asarray(out["NFR"], np.float64)))
    finally:
        dist.destroy_process_group()


def test_fewer_packets_than_ranks_merges_without_hanging(oracle_lib):
    """Three gloo ranks share two packets: the rank with an empty shard runs nothing and
    contributes zeros, every rank submits the same buffer layout, and all of them return the
    unsharded two-packet result."""
    from oracle import orc
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_few, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(3)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    m = _case()
    m["nPhotonsRequested"] = 2.0
    full = orc.oracle_mc(m, 1)
    for rank, n, nfr in got:
        assert n == 2.0
        np.testing.assert_allclose(nfr, np.asarray(full["NFR"], np.float64), rtol=1e-5, atol=1e-6 * np.max(full["NFR"]))


def test_empty_run_is_rejected_on_every_rank_before_the_collective():
    calls = []
    m = _case()
    m["nPhotonsRequested"] = 0.0
    for rank in range(2):
        with pytest.raises(ValueError):
            shard.sharded_run(m, rank, 2, run=lambda mm: calls.append(mm), allreduce=lambda a: calls.append(a))
    assert calls == []


def test_merge_layout_is_independent_of_the_rank_outputs():
    """A rank whose run lacks an output, or holds NaNs, still submits the full layout."""
    m = _case()
    sizes = []

    def fake(a):
        sizes.append(a.size)
        return a
    shard.merge(None, m, 0, 2, fake)
    shard.merge({"NFR": np.full((2, 2, 2, 1), np.nan), "nPhotons": 1.0, "nPhotonsCollected": 0.0, "nThreads": 1.0},
                m, 1, 2, fake)
    assert sizes[0] == sizes[1] and sizes[0] > 3


def _grad_case():
    import gradcase
    mc_in, obj = gradcase.case(n=20, nPhotons=3001)
    return mc_in, obj


def _rank_grad(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import orc
        mc_in, obj = _grad_case()
        out, g = shard.sharded_mc_grad(mc_in, run=lambda m, **o: orc.oracle_mc_grad(m, nthreads=2, **o), **obj)
        if rank == 0:
            q.put((float(out["nPhotons"]), np.asarray(out["NI_zneg"], np.float64), g))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_merge_gradients_to_the_unsharded_run(oracle_lib):
    """Perturbation-MC gradients sharded over two gloo ranks (the oracle as each rank's transport):
    the merged objective values and derivatives equal the unsharded run of the same seed up to
    floating-point summation order, and so do the forward outputs merged in the same all-reduce."""
    from oracle import orc
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_grad, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    nph, ni, g = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    mc_in, obj = _grad_case()
    full_out, full = orc.oracle_mc_grad(mc_in, nthreads=4, **obj)
    assert nph == full_out["nPhotons"] == 3001
    b = np.asarray(full_out["NI_zneg"], np.float64)
    assert np.max(np.abs(ni - b)) <= 1e-5 * np.max(np.abs(b))
    assert abs(g["F"] - full["F"]) <= 1e-9 * abs(full["F"])
    for k in ("R", "dR_dmua", "dR_dmus", "dF_dmua", "dF_dmus"):
        a, r = np.asarray(g[k], np.float64), np.asarray(full[k], np.float64)
        assert a.shape == r.shape, k
        assert np.max(np.abs(a - r)) <= 1e-9 * np.max(np.abs(r)), k


def test_gradient_shards_reject_several_wavelengths():
    mc_in, obj = _grad_case()
    m = dict(mc_in, mua=np.repeat(np.asarray(mc_in["mua"]), 2, axis=1))
    with pytest.raises(ValueError):
        shard.sharded_grad_run(m, 0, 2, None, None, **obj)


def test_gradient_merge_of_a_rank_without_packets_contributes_zeros():
    """A rank with an empty shard submits the same buffer layout as the others (zeros), so the
    merged gradients are the running rank's values weighted by its full share."""
    mc_in, obj = _grad_case()
    mc_in = dict(mc_in, nPhotonsRequested=1.0)
    nR, nM = obj["nRadialBins"], np.asarray(mc_in["mua"]).shape[0]
    g0 = {"R": np.arange(nR, dtype=np.float64), "dR_dmua": np.ones((nR, nM)), "dR_dmus": -np.ones((nR, nM)),
          "F": 2.5, "dF_dmua": np.full(nM, 3.0), "dF_dmus": np.full(nM, -4.0)}
    bufs = []

    def ar(a):
        bufs.append(np.array(a))
        return sum(bufs) if len(bufs) == 2 else a
    shard.merge_grad({"nPhotons": 1.0}, g0, mc_in, nR, 0, 2, ar)
    res, g = shard.merge_grad(None, None, mc_in, nR, 1, 2, ar)
    assert bufs[0].shape == bufs[1].shape
    assert res["nPhotons"] == 1.0
    assert g["F"] == 2.5
    np.testing.assert_array_equal(g["R"], g0["R"])
    np.testing.assert_array_equal(g["dF_dmus"], g0["dF_dmus"])
    assert g["dR_dmua"].shape == (nR, nM)
