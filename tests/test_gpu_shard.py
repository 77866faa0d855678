"""Sharded transport on the device: shards of one seed run on one GPU one after another and
merged as the ranks' all-reduce would merge them equal the unsharded CUDA run."""
import numpy as np
import pytest

import mccases
from mcmatlab_b200 import mexargs, shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_gpu_shards_merge_to_unsharded_run(world):
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    mc_in["nPhotonsRequested"] = 200001.0
    mc_in["seed"] = 9
    full = native.mc_run(mc_in)
    acc = [None]

    def allreduce(a):
        acc[0] = a if acc[0] is None else acc[0] + a
        return acc[0]
    outs = [native.mc_run(shard.shard_model(mc_in, r, world)) for r in range(world)]
    for r in range(world):
        res = shard.merge(outs[r], mc_in, r, world, allreduce)
    assert res["nPhotons"] == full["nPhotons"] == 200001
    for k in ("NFR", "NI_zneg", "NI_xpos"):
        a, b = np.asarray(res[k], np.float64), np.asarray(full[k], np.float64)
        assert np.max(np.abs(a - b)) <= 2e-5 * np.max(np.abs(b)), k


def test_gpu_gradient_shards_merge_to_unsharded_run():
    """Perturbation-MC gradients: two shards of one seed run one after another on the GPU and
    merged as the ranks' all-reduce would merge them equal the unsharded gradient run (the
    gradient tallies are FP32 per thread, so to FP32 summation order)."""
    import gradcase
    from mcmatlab_b200 import native
    mc_in, obj = gradcase.case(n=24, nPhotons=100001)
    full_out, full = native.mc_grad(mc_in, **obj)
    acc = [None]

    def allreduce(a):
        acc[0] = a if acc[0] is None else acc[0] + a
        return acc[0]
    runs = [native.mc_grad(shard.shard_model(mc_in, r, 2), **obj) for r in range(2)]
    for r in range(2):
        res, g = shard.merge_grad(runs[r][0], runs[r][1], mc_in, obj["nRadialBins"], r, 2, allreduce)
    assert res["nPhotons"] == full_out["nPhotons"] == 100001
    assert abs(g["F"] - full["F"]) <= 1e-4 * abs(full["F"])
    for k in ("R", "dR_dmua", "dR_dmus", "dF_dmua", "dF_dmus"):
        a, b = np.asarray(g[k], np.float64), np.asarray(full[k], np.float64)
        assert np.max(np.abs(a - b)) <= 1e-4 * np.max(np.abs(b)), k
