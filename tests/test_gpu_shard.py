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
