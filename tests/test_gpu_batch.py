"""Batched transport: many models of different grids, wavelengths, media and photon counts in
one launch give the same results as running each model alone (same seed-keyed streams)."""
import numpy as np
import pytest

from mcmatlab_b200 import configs, mexargs

pytestmark = pytest.mark.gpu


def test_batch_equals_single_runs():
    from mcmatlab_b200 import native
    models = configs.batched_sweep(n_instances=6, seed=3, min_grid=(24, 24, 20), max_grid=(40, 40, 30),
                                   photons=(1e4, 5e4))
    ins = [mexargs.prepare_mc(m) for m in models]
    batch = native.mc_run_batch(ins)
    for k, mc_in in enumerate(ins):
        single = native.mc_run(mc_in)
        b = batch[k]
        assert b["nPhotons"] == single["nPhotons"] == mc_in["nPhotonsRequested"]
        assert b["nPhotonsCollected"] == single["nPhotonsCollected"]
        for key in ("NFR", "NI_zneg", "NI_zpos", "image"):
            if key in single:
                a, c = b[key], single[key]
                np.testing.assert_allclose(a, c, rtol=1e-6, atol=1e-6 * float(np.max(np.abs(c)) + 1e-30))


def test_batch_rejects_open_ended_models():
    from mcmatlab_b200 import native
    models = configs.batched_sweep(n_instances=2, seed=4, min_grid=(20, 20, 20), max_grid=(24, 24, 24),
                                   photons=(1e4, 2e4))
    ins = [mexargs.prepare_mc(m) for m in models]
    ins[1]["nPhotonsRequested"] = float("nan")
    with pytest.raises(native.MCBError):
        native.mc_run_batch(ins)
