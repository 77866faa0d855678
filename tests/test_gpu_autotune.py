"""The transport autotuner (mcb_mc_autotune): it times the 16 (refillMin, scatterMin) candidates,
keeps the fastest for the model's size class, records it in the tuning file, and the results of
later runs do not change (each packet's random stream is fixed; only the scheduling moves)."""
import numpy as np
import pytest

import mccases
from mcmatlab_b200 import mexargs

pytestmark = pytest.mark.gpu


def test_gpu_autotune_chooses_fastest_and_keeps_results(tmp_path, monkeypatch):
    from mcmatlab_b200 import native
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("MCB_TUNE_FILE", str(path))
    mc_in = mexargs.prepare_mc(mccases.c0_small())
    before = native.mc_run(mc_in)
    t = native.mc_autotune(mc_in, 5e4)
    table = t["table"]
    assert table.shape == (16, 3) and np.all(table[:, 2] > 0)
    best = table[np.argmin(table[:, 2])]
    assert (t["refillMin"], t["scatterMin"]) == (int(best[0]), int(best[1]))
    after = native.mc_run(mc_in)
    assert after["nPhotons"] == before["nPhotons"] and after["propagationSteps"] == before["propagationSteps"]
    np.testing.assert_allclose(after["NFR"], before["NFR"], rtol=1e-6, atol=1e-9 * float(before["NFR"].max()))
    lines = path.read_text().strip().splitlines()
    assert len(lines) == 1
    name, cls, r, s = lines[0].split("\t")
    assert int(cls) == t["sizeClass"] and (int(r), int(s)) == (t["refillMin"], t["scatterMin"])
