"""Generates the golden fixtures in this folder by running the reference's own C code.

The reference has no golden vectors or known-answer tests of its own, so parity is
pinned on outputs of the reference MEX sources compiled here (oracle/_ref, built by
`make -C oracle`) on seeded inputs:

  mc_ref_summaries.json   K reference batches (pinned dSFMT seeds 101..) of summary
                          statistics (tests/mcstats.py) for every case in tests/mccases.py
                          (CASES as MC runs, FLUO_CASES as fluorescence runs)
  heat_ref.npz            reference FP32 heat MEX outputs for small seeded problems

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from mcmatlab_b200 import mexargs  # noqa: E402
from oracle import ref  # noqa: E402
import mccases  # noqa: E402
import mcstats  # noqa: E402
import heatcases  # noqa: E402

K = 8


def main():
    R = ref.RefMC()
    out = {}
    for name, fn in mccases.CASES.items():
        mc_in = mexargs.prepare_mc(fn())
        tree = mexargs.mex_model_tree(mc_in)
        out[name] = [mcstats.summaries(R.run(tree, seed=101 + s), mc_in) for s in range(K)]
        print(name, "done", flush=True)
    for name, fn in mccases.FLUO_CASES.items():
        mc_in = mexargs.prepare_mc(fn(), 2)
        tree = mexargs.mex_model_tree(mc_in)  # filled FMC node: the MEX runs as simType 2
        out[name] = [mcstats.summaries(R.run(tree, seed=101 + s), mc_in) for s in range(K)]
        print(name, "done", flush=True)
    with open(os.path.join(HERE, "mc_ref_summaries.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    H = ref.RefHeat()
    arrays = {}
    for name, fn in heatcases.CASES.items():
        case = fn()
        T, Om, S, Mx = H.run(case["T0"], case["Omega0"] if case["Omega0"] is not None else np.float32(np.nan), case["hp"])
        arrays[name + "_T"] = T
        if case["Omega0"] is not None:
            arrays[name + "_Omega"] = Om
        arrays[name + "_sensorTemps"] = S
        arrays[name + "_maxMediaTemps"] = Mx
        print(name, "done", flush=True)
    np.savez_compressed(os.path.join(HERE, "heat_ref.npz"), **arrays)


if __name__ == "__main__":
    main()
