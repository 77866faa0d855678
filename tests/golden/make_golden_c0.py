"""Generates mc_c0_ref.npz: the reference MC MEX on the 100^3 standard-tissue cube with 1e6
packets per batch (the transport benchmark's own configuration), K = 32 batches with pinned
dSFMT seeds 1001..1032, each batch single-threaded in one of several worker processes.

Stored (the voxel-wise parity test in tests/test_gpu_mc_c0.py reads it):

  summaries      [K x S] float64  per-batch summary statistics (tests/mcstats.py), names in `keys`
  mask           packed bits      voxels (column-major linear index) whose batch coefficient
                                  of variation is below CV_MAX: the voxels with adequate counts
  nfr_mean       float32          per-voxel mean of the K batch NFR values, masked voxels
  nfr_sd         float32          per-voxel standard deviation of the batch values (ddof 1)
  K, cv_max

Run from the repository root (needs oracle/_ref/libref_mc.so, i.e. `make -C oracle ref`):
    python tests/golden/make_golden_c0.py [workers]
"""
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

K = 32
FIRST_SEED = 1001
CV_MAX = 0.1
N_GRID = 100
PACKETS = 1e6


def c0_inputs():
    from mcmatlab_b200 import configs, mexargs
    return mexargs.prepare_mc(configs.standard_tissue_cube(n=N_GRID, nPhotons=PACKETS, seed=1))


def one_batch(seed):
    import mcstats
    from mcmatlab_b200 import mexargs
    from oracle import ref
    mc_in = c0_inputs()
    out = ref.RefMC().run(mexargs.mex_model_tree(mc_in), seed=seed)
    s = mcstats.summaries(out, mc_in)
    NFR = np.asarray(out["NFR"], dtype=np.float32)
    NFR = NFR[..., 0] if NFR.ndim == 4 else NFR
    return seed, s, NFR.ravel(order="F")


def main():
    workers = int(sys.argv[1]) if len(sys.argv) > 1 else os.cpu_count()
    ctx = mp.get_context("spawn")
    seeds = list(range(FIRST_SEED, FIRST_SEED + K))
    with ctx.Pool(workers) as pool:
        res = sorted(pool.map(one_batch, seeds), key=lambda r: r[0])
    keys = sorted(res[0][1])
    summ = np.array([[r[1][k] for k in keys] for r in res], dtype=np.float64)
    X = np.stack([r[2] for r in res]).astype(np.float64)  # [K, L]
    mean = X.mean(axis=0)
    sd = X.std(axis=0, ddof=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        cv = np.where(mean > 0, sd / mean, np.inf)
    mask = cv < CV_MAX
    print("voxels with CV < %.2f: %d of %d" % (CV_MAX, int(mask.sum()), mask.size))
    np.savez_compressed(os.path.join(HERE, "mc_c0_ref.npz"), summaries=summ, keys=np.array(keys),
                        mask=np.packbits(mask), nfr_mean=mean[mask].astype(np.float32),
                        nfr_sd=sd[mask].astype(np.float32), K=K, cv_max=CV_MAX)


if __name__ == "__main__":
    main()
