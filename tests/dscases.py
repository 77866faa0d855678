"""Seeded inputs for the sub-media binning (getDownsampledParamVals): random (mua, mus, g)
clouds with rows that vary or not, many exact ties, a single point, more bins than points."""
import numpy as np


def cases(count=120, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        kind = t % 6
        n = int(rng.integers(1, 2500))
        nb = int(rng.integers(1, 48))
        par = np.zeros((3, n), np.float32)
        par[0] = rng.uniform(0.1, 10, n)
        par[1] = rng.uniform(10, 100, n) if kind != 1 else 50.0
        par[2] = rng.uniform(0.7, 0.95, n) if kind != 2 else 0.0
        if kind == 3:
            par[0] = np.round(par[0])  # many exact ties
        if kind == 4:
            par[:] = 1.0
            par[0, ::7] = 2.0
        if kind == 5:
            n = int(rng.integers(1, 6))
            par = rng.uniform(0, 1, (3, n)).astype(np.float32)
            nb = int(rng.integers(1, 12))  # possibly more bins than points
        out.append((np.asfortranarray(par), nb))
    out.append((np.ones((3, 50), np.float32, order="F"), 5))  # nothing varies
    out.append((np.asfortranarray(rng.uniform(0, 1, (3, 300)).astype(np.float32)), 1))  # one bin
    out.append((np.asfortranarray(rng.uniform(0, 1, (3, 300)).astype(np.float32)), 255))  # the most bins
    return out
