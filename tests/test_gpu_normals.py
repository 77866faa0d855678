"""Interface normals on the device (mcb_interface_normals through the C ABI) against the host
restatement (prep.interface_normals: Sobel per refractive-index class, then the smoothn
smoothing), compared as unit vectors at the voxels where the refractive index changes (the
only voxels whose normals the transport reads)."""
import numpy as np
import pytest

from mcmatlab_b200 import prep

pytestmark = pytest.mark.gpu


def _grid(shape, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    M1 = np.ones(shape, dtype=np.uint8)
    M1[Z >= nz // 3] = 2
    M1[Z >= 2 * nz // 3] = 3
    c = rng.uniform(0.3, 0.7, 3) * np.array(shape)
    M1[((X - c[0]) / (0.25 * nx)) ** 2 + ((Y - c[1]) / (0.2 * ny)) ** 2 + ((Z - c[2]) / (0.2 * nz)) ** 2 < 1] = 4
    n = np.array([[1.0], [1.37], [1.4], [1.37]])  # media 2 and 4 share a refractive index
    return M1, n


def _interface(M1, n):
    ri = n[M1.astype(np.int64) - 1, 0]
    edge = np.zeros(M1.shape, bool)
    for ax in range(3):
        d = np.diff(ri, axis=ax) != 0
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[ax] = slice(0, -1)
        sl_hi[ax] = slice(1, None)
        edge[tuple(sl_lo)] |= d
        edge[tuple(sl_hi)] |= d
    return edge.reshape(-1, order="F")


def _unit(tp):
    th, ph = tp[0].astype(np.float64), tp[1].astype(np.float64)
    return np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])


@pytest.mark.parametrize("shape,d,ls,tol", [((40, 36, 30), (0.0025, 0.0025, 0.0025), 0.0, 1e-5),
                                            ((40, 36, 30), (0.0025, 0.0025, 0.0025), 0.1, 1e-3),
                                            ((24, 20, 16), (0.004, 0.003, 0.005), 0.02, 1e-3)])
def test_device_normals_match_host(shape, d, ls, tol):
    from mcmatlab_b200 import native
    M1, n = _grid(shape, 1)
    host = prep.interface_normals(M1, n, *d, smoothingLengthScale=ls)
    dev = native.interface_normals(M1, n, *d, smoothingLengthScale=ls)
    edge = _interface(M1, n)
    ang = np.arccos(np.clip(np.sum(_unit(host)[:, edge] * _unit(dev)[:, edge], axis=0), -1, 1))
    assert np.max(ang) <= tol, np.max(ang)
