"""The gradient smoothing of the interface normals restates smoothn's fixed-smoothness path
(+MCmatlab/@model/private/smoothn.m:348-469 with no weights and no robust step): it must equal
the penalised least-squares solution z = (I + s L^2)^-1 y, where L is the Kronecker sum of the
per-axis second-difference matrices with reflective ends, scaled by 1 / h_i^2."""
import numpy as np

from mcmatlab_b200 import prep


def _second_difference(n):
    D = np.zeros((n, n))
    for i in range(n):
        if i > 0:
            D[i, i - 1] = 1.0
            D[i, i] -= 1.0
        if i < n - 1:
            D[i, i + 1] = 1.0
            D[i, i] -= 1.0
    return D


def test_smoothing_is_the_penalised_least_squares_solution():
    shape = (5, 4, 6)
    spacing = np.array([0.002, 0.001, 0.0015])
    h = spacing / spacing.max()
    s = 7.0
    rng = np.random.default_rng(3)
    y = rng.standard_normal(shape)
    # column-major-free construction: axis 0 is the slowest index of a C-order flattening
    L = np.zeros((y.size, y.size))
    for ax, n in enumerate(shape):
        mats = [np.eye(m) for m in shape]
        mats[ax] = _second_difference(n) / h[ax] ** 2
        K = mats[0]
        for m in mats[1:]:
            K = np.kron(K, m)
        L += K
    z_ref = np.linalg.solve(np.eye(y.size) + s * L @ L, y.reshape(-1)).reshape(shape)
    z = prep.smooth_gradients([y], s, spacing)[0]
    assert np.max(np.abs(z - z_ref)) <= 1e-10 * np.max(np.abs(z_ref))


def test_normals_of_a_flat_interface_stay_normal_after_smoothing():
    M1 = np.ones((12, 10, 8), dtype=np.uint8)
    M1[:, :, 4:] = 2
    n = np.array([[1.0], [1.4]])
    tp = prep.interface_normals(M1, n, 0.01, 0.01, 0.01, smoothingLengthScale=0.05)
    theta = tp[0].reshape(M1.shape, order="F")
    # at the interface the smoothed gradient still points along z (theta = 0 or pi)
    assert np.allclose(np.sin(theta[3:9, 3:7, 3:5]), 0, atol=1e-6)
