"""Small seeded heat problems on the standard tissue geometry.

Each case returns the MEX-level inputs of finiteElementHeatPropagator: initial T,
initial Omega (or None for no damage), the heatSimParameters dict and the grid size.
"""
from __future__ import annotations

import numpy as np

from mcmatlab_b200 import configs, mexargs, prep


def _base(n, seed, heatSinked, lightsOn, nt, dt_factor, with_damage, hot=False):
    m = configs.standard_tissue_cube(n=n, nPhotons=1e4)
    G = m.G
    media = G.mediaPropertiesFunc([])
    th = prep.thermal_media_properties(media, G.M_raw)
    rng = np.random.default_rng(seed)
    X, Y, Z = np.meshgrid(G.x, G.y, G.z, indexing="ij")
    NA = (200.0 * np.exp(-(X ** 2 + Y ** 2) / 0.02 ** 2 - Z / 0.03) + 5.0 * rng.random((n, n, n)))
    c, Q = prep.calc_dTdt_arrays(th["VHC"], th["TC"], G.dx, G.dy, G.dz, NA, 1.0, th["M"])
    dtmax = prep.calc_dtmax(th["M"], th["TC"], th["VHC"], G.dx, G.dy, G.dz)
    li, w = prep.convert_temp_sensor_pos([[0.0, 0.0, 0.04], [0.01, -0.02, 0.003], [0.049, 0.049, 0.099]], G.x, G.y, G.z)
    hp = mexargs.heat_mex_params(th["M"], th["A"], th["E"], c, Q, True, heatSinked, li, w, lightsOn, nt,
                                 dt_factor * dtmax)
    T0 = (37.0 + rng.random((n, n, n)) * (30.0 if hot else 1.0)).astype(np.float32)
    O0 = (rng.random((n, n, n)) * 1e-3).astype(np.float32) if with_damage else None
    return dict(T0=np.asfortranarray(T0), Omega0=None if O0 is None else np.asfortranarray(O0), hp=hp, n=(n, n, n))


def insulated_on():
    return _base(20, 1, 0, True, 30, 0.9, True)


def sinked_off():
    return _base(18, 2, 1, False, 25, 1.5, True)


def hot_damage():
    return _base(16, 3, 0, True, 20, 0.9, True, hot=True)


def no_damage_single_step():
    return _base(22, 4, 0, True, 1, 0.9, False)


CASES = {
    "insulated_on": insulated_on,
    "sinked_off": sinked_off,
    "hot_damage": hot_damage,
    "no_damage_single_step": no_damage_single_step,
}


def shaped(shape, seed=5, heatSinked=0, lightsOn=True, nt=12, dt_factor=0.9, with_damage=True, size=(1.0, 1.0, 0.6)):
    """A seeded 4-medium box of any shape (bulk, top layer, deep layer, ellipsoidal target with
    Arrhenius damage; configs.heat_adjoint_case) with a non-uniform initial temperature, an initial
    damage field and three temperature sensors: exercises every line-length class of the stepper."""
    nx, ny, nz = shape
    c = configs.heat_adjoint_case(shape=shape, size=size, nt=nt, seed=seed, dtFactor=dt_factor, heatBoundaryType=heatSinked)
    hp = dict(c["hp"])
    dx, dy, dz = c["d"]
    x = (np.arange(nx) + 0.5) * dx - size[0] / 2
    y = (np.arange(ny) + 0.5) * dy - size[1] / 2
    z = (np.arange(nz) + 0.5) * dz
    li, w = prep.convert_temp_sensor_pos([[0.0, 0.0, 0.5 * size[2]], [0.21 * size[0], -0.13 * size[1], 0.11 * size[2]],
                                          [-0.4 * size[0], 0.37 * size[1], 0.83 * size[2]]], x, y, z)
    hp = mexargs.heat_mex_params(c["M1"], hp["A"], hp["E"], hp["dTdtperdeltaT"], hp["dTdt_abs"], True, heatSinked, li, w,
                                 lightsOn, nt, hp["dt"])
    rng = np.random.default_rng(seed + 100)
    # hot enough (50-60 degC) that the Arrhenius damage of a few steps is well above FP32 rounding
    T0 = (50.0 + 10.0 * rng.random(shape)).astype(np.float32)
    O0 = (rng.random(shape) * 1e-3).astype(np.float32) if with_damage else None
    return dict(T0=np.asfortranarray(T0), Omega0=None if O0 is None else np.asfortranarray(O0), hp=hp, n=tuple(shape))
