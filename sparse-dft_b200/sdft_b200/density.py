"""Density-side entry points of the C ABI: PBE per point, band density,
one-centre occupations. Host numpy arrays in, numpy out; all arithmetic on
the device."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from .operator import Context

PBE_FIELDS = ("energy_density", "energy_per_particle", "exchange_energy_density", "correlation_energy_density",
              "exchange_potential", "correlation_potential", "gradient_squared_coefficient")


def pbe_points(context: Context, density, gradient) -> np.ndarray:
    """(count, 7) PbeXcPoint fields for densities n > 0 and gradient magnitudes |grad n|."""
    lib = C.library()
    n = np.ascontiguousarray(density, dtype=np.float64).ravel()
    g = np.ascontiguousarray(gradient, dtype=np.float64).ravel()
    if n.shape != g.shape:
        raise ValueError("density and gradient must have the same length")
    out = np.zeros((n.size, 7))
    C.check(lib.sdft_b200_pbe_points(context.handle, ctypes.c_void_p(n.ctypes.data), ctypes.c_void_p(g.ctypes.data),
                                     n.size, ctypes.c_void_p(out.ctypes.data), C.HOST))
    return out
