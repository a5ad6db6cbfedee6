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


def band_density(context: Context, hkl, coefficients, occupations, volume: float, support):
    """n(G) at the support keys from band-major coefficients (bands, npw), the
    reference's plane_wave_density_fft arithmetic on the device. A torch CUDA
    complex128 `coefficients` tensor runs the device-memory path and returns a
    CUDA tensor; numpy arrays run the host path and return numpy."""
    lib = C.library()
    keys = np.ascontiguousarray(hkl, dtype=np.int32).reshape(-1, 3)
    sup = np.ascontiguousarray(support, dtype=np.int32).reshape(-1, 3)
    occ = np.ascontiguousarray(occupations, dtype=np.float64).ravel()
    if getattr(coefficients, "is_cuda", False):
        import torch
        psi = coefficients.contiguous()
        if psi.dtype != torch.complex128 or psi.numel() != occ.size * keys.shape[0]:
            raise ValueError("coefficients must be a (bands, npw) complex128 tensor")
        out = torch.empty(sup.shape[0], dtype=torch.complex128, device=psi.device)
        pin, pout, memory = ctypes.c_void_p(psi.data_ptr()), ctypes.c_void_p(out.data_ptr()), C.DEVICE
    else:
        psi = np.ascontiguousarray(coefficients, dtype=np.complex128).reshape(occ.size, keys.shape[0])
        out = np.zeros(sup.shape[0], dtype=np.complex128)
        pin, pout, memory = ctypes.c_void_p(psi.ctypes.data), ctypes.c_void_p(out.ctypes.data), C.HOST
    C.check(lib.sdft_b200_band_density(context.handle, keys.ctypes.data_as(C.I32), keys.shape[0], pin,
                                       occ.ctypes.data_as(C.D), occ.size, float(volume), sup.ctypes.data_as(C.I32),
                                       sup.shape[0], pout, memory))
    return out
