"""Density-side entry points of the C ABI: PBE per point, band density,
one-centre occupations, compensation charge and its adjoint, the Hartree +
XC functionals. Host numpy arrays in, numpy out; all arithmetic on the
device. With torch CUDA tensors the calls are ordered on the context's
stream only: a caller whose tensors come from another stream synchronises
that stream before the call and the context after it (or builds the context
on its torch stream)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from .operator import Context

def fast_length(minimum: int) -> int:
    """Smallest 2/3/5/7-smooth length >= minimum (the density grid rounding)."""
    n = minimum
    while True:
        r = n
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return n
        n += 1


PBE_FIELDS = ("energy_density", "energy_per_particle", "exchange_energy_density", "correlation_energy_density",
              "exchange_potential", "correlation_potential", "gradient_squared_coefficient")


def pbe_points(context: Context, density, gradient):
    """(count, 7) PbeXcPoint fields for densities n > 0 and gradient magnitudes
    |grad n|. numpy in, numpy out (host path); torch CUDA float64 tensors in,
    a CUDA tensor out (device path)."""
    lib = C.library()
    if getattr(density, "is_cuda", False):
        import torch
        n = density.contiguous().view(-1)
        g = gradient.contiguous().view(-1)
        if n.dtype != torch.float64 or g.dtype != torch.float64 or n.numel() != g.numel():
            raise ValueError("density and gradient must be float64 tensors of the same length")
        out = torch.empty((n.numel(), 7), dtype=torch.float64, device=n.device)
        C.check(lib.sdft_b200_pbe_points(context.handle, ctypes.c_void_p(n.data_ptr()), ctypes.c_void_p(g.data_ptr()),
                                         n.numel(), ctypes.c_void_p(out.data_ptr()), C.DEVICE))
        return out
    n = np.ascontiguousarray(density, dtype=np.float64).ravel()
    g = np.ascontiguousarray(gradient, dtype=np.float64).ravel()
    if n.shape != g.shape:
        raise ValueError("density and gradient must have the same length")
    out = np.zeros((n.size, 7))
    C.check(lib.sdft_b200_pbe_points(context.handle, ctypes.c_void_p(n.ctypes.data), ctypes.c_void_p(g.ctypes.data),
                                     n.size, ctypes.c_void_p(out.ctypes.data), C.HOST))
    return out


def density_functionals(context: Context | None, lattice, hkl, density, core_hkl=None, core=None,
                        quadrature_padding: int = 0, support_only: bool = False):
    """Hartree + PBE XC functional of a Fourier density on the device (the
    reference's evaluate_density_functionals). Returns a dict with the union
    support keys `hkl` (lexicographic order), `potential` (Hartree + v_xc),
    `xc_potential` and the DensityFunctionals scalars; with support_only the
    keys alone (host only, context may be None)."""
    lib = C.library()
    lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
    keys = np.ascontiguousarray(hkl, dtype=np.int32).reshape(-1, 3)
    values = np.ascontiguousarray(density, dtype=np.complex128).reshape(-1)
    if values.shape[0] != keys.shape[0]:
        raise ValueError("density keys and values disagree")
    if core_hkl is not None:
        ckeys = np.ascontiguousarray(core_hkl, dtype=np.int32).reshape(-1, 3)
        cvalues = np.ascontiguousarray(core, dtype=np.complex128).reshape(-1)
        if cvalues.shape[0] != ckeys.shape[0]:
            raise ValueError("core keys and values disagree")
    else:
        ckeys = np.zeros((0, 3), dtype=np.int32)
        cvalues = np.zeros(0, dtype=np.complex128)
    handle = context.handle if context is not None else None
    count = ctypes.c_size_t()
    result = C.Functionals()
    args = (lat.ctypes.data_as(C.D), keys.shape[0], keys.ctypes.data_as(C.I32), values.ctypes.data_as(C.D),
            ckeys.shape[0], ckeys.ctypes.data_as(C.I32), cvalues.ctypes.data_as(C.D), int(quadrature_padding))
    C.check(lib.sdft_b200_density_functionals(handle, *args, None, None, None, 0, ctypes.byref(count),
                                              ctypes.byref(result)))
    n = count.value
    if support_only:
        return _support_keys(keys, ckeys)
    support = np.zeros((n, 3), dtype=np.int32)
    potential = np.zeros(n, dtype=np.complex128)
    xc = np.zeros(n, dtype=np.complex128)
    C.check(lib.sdft_b200_density_functionals(handle, *args, support.ctypes.data_as(C.I32),
                                              potential.ctypes.data_as(C.D), xc.ctypes.data_as(C.D), n,
                                              ctypes.byref(count), ctypes.byref(result)))
    out = result.as_dict()
    out.update({"hkl": support, "potential": potential, "xc_potential": xc})
    return out


def collinear_functionals(context: Context | None, lattice, up_hkl, up, down_hkl, down, core_hkl=None, core=None,
                          padding: int = 0, support_only: bool = False):
    """Collinear spin form of the functional on the device (the reference's
    evaluate_collinear_density_functionals): the union support keys `hkl` and
    per channel ("up", "down") a dict with `potential`, `xc_potential` and the
    scalars; with support_only the keys alone (host only, context may be None)."""
    lib = C.library()
    lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
    channels = []
    for keys, values in ((up_hkl, up), (down_hkl, down)):
        k = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3)
        v = np.ascontiguousarray(values, dtype=np.complex128).reshape(-1)
        if v.shape[0] != k.shape[0]:
            raise ValueError("spin density keys and values disagree")
        channels.append((k, v))
    if core_hkl is not None:
        ck = np.ascontiguousarray(core_hkl, dtype=np.int32).reshape(-1, 3)
        cv = np.ascontiguousarray(core, dtype=np.complex128).reshape(-1)
    else:
        ck, cv = np.zeros((0, 3), dtype=np.int32), np.zeros(0, dtype=np.complex128)
    handle = context.handle if context is not None else None
    args = [lat.ctypes.data_as(C.D)]
    for k, v in channels:
        args += [k.shape[0], k.ctypes.data_as(C.I32), v.ctypes.data_as(C.D)]
    args += [ck.shape[0], ck.ctypes.data_as(C.I32), cv.ctypes.data_as(C.D), int(padding)]
    count = ctypes.c_size_t()
    results = (C.Functionals * 2)()
    C.check(lib.sdft_b200_collinear_functionals(handle, *args, None, None, None, None, None, 0, ctypes.byref(count),
                                                results))
    if support_only:
        return _support_keys(np.concatenate([channels[0][0], channels[1][0]]), ck)
    n = count.value
    support = np.zeros((n, 3), dtype=np.int32)
    arrays = [np.zeros(n, dtype=np.complex128) for _ in range(4)]
    C.check(lib.sdft_b200_collinear_functionals(handle, *args, support.ctypes.data_as(C.I32),
                                                *[a.ctypes.data_as(C.D) for a in arrays], n, ctypes.byref(count),
                                                results))
    out = {"hkl": support}
    for c, name in enumerate(("up", "down")):
        channel = results[c].as_dict()
        channel.update({"hkl": support, "potential": arrays[c], "xc_potential": arrays[2 + c]})
        out[name] = channel
    return out


def _support_keys(keys, core_keys) -> np.ndarray:
    """Union of the key sets in lexicographic order (the library's support order)."""
    union = {tuple(int(v) for v in k) for k in keys} | {tuple(int(v) for v in k) for k in core_keys}
    return np.array(sorted(union), dtype=np.int32).reshape(-1, 3)


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


def onsite_density(context: Context, amplitudes, rows: int, occupations) -> np.ndarray:
    """(atoms, rows, rows) one-centre occupations from the all-atom projection
    (atoms*rows, bands), the reference's onsite_density_from_amplitudes per atom."""
    lib = C.library()
    p = np.asfortranarray(amplitudes, dtype=np.complex128)
    occ = np.ascontiguousarray(occupations, dtype=np.float64).ravel()
    total, bands = p.shape
    if total % rows or bands != occ.size:
        raise ValueError("amplitudes must be (atoms*rows, bands) with one occupation per band")
    atoms = total // rows
    out = np.zeros((atoms, rows, rows), dtype=np.complex128)
    C.check(lib.sdft_b200_onsite_density(context.handle, rows, atoms, bands, ctypes.c_void_p(p.ctypes.data), total,
                                         occ.ctypes.data_as(C.D), ctypes.c_void_p(out.ctypes.data), C.HOST))
    return out


class CompensationCharge:
    """Device compensation charge of atoms sharing one augmentation on a
    reciprocal support (the reference's PawCompensationOperator::density_sum)."""

    def __init__(self, context: Context, lattice, fractional, keys, augmentation: dict, transform):
        lib = C.library()
        self._lib = lib
        self.context = context
        lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
        frac = np.ascontiguousarray(fractional, dtype=np.float64).reshape(-1, 3)
        self.keys = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3)
        r = np.ascontiguousarray(augmentation["radial_grid"], dtype=np.float64)
        r2 = np.ascontiguousarray(augmentation["compensation_r2"], dtype=np.float64)
        t = np.ascontiguousarray(transform, dtype=np.complex128)
        self.atoms = frac.shape[0]
        self.dimension = int(round(np.sqrt(t.shape[1])))
        handle = ctypes.c_void_p()
        C.check(lib.sdft_b200_compensation_create(
            context.handle, lat.ctypes.data_as(C.D), self.atoms, frac.ctypes.data_as(C.D),
            self.keys.ctypes.data_as(C.I32), self.keys.shape[0], int(augmentation["max_l"]), r.size,
            r.ctypes.data_as(C.D), r2.ctypes.data_as(C.D), self.dimension, t.view(np.float64).ctypes.data_as(C.D),
            ctypes.byref(handle)))
        self.handle = handle

    def density(self, onsite):
        """onsite: (atoms, dim, dim) numpy (host path) or a torch CUDA tensor (device path)."""
        if getattr(onsite, "is_cuda", False):
            import torch
            rho = onsite.contiguous()
            out = torch.empty(self.keys.shape[0], dtype=torch.complex128, device=rho.device)
            C.check(self._lib.sdft_b200_compensation_density(self.handle, ctypes.c_void_p(rho.data_ptr()),
                                                             ctypes.c_void_p(out.data_ptr()), C.DEVICE))
            return out
        rho = np.ascontiguousarray(onsite, dtype=np.complex128)
        out = np.zeros(self.keys.shape[0], dtype=np.complex128)
        C.check(self._lib.sdft_b200_compensation_density(self.handle, ctypes.c_void_p(rho.ctypes.data),
                                                         ctypes.c_void_p(out.ctypes.data), C.HOST))
        return out

    def project(self, potential):
        """The adjoint (the reference's project_potential_batch): potential on the
        support keys (numpy, host path; or a torch CUDA tensor, device path) ->
        (atoms, dim, dim) projections."""
        shape = (self.atoms, self.dimension, self.dimension)
        if getattr(potential, "is_cuda", False):
            import torch
            v = potential.contiguous()
            out = torch.empty(shape, dtype=torch.complex128, device=v.device)
            C.check(self._lib.sdft_b200_compensation_project(self.handle, ctypes.c_void_p(v.data_ptr()),
                                                             ctypes.c_void_p(out.data_ptr()), C.DEVICE))
            return out
        v = np.ascontiguousarray(potential, dtype=np.complex128).ravel()
        if v.size != self.keys.shape[0]:
            raise ValueError("potential must hold one value per support key")
        out = np.zeros(shape, dtype=np.complex128)
        C.check(self._lib.sdft_b200_compensation_project(self.handle, ctypes.c_void_p(v.ctypes.data),
                                                         ctypes.c_void_p(out.ctypes.data), C.HOST))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self._lib.sdft_b200_compensation_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
