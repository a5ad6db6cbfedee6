"""ctypes access to the reference's own CPU implementation (oracle/_ref/libsdft_ref.so).

TEST INFRASTRUCTURE ONLY. This module is the checker: only tests/, the smoke
check in __graft_entry__ and bench.py's CPU-baseline leg may import it. The
library is the reference's unmodified src/*.cpp compiled by oracle/ref/Makefile
against this project's FFTW3-API shim and the OpenBLAS found in the image.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIBRARY = HERE / "_ref" / "libsdft_ref.so"
REPLAY = HERE / "_ref" / "sdft_solver_replay"

_dbl = ctypes.POINTER(ctypes.c_double)
_int = ctypes.POINTER(ctypes.c_int)
_long = ctypes.POINTER(ctypes.c_long)


def available() -> bool:
    return LIBRARY.exists()


def _ptr(array, kind=_dbl):
    return array.ctypes.data_as(kind)


class ReferenceLibrary:
    def __init__(self, path: pathlib.Path = LIBRARY):
        if not path.exists():
            raise FileNotFoundError(f"reference oracle library not built: {path} (make -C oracle/ref)")
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        L.ref_enumerate_g_vectors.restype = ctypes.c_long
        L.ref_enumerate_g_vectors.argtypes = [_dbl, ctypes.c_double, _dbl, ctypes.c_double, _int, _dbl, _dbl,
                                              ctypes.c_long]
        L.ref_operator_create.restype = ctypes.c_void_p
        L.ref_operator_create.argtypes = [ctypes.c_long, _int, _dbl, _dbl, ctypes.c_long, _int, _dbl,
                                          ctypes.c_long, _long, _dbl, _dbl, _dbl, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_ulonglong, ctypes.c_char_p, ctypes.c_long]
        L.ref_operator_destroy.argtypes = [ctypes.c_void_p]
        L.ref_operator_grid.restype = ctypes.c_long
        L.ref_operator_grid.argtypes = [ctypes.c_void_p]
        L.ref_apply.restype = ctypes.c_int
        L.ref_apply.argtypes = [ctypes.c_void_p, ctypes.c_int, _dbl, ctypes.c_long, _dbl, ctypes.c_int,
                                ctypes.c_char_p, ctypes.c_long]
        L.ref_apply_pair.restype = ctypes.c_int
        L.ref_apply_pair.argtypes = [ctypes.c_void_p, _dbl, ctypes.c_long, _dbl, _dbl, ctypes.c_int,
                                     ctypes.c_char_p, ctypes.c_long]
        L.ref_project.restype = ctypes.c_int
        L.ref_project.argtypes = [ctypes.c_void_p, _dbl, ctypes.c_long, _dbl, ctypes.c_char_p, ctypes.c_long]
        L.ref_projector_rows.restype = ctypes.c_long
        L.ref_projector_rows.argtypes = [ctypes.c_void_p]
        L.ref_overlap_signature.restype = ctypes.c_int
        L.ref_overlap_signature.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_char_p,
                                            ctypes.c_long]
        L.ref_davidson.restype = ctypes.c_int
        L.ref_davidson.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_double, _dbl, _dbl, _dbl,
                                   _dbl, _int, _long, ctypes.c_char_p, ctypes.c_long]
        L.ref_rmm_trial.restype = ctypes.c_int
        L.ref_rmm_trial.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_double, _dbl, _dbl, _dbl,
                                    _dbl, ctypes.POINTER(ctypes.c_int), _long, ctypes.POINTER(ctypes.c_int),
                                    ctypes.c_char_p, ctypes.c_long]
        L.ref_band_groups.restype = ctypes.c_int
        L.ref_band_groups.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_double, _dbl, _dbl,
                                      _dbl, _dbl, ctypes.POINTER(ctypes.c_int), _long, ctypes.c_char_p,
                                      ctypes.c_long]
        L.ref_kinetic_preconditioner.restype = ctypes.c_double
        L.ref_kinetic_preconditioner.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_save_snapshot.restype = ctypes.c_int
        L.ref_save_snapshot.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_long, ctypes.c_long,
                                        ctypes.c_double, _dbl, ctypes.c_long, ctypes.c_char_p, ctypes.c_long]
        L.ref_load_snapshot.restype = ctypes.c_void_p
        L.ref_load_snapshot.argtypes = [ctypes.c_char_p, _long, _long, _dbl, ctypes.c_char_p, ctypes.c_long]
        L.ref_plane_wave_density_fft.restype = ctypes.c_int
        L.ref_plane_wave_density_fft.argtypes = [ctypes.c_long, _int, ctypes.c_long, _dbl, _dbl, ctypes.c_double,
                                                 ctypes.c_long, _int, _dbl, ctypes.c_char_p, ctypes.c_long]
        L.ref_pbe_collinear.restype = ctypes.c_int
        L.ref_pbe_collinear.argtypes = [ctypes.c_long, _dbl, _dbl, _dbl, _dbl, _dbl, ctypes.c_char_p, ctypes.c_long]
        L.ref_pbe_unpolarized.restype = None
        L.ref_pbe_unpolarized.argtypes = [ctypes.c_long, _dbl, _dbl, _dbl]
        L.ref_refresh_environment.restype = None
        L.ref_onsite_density.restype = ctypes.c_int
        L.ref_onsite_density.argtypes = [ctypes.c_long, ctypes.c_long, _dbl, ctypes.c_long, _dbl, _dbl,
                                         ctypes.c_char_p, ctypes.c_long]
        L.ref_lm_transform.restype = ctypes.c_int
        L.ref_lm_transform.argtypes = [ctypes.c_long, _int, ctypes.c_int, ctypes.c_long, _dbl, _dbl, _dbl, _dbl,
                                       ctypes.c_char_p, ctypes.c_long]
        L.ref_compensation_density.restype = ctypes.c_int
        L.ref_compensation_density.argtypes = [_dbl, ctypes.c_long, _dbl, ctypes.c_long, _int, ctypes.c_long, _int,
                                               ctypes.c_int, ctypes.c_long, _dbl, _dbl, _dbl, _dbl, _dbl,
                                               ctypes.c_char_p, ctypes.c_long]
        L.ref_compensation_project.restype = ctypes.c_int
        L.ref_compensation_project.argtypes = [_dbl, ctypes.c_long, _dbl, ctypes.c_long, _int, ctypes.c_long, _int,
                                               ctypes.c_int, ctypes.c_long, _dbl, _dbl, _dbl, ctypes.c_long, _int,
                                               _dbl, _dbl, ctypes.c_char_p, ctypes.c_long]
        L.ref_collinear_functionals.restype = ctypes.c_long
        L.ref_collinear_functionals.argtypes = [_dbl, ctypes.c_long, _int, _dbl, ctypes.c_long, _int, _dbl,
                                                ctypes.c_long, _int, _dbl, ctypes.c_int, ctypes.c_long, _int, _dbl,
                                                _dbl, _dbl, ctypes.c_char_p, ctypes.c_long]
        L.ref_density_functionals.restype = ctypes.c_long
        L.ref_density_functionals.argtypes = [_dbl, ctypes.c_long, _int, _dbl, ctypes.c_long, _int, _dbl,
                                              ctypes.c_int, ctypes.c_long, _int, _dbl, _dbl, _dbl, ctypes.c_char_p,
                                              ctypes.c_long]

    # -- basis ---------------------------------------------------------------
    def enumerate_g_vectors(self, reciprocal, cutoff_ev, kpoint=(0.0, 0.0, 0.0), hartree_to_ev=27.211386245988):
        recip = np.ascontiguousarray(reciprocal, dtype=np.float64).reshape(9)
        k = np.ascontiguousarray(kpoint, dtype=np.float64)
        dummy_i = np.zeros(3, dtype=np.int32)
        dummy_d = np.zeros(3)
        n = self.lib.ref_enumerate_g_vectors(_ptr(recip), cutoff_ev, _ptr(k), hartree_to_ev, _ptr(dummy_i, _int),
                                             _ptr(dummy_d), _ptr(dummy_d), 0)
        hkl = np.zeros((n, 3), dtype=np.int32)
        cart = np.zeros((n, 3))
        kin = np.zeros(n)
        self.lib.ref_enumerate_g_vectors(_ptr(recip), cutoff_ev, _ptr(k), hartree_to_ev, _ptr(hkl, _int),
                                         _ptr(cart), _ptr(kin), n)
        return hkl, cart, kin

    def kinetic_preconditioner(self, kinetic, wavefunction_kinetic):
        return self.lib.ref_kinetic_preconditioner(kinetic, wavefunction_kinetic)

    def pbe(self, density, gradient):
        n = np.ascontiguousarray(density, dtype=np.float64)
        g = np.ascontiguousarray(gradient, dtype=np.float64)
        out = np.zeros((n.size, 7))
        self.lib.ref_pbe_unpolarized(n.size, _ptr(n), _ptr(g), _ptr(out))
        return out

    def pbe_collinear(self, up, down, gradient_up, gradient_down):
        """(count, 9): energy density, v_up, v_down, gradient responses up (3) and down (3)."""
        u = np.ascontiguousarray(up, dtype=np.float64)
        d = np.ascontiguousarray(down, dtype=np.float64)
        gu = np.ascontiguousarray(gradient_up, dtype=np.float64).reshape(-1, 3)
        gd = np.ascontiguousarray(gradient_down, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((u.size, 9))
        err = ctypes.create_string_buffer(512)
        self._check(self.lib.ref_pbe_collinear(u.size, _ptr(u), _ptr(d), _ptr(gu), _ptr(gd), _ptr(out), err, 512),
                    err)
        return out

    @staticmethod
    def _check(rc, err):
        if rc:
            raise RuntimeError(err.value.decode())

    def onsite_density(self, amplitudes, occupations):
        """rho_ij of one atom from amplitudes (rows, bands) (src/onsite_density.hpp:13)."""
        p = np.asfortranarray(amplitudes, dtype=np.complex128)
        occ = np.ascontiguousarray(occupations, dtype=np.float64)
        out = np.zeros((p.shape[0], p.shape[0]), dtype=np.complex128)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_onsite_density(p.shape[0], p.shape[1], p.ravel(order="F").view(np.float64).ctypes.data_as(_dbl),
                                         p.shape[0], _ptr(occ), out.view(np.float64).ctypes.data_as(_dbl), err, 512)
        self._check(rc, err)
        return out

    @staticmethod
    def _augmentation(aug):
        return (np.ascontiguousarray(aug["channel_l"], dtype=np.int32), int(aug["max_l"]),
                np.ascontiguousarray(aug["radial_grid"], dtype=np.float64),
                np.ascontiguousarray(aug["aug_moment"], dtype=np.float64),
                np.ascontiguousarray(aug["compensation_r2"], dtype=np.float64))

    def lm_transform(self, aug):
        """[lm, i*dim+j] moments of unit occupations (src/paw_augmentation.cpp:490; src/paw_compensation.cpp:228-236)."""
        ch, max_l, r, mom, r2 = self._augmentation(aug)
        dim = int(np.sum(2 * ch + 1))
        out = np.zeros(((max_l + 1) ** 2, dim * dim), dtype=np.complex128)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_lm_transform(ch.size, _ptr(ch, _int), max_l, r.size, _ptr(r), _ptr(mom), _ptr(r2),
                                       out.view(np.float64).ctypes.data_as(_dbl), err, 512)
        self._check(rc, err)
        return out

    def compensation_density(self, lattice, fractional, keys, aug, onsite):
        """PawCompensationOperator::density_sum over atoms sharing one geometry (src/paw_compensation.cpp:465)."""
        ch, max_l, r, mom, r2 = self._augmentation(aug)
        lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
        frac = np.ascontiguousarray(fractional, dtype=np.float64).reshape(-1, 3)
        k = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3)
        rho = np.ascontiguousarray(onsite, dtype=np.complex128)
        out = np.zeros(k.shape[0], dtype=np.complex128)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_compensation_density(_ptr(lat), frac.shape[0], _ptr(frac), k.shape[0], _ptr(k, _int),
                                               ch.size, _ptr(ch, _int), max_l, r.size, _ptr(r), _ptr(mom), _ptr(r2),
                                               rho.view(np.float64).ctypes.data_as(_dbl),
                                               out.view(np.float64).ctypes.data_as(_dbl), err, 512)
        self._check(rc, err)
        return out

    def compensation_project(self, lattice, fractional, keys, aug, potential_keys, potential):
        """PawCompensationOperator::project_potential_batch (src/paw_compensation.cpp:552):
        (atoms, dim, dim) projections of the potential given on potential_keys."""
        ch, max_l, r, mom, r2 = self._augmentation(aug)
        lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
        frac = np.ascontiguousarray(fractional, dtype=np.float64).reshape(-1, 3)
        k = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3)
        pk = np.ascontiguousarray(potential_keys, dtype=np.int32).reshape(-1, 3)
        pv = np.ascontiguousarray(potential, dtype=np.complex128)
        dim = int(np.sum(2 * np.asarray(aug["channel_l"]) + 1))
        out = np.zeros((frac.shape[0], dim, dim), dtype=np.complex128)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_compensation_project(_ptr(lat), frac.shape[0], _ptr(frac), k.shape[0], _ptr(k, _int),
                                               ch.size, _ptr(ch, _int), max_l, r.size, _ptr(r), _ptr(mom), _ptr(r2),
                                               pk.shape[0], _ptr(pk, _int), pv.view(np.float64).ctypes.data_as(_dbl),
                                               out.view(np.float64).ctypes.data_as(_dbl), err, 512)
        self._check(rc, err)
        return out

    def density_functionals(self, lattice, keys, values, core_keys=None, core_values=None, padding: int = 0):
        """evaluate_density_functionals (src/density_functionals.cpp:696-729): the
        potential's keys in map order, potential, xc_potential and the scalars."""
        lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
        k = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3)
        v = np.ascontiguousarray(values, dtype=np.complex128).reshape(-1)
        if core_keys is None:
            ck, cv = np.zeros((0, 3), dtype=np.int32), np.zeros(0, dtype=np.complex128)
        else:
            ck = np.ascontiguousarray(core_keys, dtype=np.int32).reshape(-1, 3)
            cv = np.ascontiguousarray(core_values, dtype=np.complex128).reshape(-1)
        err = ctypes.create_string_buffer(512)
        scalars = np.zeros(25)
        args = (_ptr(lat), k.shape[0], _ptr(k, _int), v.view(np.float64).ctypes.data_as(_dbl), ck.shape[0],
                _ptr(ck, _int), cv.view(np.float64).ctypes.data_as(_dbl), int(padding))
        size = self.lib.ref_density_functionals(*args, 0, None, None, None, _ptr(scalars), err, 512)
        if size < 0:
            raise ValueError(err.value.decode(errors="replace"))
        out_keys = np.zeros((size, 3), dtype=np.int32)
        potential = np.zeros(size, dtype=np.complex128)
        xc = np.zeros(size, dtype=np.complex128)
        size = self.lib.ref_density_functionals(*args, size, _ptr(out_keys, _int),
                                                potential.view(np.float64).ctypes.data_as(_dbl),
                                                xc.view(np.float64).ctypes.data_as(_dbl), _ptr(scalars), err, 512)
        if size < 0:
            raise ValueError(err.value.decode(errors="replace"))
        names = ("hartree_energy", "xc_energy", "vxc_density", "sampled_electrons", "minimum_density",
                 "clipped_density_points", "grid_points")
        out = {name: float(scalars[i]) for i, name in enumerate(names)}
        out["clipped_density_points"] = int(out["clipped_density_points"])
        out["grid_points"] = int(out["grid_points"])
        out["hartree_stress"] = scalars[7:16].reshape(3, 3).copy()
        out["xc_stress"] = scalars[16:25].reshape(3, 3).copy()
        out.update({"hkl": out_keys, "potential": potential, "xc_potential": xc})
        return out

    def collinear_functionals(self, lattice, up_keys, up, down_keys, down, core_keys=None, core=None,
                              padding: int = 0):
        """evaluate_collinear_density_functionals (src/density_functionals.cpp:732-806):
        {"hkl", "up": {...}, "down": {...}} with each channel's potential, xc_potential and scalars."""
        lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
        arrays = []
        for keys, values in ((up_keys, up), (down_keys, down),
                             (core_keys if core_keys is not None else np.zeros((0, 3)),
                              core if core is not None else np.zeros(0))):
            arrays.append((np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3),
                           np.ascontiguousarray(values, dtype=np.complex128).reshape(-1)))
        args = [_ptr(lat)]
        for k, v in arrays:
            args += [k.shape[0], _ptr(k, _int), v.view(np.float64).ctypes.data_as(_dbl)]
        args.append(int(padding))
        err = ctypes.create_string_buffer(512)
        scalars = np.zeros(50)
        size = self.lib.ref_collinear_functionals(*args, 0, None, None, None, _ptr(scalars), err, 512)
        if size < 0:
            raise ValueError(err.value.decode(errors="replace"))
        keys = np.zeros((size, 3), dtype=np.int32)
        potential = np.zeros(2 * size, dtype=np.complex128)
        xc = np.zeros(2 * size, dtype=np.complex128)
        size = self.lib.ref_collinear_functionals(*args, size, _ptr(keys, _int),
                                                  potential.view(np.float64).ctypes.data_as(_dbl),
                                                  xc.view(np.float64).ctypes.data_as(_dbl), _ptr(scalars), err, 512)
        if size < 0:
            raise ValueError(err.value.decode(errors="replace"))
        names = ("hartree_energy", "xc_energy", "vxc_density", "sampled_electrons", "minimum_density",
                 "clipped_density_points", "grid_points")
        out = {"hkl": keys}
        for s, channel in enumerate(("up", "down")):
            o = scalars[25 * s:25 * (s + 1)]
            r = {name: float(o[i]) for i, name in enumerate(names)}
            r["clipped_density_points"] = int(r["clipped_density_points"])
            r["grid_points"] = int(r["grid_points"])
            r["hartree_stress"] = o[7:16].reshape(3, 3).copy()
            r["xc_stress"] = o[16:25].reshape(3, 3).copy()
            r.update({"hkl": keys, "potential": potential[s * size:(s + 1) * size],
                      "xc_potential": xc[s * size:(s + 1) * size]})
            out[channel] = r
        return out

    def density(self, hkl, coefficients, occupations, volume, support_hkl):
        hkl = np.ascontiguousarray(hkl, dtype=np.int32)
        coeff = np.ascontiguousarray(coefficients, dtype=np.complex128)  # (bands, n) band-major
        occ = np.ascontiguousarray(occupations, dtype=np.float64)
        sup = np.ascontiguousarray(support_hkl, dtype=np.int32)
        out = np.zeros(sup.shape[0], dtype=np.complex128)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_plane_wave_density_fft(hkl.shape[0], _ptr(hkl, _int), occ.size,
                                                 coeff.view(np.float64).ctypes.data_as(_dbl), _ptr(occ), volume,
                                                 sup.shape[0], _ptr(sup, _int), out.view(np.float64).ctypes.data_as(_dbl),
                                                 err, 512)
        if rc:
            raise RuntimeError(err.value.decode())
        return out


class ReferenceOperator:
    """The reference's PlaneWaveOperator built from synthetic OperatorInputs."""

    def __init__(self, lib: ReferenceLibrary, inputs=None, handle=None, projector_identity: int = 0):
        self.lib = lib
        if handle is not None:
            self.handle = handle
            return
        x = inputs
        hkl = np.ascontiguousarray(x.hkl, dtype=np.int32)
        cart = np.ascontiguousarray(x.cartesian, dtype=np.float64)
        kin = np.ascontiguousarray(x.kinetic_ev, dtype=np.float64)
        vh = np.ascontiguousarray(x.v_hkl, dtype=np.int32)
        vv = np.ascontiguousarray(x.v_values, dtype=np.complex128)
        proj = np.ascontiguousarray(x.projectors, dtype=np.int64)
        amp = np.ascontiguousarray(x.amplitudes, dtype=np.complex128)
        d = np.ascontiguousarray(x.d, dtype=np.complex128)
        q = np.ascontiguousarray(x.q, dtype=np.complex128)
        self._keep = (hkl, cart, kin, vh, vv, proj, amp, d, q)
        err = ctypes.create_string_buffer(1024)
        self.handle = lib.lib.ref_operator_create(
            hkl.shape[0], _ptr(hkl, _int), _ptr(cart), _ptr(kin), vh.shape[0], _ptr(vh, _int),
            vv.view(np.float64).ctypes.data_as(_dbl), proj.size, _ptr(proj, _long),
            amp.view(np.float64).ctypes.data_as(_dbl), d.view(np.float64).ctypes.data_as(_dbl),
            q.view(np.float64).ctypes.data_as(_dbl), x.hartree_to_ev, x.regularization, projector_identity, err, 1024)
        if not self.handle:
            raise ValueError(err.value.decode())
        self.n = hkl.shape[0]

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.lib.ref_operator_destroy(self.handle)
            self.handle = None

    @property
    def grid_points(self) -> int:
        return self.lib.lib.ref_operator_grid(self.handle)

    def _call(self, fn, *args):
        err = ctypes.create_string_buffer(1024)
        rc = fn(*args, err, 1024)
        if rc:
            raise RuntimeError(err.value.decode())

    def apply(self, x, overlap=False, exact=True):
        """x: (n, cols) complex128 -> H~x or S~x, column-major blocks."""
        xf = np.asfortranarray(x, dtype=np.complex128)
        cols = xf.shape[1]
        y = np.zeros_like(xf, order="F")
        self._call(self.lib.lib.ref_apply, self.handle, int(overlap), xf.ctypes.data_as(_dbl), cols,
                   y.ctypes.data_as(_dbl), int(exact))
        return y

    def apply_pair(self, x, exact=True):
        xf = np.asfortranarray(x, dtype=np.complex128)
        cols = xf.shape[1]
        hy = np.zeros_like(xf, order="F")
        sy = np.zeros_like(xf, order="F")
        self._call(self.lib.lib.ref_apply_pair, self.handle, xf.ctypes.data_as(_dbl), cols, hy.ctypes.data_as(_dbl),
                   sy.ctypes.data_as(_dbl), int(exact))
        return hy, sy

    def project(self, x):
        xf = np.asfortranarray(x, dtype=np.complex128)
        rows = self.lib.lib.ref_projector_rows(self.handle)
        p = np.zeros((rows, xf.shape[1]), dtype=np.complex128, order="F")
        self._call(self.lib.lib.ref_project, self.handle, xf.ctypes.data_as(_dbl), xf.shape[1], p.ctypes.data_as(_dbl))
        return p

    def overlap_signature(self):
        """overlap()'s signature decision: {'indefinite': bool}; a numerically
        singular S~ raises RuntimeError with the reference's message."""
        flag = ctypes.c_int(0)
        self._call(self.lib.lib.ref_overlap_signature, self.handle, ctypes.byref(flag))
        return {"indefinite": bool(flag.value)}

    def davidson(self, roots, max_iterations=256, tolerance=1e-12, initial=None):
        eig = np.zeros(roots)
        res = np.zeros(roots)
        vec = np.zeros((roots, self.n), dtype=np.complex128)  # band-major
        conv = ctypes.c_int(0)
        iters = ctypes.c_long(0)
        init = None
        if initial is not None:
            init = np.ascontiguousarray(initial, dtype=np.complex128)
        self._call(self.lib.lib.ref_davidson, self.handle, roots, max_iterations, tolerance,
                   init.ctypes.data_as(_dbl) if init is not None else None, _ptr(eig), vec.ctypes.data_as(_dbl),
                   _ptr(res), ctypes.byref(conv), ctypes.byref(iters))
        return {"eigenvalues": eig, "eigenvectors": vec, "residuals": res, "converged": bool(conv.value),
                "iterations": int(iters.value)}

    def band_groups(self, roots, max_iterations=256, tolerance=1e-10, initial=None):
        """solve_generalized_hermitian_band_groups (src/band_group_solver.cpp:55-212)."""
        eig = np.zeros(roots)
        res = np.zeros(roots)
        vec = np.zeros((roots, self.n), dtype=np.complex128)
        conv, iters = ctypes.c_int(0), ctypes.c_long(0)
        init = None if initial is None else np.ascontiguousarray(initial, dtype=np.complex128)
        self._call(self.lib.lib.ref_band_groups, self.handle, roots, max_iterations, tolerance,
                   init.ctypes.data_as(_dbl) if init is not None else None, _ptr(eig), vec.ctypes.data_as(_dbl),
                   _ptr(res), ctypes.byref(conv), ctypes.byref(iters))
        return {"eigenvalues": eig, "eigenvectors": vec, "residuals": res, "converged": bool(conv.value),
                "iterations": int(iters.value)}

    def rmm_trial(self, roots, initial, max_iterations=256, tolerance=1e-6):
        """solve_generalized_hermitian_rmm_trial as an SCF warm request."""
        eig = np.zeros(roots)
        res = np.zeros(roots)
        vec = np.zeros((roots, self.n), dtype=np.complex128)
        conv, manifold, iters = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_long(0)
        init = np.ascontiguousarray(initial, dtype=np.complex128)
        self._call(self.lib.lib.ref_rmm_trial, self.handle, roots, max_iterations, tolerance,
                   init.ctypes.data_as(_dbl), _ptr(eig), vec.ctypes.data_as(_dbl), _ptr(res), ctypes.byref(conv),
                   ctypes.byref(iters), ctypes.byref(manifold))
        return {"eigenvalues": eig, "eigenvectors": vec, "residuals": res, "converged": bool(conv.value),
                "iterations": int(iters.value), "trial_manifold": bool(manifold.value)}

    @classmethod
    def from_snapshot(cls, lib: ReferenceLibrary, path):
        """The reference's PlaneWaveOperator::load_solver_snapshot; the warm
        vectors are read from the file (the driver does not return them)."""
        import pathlib
        import struct
        raw = pathlib.Path(path).read_bytes()
        n, roots_h = struct.unpack_from("<Q", raw, 8)[0], struct.unpack_from("<Q", raw, 56)[0]
        warm = struct.unpack_from("<Q", raw, 72)[0]
        roots, iterations, tolerance = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        err = ctypes.create_string_buffer(1024)
        handle = lib.lib.ref_load_snapshot(str(path).encode(), ctypes.byref(roots), ctypes.byref(iterations),
                                           ctypes.byref(tolerance), err, 1024)
        if not handle:
            raise RuntimeError(err.value.decode(errors="replace"))
        op = cls(lib, handle=handle)
        op.n = int(n)
        initial = None
        if warm:
            initial = np.frombuffer(raw, dtype="<c16", count=warm, offset=len(raw) - 16 * warm).reshape(roots_h, n).copy()
        return {"operator": op, "roots": roots.value, "iterations": iterations.value, "tolerance": tolerance.value,
                "initial": initial}

    def save_snapshot(self, path, roots, iterations, tolerance, initial=None):
        init = np.ascontiguousarray(initial if initial is not None else np.zeros(0), dtype=np.complex128)
        self._call(self.lib.lib.ref_save_snapshot, self.handle, str(path).encode(), roots, iterations, tolerance,
                   init.ctypes.data_as(_dbl), init.size)
