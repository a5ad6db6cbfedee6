"""ctypes binding of the C ABI in include/sdft_b200.h (libsdft_b200.so, built in-tree).

There is no Python or CPU implementation behind this module: if the shared
library is missing, importing the bindings raises immediately.
"""
from __future__ import annotations

import ctypes
import pathlib
import re

import numpy as np

LIBRARY = pathlib.Path(__file__).resolve().parent / "_lib" / "libsdft_b200.so"
HEADER = pathlib.Path(__file__).resolve().parents[2] / "include" / "sdft_b200.h"

OK, INVALID_ARGUMENT, OVERFLOW, RUNTIME_ERROR, CUDA_ERROR, OUT_OF_MEMORY, NONFINITE, NOT_READY, UNSUPPORTED = range(9)
FP64, MIXED = 0, 1
HOST, DEVICE = 0, 1
HAMILTONIAN, OVERLAP = 0, 1


class SdftError(RuntimeError):
    """A non-OK status from the library; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


class InvalidArgument(SdftError, ValueError):
    pass


class OverflowFailure(SdftError, OverflowError):
    pass


class Unsupported(SdftError):
    """The reference routes this case to a solver the library does not provide."""


_ERRORS = {INVALID_ARGUMENT: InvalidArgument, OVERFLOW: OverflowFailure, UNSUPPORTED: Unsupported}

_lib = None


def library() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise ImportError(f"libsdft_b200.so is not built ({LIBRARY}); run __graft_entry__.build() or "
                              "make -C sparse-dft_b200")
        _lib = ctypes.CDLL(str(LIBRARY))
        _declare(_lib)
    return _lib


def declared_symbols() -> list[str]:
    """Every function the public header declares."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"SDFT_B200_API\s+[\w\s\*]*?\b(sdft_b200_\w+)\s*\(", text)))


P = ctypes.c_void_p
D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int32)
U64 = ctypes.POINTER(ctypes.c_uint64)
SZ = ctypes.c_size_t
SZP = ctypes.POINTER(ctypes.c_size_t)


class SnapshotInfo(ctypes.Structure):
    _fields_ = [("npw", ctypes.c_size_t), ("grid_points", ctypes.c_size_t), ("projectors", ctypes.c_size_t),
                ("atoms", ctypes.c_size_t), ("roots", ctypes.c_size_t), ("iterations", ctypes.c_size_t),
                ("initial_values", ctypes.c_size_t), ("shape", ctypes.c_int32 * 3), ("regularization", ctypes.c_double),
                ("tolerance", ctypes.c_double)]

    def as_dict(self) -> dict:
        out = {name: getattr(self, name) for name, _ in self._fields_}
        out["shape"] = tuple(int(v) for v in self.shape)
        return out


class Functionals(ctypes.Structure):
    _fields_ = [("hartree_energy", ctypes.c_double), ("xc_energy", ctypes.c_double), ("vxc_density", ctypes.c_double),
                ("hartree_stress", ctypes.c_double * 9), ("xc_stress", ctypes.c_double * 9),
                ("sampled_electrons", ctypes.c_double), ("minimum_density", ctypes.c_double),
                ("clipped_density_points", ctypes.c_uint64), ("grid_points", ctypes.c_uint64),
                ("grid", ctypes.c_int32 * 3)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            value = getattr(self, name)
            if name.endswith("stress"):
                value = np.array(list(value)).reshape(3, 3)
            elif name == "grid":
                value = tuple(int(v) for v in value)
            out[name] = value
        return out


class SolveTiming(ctypes.Structure):
    _fields_ = [("slot", ctypes.c_int), ("footprint", ctypes.c_size_t), ("submitted", ctypes.c_double),
                ("started", ctypes.c_double), ("finished", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class DavidsonOptions(ctypes.Structure):
    _fields_ = [("roots", ctypes.c_size_t), ("max_iterations", ctypes.c_size_t), ("tolerance", ctypes.c_double),
                ("precision", ctypes.c_int), ("subspace_factor", ctypes.c_int), ("handoff", ctypes.c_double),
                ("correction_steps", ctypes.c_int)]


class DavidsonStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_size_t), ("converged", ctypes.c_int), ("max_residual", ctypes.c_double),
                ("seconds", ctypes.c_double), ("rayleigh_ritz_seconds", ctypes.c_double),
                ("h_columns_search", ctypes.c_size_t), ("h_columns_fp64", ctypes.c_size_t),
                ("s_columns_search", ctypes.c_size_t), ("s_columns_fp64", ctypes.c_size_t),
                ("rayleigh_ritz_calls", ctypes.c_int), ("restarts", ctypes.c_int), ("fp64_refreshes", ctypes.c_int),
                ("certifications", ctypes.c_int), ("handoff_iteration", ctypes.c_int),
                ("block_rank_fallbacks", ctypes.c_int), ("correction_columns", ctypes.c_size_t),
                ("polish_steps", ctypes.c_int), ("polish_accepted", ctypes.c_int), ("manifold_steps", ctypes.c_int),
                ("manifold_accepted", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _declare(lib: ctypes.CDLL) -> None:
    def fn(name, args, res=ctypes.c_int):
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res

    fn("sdft_b200_last_error", [ctypes.c_char_p, SZ], SZ)
    fn("sdft_b200_version", [], ctypes.c_char_p)
    fn("sdft_b200_kernel_launches", [], ctypes.c_ulonglong)
    fn("sdft_b200_context_create", [ctypes.c_int, P, ctypes.POINTER(P)])
    fn("sdft_b200_context_destroy", [P])
    fn("sdft_b200_context_synchronize", [P])
    fn("sdft_b200_context_release_memory", [P])
    fn("sdft_b200_enumerate_g_vectors", [D, ctypes.c_double, D, ctypes.c_double, I32, D, D, SZ, SZP])
    fn("sdft_b200_operator_create", [P, SZ, I32, D, SZ, I32, D, SZ, U64, D, D, D, ctypes.c_double, ctypes.c_double,
                                     ctypes.POINTER(P)])
    fn("sdft_b200_operator_destroy", [P])
    fn("sdft_b200_operator_update", [P, SZ, I32, D, D, D])
    fn("sdft_b200_rmm_trial", [P, ctypes.POINTER(DavidsonOptions), P, D, P, D, ctypes.POINTER(DavidsonStats),
                               ctypes.POINTER(ctypes.c_int), ctypes.c_int])
    fn("sdft_b200_band_groups", [P, ctypes.POINTER(DavidsonOptions), P, D, P, D, ctypes.POINTER(DavidsonStats),
                                 ctypes.c_int])
    fn("sdft_b200_density_functionals", [P, D, SZ, I32, D, SZ, I32, D, ctypes.c_int, I32, D, D, SZ, SZP,
                                         ctypes.POINTER(Functionals)])
    fn("sdft_b200_collinear_functionals", [P, D, SZ, I32, D, SZ, I32, D, SZ, I32, D, ctypes.c_int, I32, D, D, D, D,
                                           SZ, SZP, ctypes.POINTER(Functionals)])
    fn("sdft_b200_operator_info", [P, I32, SZP, SZP, SZP, SZP])
    fn("sdft_b200_operator_metric_signature", [P, D, ctypes.POINTER(ctypes.c_int)])
    fn("sdft_b200_apply_local", [P, P, SZ, P, ctypes.c_int, ctypes.c_int])
    fn("sdft_b200_apply_local_noalloc", [P, P, SZ, P, ctypes.c_int])
    fn("sdft_b200_pbe_points", [P, P, P, SZ, P, ctypes.c_int])
    fn("sdft_b200_rayleigh_ritz", [P, SZ, SZ, P, P, P, P, ctypes.c_int])
    fn("sdft_b200_band_density", [P, I32, SZ, P, D, SZ, ctypes.c_double, I32, SZ, P, ctypes.c_int])
    fn("sdft_b200_onsite_density", [P, SZ, SZ, SZ, P, SZ, D, P, ctypes.c_int])
    fn("sdft_b200_compensation_create", [P, D, SZ, D, I32, SZ, ctypes.c_int, SZ, D, D, SZ, D, ctypes.POINTER(P)])
    fn("sdft_b200_compensation_destroy", [P])
    fn("sdft_b200_compensation_density", [P, P, P, ctypes.c_int])
    fn("sdft_b200_compensation_project", [P, P, P, ctypes.c_int])
    fn("sdft_b200_local_hamiltonian", [P, I32, U64, SZ, D, D, P, SZ, P, ctypes.c_int, ctypes.c_uint64])
    fn("sdft_b200_paw_pair", [P, ctypes.c_uint64, SZ, SZ, SZ, P, P, P, P, P, P, ctypes.c_int, ctypes.c_uint64])
    fn("sdft_b200_complex_gemm", [P, ctypes.c_int, ctypes.c_int, SZ, SZ, SZ, P, SZ, P, SZ, P, SZ, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int])
    fn("sdft_b200_complex_gemm_immutable_left", [P, ctypes.c_uint64, ctypes.c_int, SZ, SZ, SZ, P, SZ, P, SZ, P, SZ,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_int])
    fn("sdft_b200_complex_gemm_triple_right", [P, SZ, SZ, SZ, ctypes.POINTER(P), SZ, P, SZ, ctypes.POINTER(P), SZ,
                                               ctypes.c_int, ctypes.c_int])
    fn("sdft_b200_gemm_tuned_classes", [SZ, I32, SZP])
    fn("sdft_b200_operator_arrays", [P, U64, D, D, D, D])
    fn("sdft_b200_apply", [P, ctypes.c_int, P, SZ, P, ctypes.c_int, ctypes.c_int])
    fn("sdft_b200_apply_pair", [P, P, SZ, P, P, ctypes.c_int, ctypes.c_int])
    fn("sdft_b200_project", [P, P, SZ, P, ctypes.c_int, ctypes.c_int])
    fn("sdft_b200_davidson", [P, ctypes.POINTER(DavidsonOptions), P, D, P, D, ctypes.POINTER(DavidsonStats),
                              ctypes.c_int])
    fn("sdft_b200_snapshot_read_info", [ctypes.c_char_p, ctypes.POINTER(SnapshotInfo)])
    fn("sdft_b200_operator_from_snapshot", [P, ctypes.c_char_p, ctypes.POINTER(P), P])
    fn("sdft_b200_server_create", [ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(P)])
    fn("sdft_b200_server_destroy", [P])
    fn("sdft_b200_server_submit", [P, SZ, I32, D, SZ, I32, D, SZ, U64, D, D, D, ctypes.c_double, ctypes.c_double,
                                   ctypes.POINTER(DavidsonOptions), ctypes.c_int, U64])
    fn("sdft_b200_server_wait", [P, ctypes.c_uint64, ctypes.c_double, D, P, D, ctypes.POINTER(DavidsonStats),
                                 ctypes.POINTER(SolveTiming)])
    fn("sdft_b200_server_memory", [P, U64, U64, U64])
    fn("sdft_b200_solve_footprint", [SZ, I32, SZ, SZ, ctypes.c_int, U64])


def gemm_tuned_classes() -> list:
    """The tensor-core GEMM autotuner's table: (rows, real columns, K blocks,
    tile width, split-K count) per shape class, rows and columns rounded up."""
    lib = library()
    count = ctypes.c_size_t()
    check(lib.sdft_b200_gemm_tuned_classes(0, None, ctypes.byref(count)))
    table = np.zeros((max(count.value, 1), 5), dtype=np.int32)
    check(lib.sdft_b200_gemm_tuned_classes(table.shape[0], table.ctypes.data_as(I32), ctypes.byref(count)))
    return [tuple(int(v) for v in row) for row in table[:min(count.value, table.shape[0])]]


def last_error() -> str:
    lib = library()
    buf = ctypes.create_string_buffer(4096)
    lib.sdft_b200_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != OK:
        raise _ERRORS.get(status, SdftError)(status, last_error())
