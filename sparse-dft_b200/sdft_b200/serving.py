"""Solve server: continuous batching of independent Davidson solves on one GPU.

Host-side binding of the library's server (sdft_b200_server_*): each request
is one operator (one cell, one k-point) and its solve; the library queues it,
admits it once a worker slot is free and its device footprint fits under the
memory cap, and runs admitted solves concurrently, each on its own stream.
This is how uneven k-points and request streams are served: the reference
runs one PlaneWaveOperator and solve per k-team (src/scf_core.cpp:2974-3061).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from .operator import _precision


def _operator_arrays(x):
    return (np.ascontiguousarray(x.hkl, dtype=np.int32), np.ascontiguousarray(x.kinetic_ev, dtype=np.float64),
            np.ascontiguousarray(x.v_hkl, dtype=np.int32), np.ascontiguousarray(x.v_values, dtype=np.complex128),
            np.ascontiguousarray(x.projectors, dtype=np.uint64), np.ascontiguousarray(x.amplitudes, dtype=np.complex128),
            np.ascontiguousarray(x.d, dtype=np.complex128), np.ascontiguousarray(x.q, dtype=np.complex128))


def solve_footprint(inputs, roots: int, subspace_factor: int = 8) -> int:
    """Device bytes the server budgets for this solve."""
    lib = C.library()
    hkl = np.ascontiguousarray(inputs.hkl, dtype=np.int32)
    total = int(np.asarray(inputs.projectors, dtype=np.uint64).sum())
    out = ctypes.c_uint64()
    C.check(lib.sdft_b200_solve_footprint(hkl.shape[0], hkl.ctypes.data_as(C.I32), total, roots, subspace_factor,
                                          ctypes.byref(out)))
    return out.value


class SolveServer:
    """Queue + admission + concurrent workers for independent solves."""

    def __init__(self, device: int = 0, memory_cap: float = 150e9, slots: int = 4):
        self._lib = C.library()
        handle = ctypes.c_void_p()
        C.check(self._lib.sdft_b200_server_create(device, int(memory_cap), slots, ctypes.byref(handle)))
        self.handle = handle
        self._requests = {}

    def submit(self, inputs, roots: int | None = None, tolerance: float = 1e-12, precision="mixed",
               max_iterations: int = 256, subspace_factor: int = 8, handoff: float = 1e-8,
               vectors: bool = False) -> int:
        roots = int(inputs.roots if roots is None else roots)
        hkl, kin, vh, vv, proj, amp, d, q = _operator_arrays(inputs)
        opts = C.DavidsonOptions(roots=roots, max_iterations=max_iterations, tolerance=tolerance,
                                 precision=_precision(precision), subspace_factor=subspace_factor, handoff=handoff)
        ticket = ctypes.c_uint64()
        C.check(self._lib.sdft_b200_server_submit(
            self.handle, hkl.shape[0], hkl.ctypes.data_as(C.I32), kin.ctypes.data_as(C.D), vh.shape[0],
            vh.ctypes.data_as(C.I32), vv.ctypes.data_as(C.D), proj.size, proj.ctypes.data_as(C.U64),
            amp.ctypes.data_as(C.D), d.ctypes.data_as(C.D), q.ctypes.data_as(C.D), inputs.hartree_to_ev,
            inputs.regularization, ctypes.byref(opts), 1 if vectors else 0, ctypes.byref(ticket)))
        self._requests[ticket.value] = (roots, hkl.shape[0], vectors)
        return ticket.value

    def wait(self, ticket: int, timeout: float | None = None):
        """The solve's result dict, or None when it is not done within timeout
        seconds. A failed solve raises its error."""
        roots, npw, vectors = self._requests.get(ticket, (0, 0, False))
        eig = np.zeros(roots)
        res = np.zeros(roots)
        vec = np.zeros((roots, npw), dtype=np.complex128) if vectors else None
        stats = C.DavidsonStats()
        timing = C.SolveTiming()
        status = self._lib.sdft_b200_server_wait(self.handle, ticket, -1.0 if timeout is None else float(timeout),
                                                 eig.ctypes.data_as(C.D),
                                                 ctypes.c_void_p(vec.ctypes.data) if vec is not None else None,
                                                 res.ctypes.data_as(C.D), ctypes.byref(stats), ctypes.byref(timing))
        if status == C.NOT_READY:
            return None
        self._requests.pop(ticket, None)
        C.check(status)
        info = stats.as_dict()
        return {"eigenvalues": eig, "residuals": res, "eigenvectors": vec, "converged": bool(info["converged"]),
                "iterations": int(info["iterations"]), "stats": info, "timing": timing.as_dict()}

    def memory(self) -> dict:
        cap, used, peak = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        C.check(self._lib.sdft_b200_server_memory(self.handle, ctypes.byref(cap), ctypes.byref(used),
                                                  ctypes.byref(peak)))
        return {"cap": cap.value, "in_use": used.value, "peak": peak.value}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.sdft_b200_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
