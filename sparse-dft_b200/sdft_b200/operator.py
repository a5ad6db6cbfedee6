"""Host-side mirror of the reference's PlaneWaveOperator / HermitianOperator interface.

Thin wrappers over the C ABI: every numerical call runs the CUDA library.
Arrays may be numpy (host memory, synchronous) or torch CUDA tensors (device
memory, asynchronous on the context's stream).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C

_PREC = {"fp64": C.FP64, "mixed": C.MIXED, C.FP64: C.FP64, C.MIXED: C.MIXED}
CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


def _precision(value) -> int:
    try:
        return _PREC[value]
    except KeyError:
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {value!r}") from None


def _dptr(array):
    return array.ctypes.data_as(C.D)


class Context:
    """A CUDA stream plus library handles on one device (the reference's per-thread Accelerator)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        """stream: None for a private stream, or a cudaStream_t handle to share
        (0, torch's default stream, is passed on as cudaStreamLegacy)."""
        self._lib = C.library()
        handle = ctypes.c_void_p()
        raw = None if stream is None else (stream if stream != 0 else CUDA_STREAM_LEGACY)
        C.check(self._lib.sdft_b200_context_create(device, ctypes.c_void_p(raw), ctypes.byref(handle)))
        self.handle = handle
        self.device = device

    def synchronize(self) -> None:
        C.check(self._lib.sdft_b200_context_synchronize(self.handle))

    def release_memory(self) -> None:
        """Frees this context's working buffers and hands the library pool's
        unused device memory back to the device (sdft_b200_context_release_memory)."""
        C.check(self._lib.sdft_b200_context_release_memory(self.handle))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.sdft_b200_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def enumerate_g_vectors(reciprocal, cutoff_ev: float, kpoint=(0.0, 0.0, 0.0), hartree_to_ev: float = 27.211386245988):
    """Plane-wave basis (hkl int32 (n,3), cartesian (n,3), kinetic_ev (n,)) from the library's host code."""
    lib = C.library()
    recip = np.ascontiguousarray(reciprocal, dtype=np.float64).reshape(9)
    k = np.ascontiguousarray(kpoint, dtype=np.float64)
    count = ctypes.c_size_t()
    C.check(lib.sdft_b200_enumerate_g_vectors(_dptr(recip), cutoff_ev, _dptr(k), hartree_to_ev, None, None, None, 0,
                                              ctypes.byref(count)))
    n = count.value
    hkl = np.zeros((n, 3), dtype=np.int32)
    cart = np.zeros((n, 3))
    kin = np.zeros(n)
    C.check(lib.sdft_b200_enumerate_g_vectors(_dptr(recip), cutoff_ev, _dptr(k), hartree_to_ev,
                                              hkl.ctypes.data_as(C.I32), _dptr(cart), _dptr(kin), n,
                                              ctypes.byref(count)))
    return hkl, cart, kin


def snapshot_info(path) -> dict:
    """Header of a solver snapshot (the reference's SDFTPWO3 file), host only."""
    info = C.SnapshotInfo()
    C.check(C.library().sdft_b200_snapshot_read_info(str(path).encode(), ctypes.byref(info)))
    return info.as_dict()


class PlaneWaveOperator:
    """Device-resident H~ and S~ built from the reference's constructor arguments."""

    @classmethod
    def from_snapshot(cls, context: Context, path):
        """Operator from a solver snapshot (the reference's load_solver_snapshot);
        returns (operator, settings) with the snapshot's roots, iterations,
        tolerance and warm vectors (band-major roots x npw, or None)."""
        info = snapshot_info(path)
        warm = np.zeros((info["roots"], info["npw"]), dtype=np.complex128) if info["initial_values"] else None
        self = cls.__new__(cls)
        self.context = context
        self._lib = C.library()
        handle = ctypes.c_void_p()
        C.check(self._lib.sdft_b200_operator_from_snapshot(context.handle, str(path).encode(), ctypes.byref(handle),
                                                           ctypes.c_void_p(warm.ctypes.data) if warm is not None else None))
        self.handle = handle
        self._read_info()
        return self, {"roots": info["roots"], "iterations": info["iterations"], "tolerance": info["tolerance"],
                      "initial": warm}

    def __init__(self, context: Context, inputs):
        self.context = context
        self._lib = C.library()
        x = inputs
        hkl = np.ascontiguousarray(x.hkl, dtype=np.int32)
        kin = np.ascontiguousarray(x.kinetic_ev, dtype=np.float64)
        vh = np.ascontiguousarray(x.v_hkl, dtype=np.int32)
        vv = np.ascontiguousarray(x.v_values, dtype=np.complex128)
        proj = np.ascontiguousarray(x.projectors, dtype=np.uint64)
        amp = np.ascontiguousarray(x.amplitudes, dtype=np.complex128)
        d = np.ascontiguousarray(x.d, dtype=np.complex128)
        q = np.ascontiguousarray(x.q, dtype=np.complex128)
        self._block_entries = int(np.sum(proj.astype(np.int64) ** 2))
        handle = ctypes.c_void_p()
        C.check(self._lib.sdft_b200_operator_create(
            context.handle, hkl.shape[0], hkl.ctypes.data_as(C.I32), _dptr(kin), vh.shape[0],
            vh.ctypes.data_as(C.I32), vv.ctypes.data_as(C.D), proj.size, proj.ctypes.data_as(C.U64),
            amp.ctypes.data_as(C.D), d.ctypes.data_as(C.D), q.ctypes.data_as(C.D), x.hartree_to_ev, x.regularization,
            ctypes.byref(handle)))
        self.handle = handle
        self._read_info()

    def update(self, v_hkl, v_values, d, q) -> None:
        """SCF refresh: new V(G) and per-atom D/Q (the constructor's layouts) on
        the resident basis, FFT plan and B; afterwards the operator equals one
        built from the same basis and amplitudes with these values. Raises
        (operator unchanged) when a check fails."""
        vh = np.ascontiguousarray(v_hkl, dtype=np.int32).reshape(-1, 3)
        vv = np.ascontiguousarray(v_values, dtype=np.complex128).reshape(-1)
        if vv.shape[0] != vh.shape[0]:
            raise ValueError("potential keys and values disagree")
        dd = np.ascontiguousarray(d, dtype=np.complex128).reshape(-1)
        qq = np.ascontiguousarray(q, dtype=np.complex128).reshape(-1)
        entries = getattr(self, "_block_entries", None)
        if entries is None:
            raise ValueError("an operator read from a snapshot cannot be updated")
        if dd.shape[0] != entries or qq.shape[0] != entries:
            raise ValueError(f"D and Q must hold {entries} entries (sum of projectors per atom squared)")
        C.check(self._lib.sdft_b200_operator_update(self.handle, vh.shape[0], vh.ctypes.data_as(C.I32),
                                                    vv.ctypes.data_as(C.D), dd.ctypes.data_as(C.D),
                                                    qq.ctypes.data_as(C.D)))

    def _read_info(self) -> None:
        handle = self.handle
        shape = np.zeros(3, dtype=np.int32)
        grid = ctypes.c_size_t()
        nproj = ctypes.c_size_t()
        npw = ctypes.c_size_t()
        rows = ctypes.c_size_t()
        C.check(self._lib.sdft_b200_operator_info(handle, shape.ctypes.data_as(C.I32), ctypes.byref(grid),
                                                  ctypes.byref(nproj), ctypes.byref(npw), ctypes.byref(rows)))
        self.shape = tuple(int(v) for v in shape)
        self.grid_points = grid.value
        self.projectors = nproj.value
        self.npw = npw.value
        self.active_rows = rows.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.sdft_b200_operator_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def metric_signature(self) -> dict:
        """Signature of S~ as the reference's overlap() determines it: the lowest
        eigenvalue of (1+reg) I + R Q R (R = (B B^H)^(1/2)), capped at 1+reg,
        and whether S~ is indefinite. Raises SdftError (RUNTIME_ERROR) for a
        numerically singular S~."""
        minimum = ctypes.c_double()
        indefinite = ctypes.c_int()
        C.check(self._lib.sdft_b200_operator_metric_signature(self.handle, ctypes.byref(minimum),
                                                              ctypes.byref(indefinite)))
        return {"minimum": minimum.value, "indefinite": bool(indefinite.value)}

    def arrays(self) -> dict:
        n, count = self.npw, self.grid_points
        out = {"indices": np.zeros(n, dtype=np.uint64), "kinetic": np.zeros(n), "h_diagonal": np.zeros(n),
               "s_diagonal": np.zeros(n), "local_potential": np.zeros(count)}
        C.check(self._lib.sdft_b200_operator_arrays(self.handle, out["indices"].ctypes.data_as(C.U64),
                                                    _dptr(out["kinetic"]), _dptr(out["h_diagonal"]),
                                                    _dptr(out["s_diagonal"]), _dptr(out["local_potential"])))
        return out

    # -- applications --------------------------------------------------------
    def _block(self, x):
        """(pointer, columns, memory, keepalive) for a (npw, cols) block."""
        if hasattr(x, "data_ptr") and getattr(x, "is_cuda", False):
            if x.dtype.__repr__() != "torch.complex128" or x.dim() != 2 or x.shape[0] != self.npw:
                raise ValueError("device blocks must be complex128 tensors of shape (npw, columns)")
            if not (x.stride(0) == 1 and x.stride(1) == self.npw):
                raise ValueError("device blocks must be column-major with leading dimension npw")
            return ctypes.c_void_p(x.data_ptr()), int(x.shape[1]), C.DEVICE, x
        arr = np.asfortranarray(x, dtype=np.complex128)
        if arr.ndim == 1:
            arr = arr.reshape(-1, 1, order="F")
        if arr.shape[0] != self.npw:
            raise ValueError("input rows must equal the plane-wave count")
        return ctypes.c_void_p(arr.ctypes.data), int(arr.shape[1]), C.HOST, arr

    @staticmethod
    def _like(x, rows=None):
        if hasattr(x, "data_ptr") and getattr(x, "is_cuda", False):
            import torch
            r = rows if rows is not None else x.shape[0]
            return torch.empty((x.shape[1], r), dtype=x.dtype, device=x.device).T
        arr = np.asfortranarray(x, dtype=np.complex128)
        if arr.ndim == 1:
            arr = arr.reshape(-1, 1, order="F")
        r = rows if rows is not None else arr.shape[0]
        return np.zeros((r, arr.shape[1]), dtype=np.complex128, order="F")

    def apply(self, x, overlap: bool = False, precision="fp64", out=None):
        ptr, cols, mem, keep = self._block(x)
        y = self._like(keep) if out is None else out
        yptr = ctypes.c_void_p(y.data_ptr() if mem == C.DEVICE else y.ctypes.data)
        C.check(self._lib.sdft_b200_apply(self.handle, C.OVERLAP if overlap else C.HAMILTONIAN, ptr, cols, yptr,
                                          _precision(precision), mem))
        return y

    def local_apply(self, x, out=None, precision="fp64"):
        """T x + V(r) term only (the reference's Accelerator::local_hamiltonian)."""
        ptr, cols, mem, keep = self._block(x)
        y = self._like(keep) if out is None else out
        yptr = ctypes.c_void_p(y.data_ptr() if mem == C.DEVICE else y.ctypes.data)
        C.check(self._lib.sdft_b200_apply_local(self.handle, ptr, cols, yptr, _precision(precision), mem))
        return y

    def local_apply_noalloc(self, x, out, precision="fp64"):
        """local_apply on torch CUDA blocks with all scratch in the library's static
        device array (no allocation in the call; see sdft_b200_apply_local_noalloc)."""
        ptr, cols, mem, _ = self._block(x)
        optr, ocols, omem, _ = self._block(out)
        if mem != C.DEVICE or omem != C.DEVICE or ocols != cols:
            raise ValueError("x and out must be device blocks with the same column count")
        if x.device.index != self.context.device or out.device.index != self.context.device:
            raise ValueError(f"x and out must live on the context's device cuda:{self.context.device}")
        C.check(self._lib.sdft_b200_apply_local_noalloc(self.handle, ptr, cols, optr, _precision(precision)))
        return out

    def apply_pair(self, x, precision="fp64"):
        ptr, cols, mem, keep = self._block(x)
        hy, sy = self._like(keep), self._like(keep)
        hp = ctypes.c_void_p(hy.data_ptr() if mem == C.DEVICE else hy.ctypes.data)
        sp = ctypes.c_void_p(sy.data_ptr() if mem == C.DEVICE else sy.ctypes.data)
        C.check(self._lib.sdft_b200_apply_pair(self.handle, ptr, cols, hp, sp, _precision(precision), mem))
        return hy, sy

    def project(self, x, precision="fp64"):
        ptr, cols, mem, keep = self._block(x)
        p = self._like(keep, rows=self.projectors)
        pp = ctypes.c_void_p(p.data_ptr() if mem == C.DEVICE else p.ctypes.data)
        C.check(self._lib.sdft_b200_project(self.handle, ptr, cols, pp, _precision(precision), mem))
        return p

    # -- eigensolver ---------------------------------------------------------
    def davidson(self, roots: int, max_iterations: int = 256, tolerance: float = 1e-10, precision="fp64",
                 initial=None, subspace_factor: int = 8, handoff: float = 1e-8, vectors: bool = True,
                 correction_steps: int = 0):
        """Lowest eigenpairs of H~x = e S~x (the reference's solve_generalized_hermitian_davidson).

        correction_steps (mixed only): Jacobi-Davidson CG steps per expansion,
        0 = the library default, -1 = the reference's single preconditioner step.
        Returns a dict with eigenvalues, residuals (fresh FP64), eigenvectors
        (band-major roots x npw, or None), converged, iterations and stats.
        """
        opts = C.DavidsonOptions(roots=roots, max_iterations=max_iterations, tolerance=tolerance,
                                 precision=_precision(precision), subspace_factor=subspace_factor, handoff=handoff,
                                 correction_steps=correction_steps)
        stats = C.DavidsonStats()
        eig = np.zeros(roots)
        res = np.zeros(roots)
        init_ptr = None
        keep = None
        if initial is not None:
            keep = np.ascontiguousarray(initial, dtype=np.complex128).reshape(roots, self.npw)
            init_ptr = ctypes.c_void_p(keep.ctypes.data)
        vec = np.zeros((roots, self.npw), dtype=np.complex128) if vectors else None
        vec_ptr = ctypes.c_void_p(vec.ctypes.data) if vec is not None else None
        C.check(self._lib.sdft_b200_davidson(self.handle, ctypes.byref(opts), init_ptr, _dptr(eig), vec_ptr,
                                             _dptr(res), ctypes.byref(stats), C.HOST))
        info = stats.as_dict()
        return {"eigenvalues": eig, "residuals": res, "eigenvectors": vec, "converged": bool(info["converged"]),
                "iterations": int(info["iterations"]), "stats": info}

    def rmm_trial(self, roots: int, initial, max_iterations: int = 256, tolerance: float = 1e-6,
                  precision="mixed", subspace_factor: int = 8, handoff: float = 1e-8):
        """Residual-minimisation trial for an SCF warm solve (the reference's
        solve_generalized_hermitian_rmm_trial): the Davidson result dict plus
        `trial_manifold` (a residual-checked, explicitly not converged block)."""
        opts = C.DavidsonOptions(roots=roots, max_iterations=max_iterations, tolerance=tolerance,
                                 precision=_precision(precision), subspace_factor=subspace_factor, handoff=handoff)
        stats = C.DavidsonStats()
        eig = np.zeros(roots)
        res = np.zeros(roots)
        keep = np.ascontiguousarray(initial, dtype=np.complex128).reshape(roots, self.npw)
        vec = np.zeros((roots, self.npw), dtype=np.complex128)
        manifold = ctypes.c_int(0)
        C.check(self._lib.sdft_b200_rmm_trial(self.handle, ctypes.byref(opts), ctypes.c_void_p(keep.ctypes.data),
                                              _dptr(eig), ctypes.c_void_p(vec.ctypes.data), _dptr(res),
                                              ctypes.byref(stats), ctypes.byref(manifold), C.HOST))
        info = stats.as_dict()
        return {"eigenvalues": eig, "residuals": res, "eigenvectors": vec, "converged": bool(info["converged"]),
                "iterations": int(info["iterations"]), "trial_manifold": bool(manifold.value), "stats": info}

    def band_groups(self, roots: int, max_iterations: int = 256, tolerance: float = 1e-10, precision="fp64",
                    initial=None, subspace_factor: int = 8, handoff: float = 1e-8):
        """Band-group solve (the reference's solve_generalized_hermitian_band_groups):
        the Davidson result dict."""
        opts = C.DavidsonOptions(roots=roots, max_iterations=max_iterations, tolerance=tolerance,
                                 precision=_precision(precision), subspace_factor=subspace_factor, handoff=handoff)
        stats = C.DavidsonStats()
        eig = np.zeros(roots)
        res = np.zeros(roots)
        keep = None if initial is None else np.ascontiguousarray(initial, dtype=np.complex128).reshape(roots, self.npw)
        vec = np.zeros((roots, self.npw), dtype=np.complex128)
        C.check(self._lib.sdft_b200_band_groups(self.handle, ctypes.byref(opts),
                                                None if keep is None else ctypes.c_void_p(keep.ctypes.data),
                                                _dptr(eig), ctypes.c_void_p(vec.ctypes.data), _dptr(res),
                                                ctypes.byref(stats), C.HOST))
        info = stats.as_dict()
        return {"eigenvalues": eig, "residuals": res, "eigenvectors": vec, "converged": bool(info["converged"]),
                "iterations": int(info["iterations"]), "stats": info}


def complex_gemm(context: Context, a, b, adjoint_a: bool = False, precision="fp64", c=None):
    """C = op(A) B (+ c when given), the reference's complex_gemm (host arrays).

    precision 'fp64' is exact FP64; 'mixed' runs BF16 split products on the
    tensor cores with FP32 accumulation.
    """
    lib = C.library()
    a = np.asfortranarray(a, dtype=np.complex128)
    b = np.asfortranarray(b, dtype=np.complex128)
    m = a.shape[1] if adjoint_a else a.shape[0]
    k = a.shape[0] if adjoint_a else a.shape[1]
    if b.shape[0] != k:
        raise ValueError("inner dimensions differ")
    n = b.shape[1]
    add = c is not None
    out = np.asfortranarray(c, dtype=np.complex128).copy(order="F") if add else np.zeros((m, n), np.complex128, order="F")
    C.check(lib.sdft_b200_complex_gemm(context.handle, 1 if adjoint_a else 0, 0, m, n, k, ctypes.c_void_p(a.ctypes.data),
                                       a.shape[0], ctypes.c_void_p(b.ctypes.data), b.shape[0],
                                       ctypes.c_void_p(out.ctypes.data), m, _precision(precision), int(add), C.HOST))
    return out


def complex_gemm_immutable_left(context: Context, identity: int, a, b, adjoint_a: bool = False, precision="fp64",
                                c=None):
    """C = op(A) B (+ c when given) with A cached on the device for `identity`
    (the reference's complex_gemm_immutable_left; host arrays)."""
    lib = C.library()
    a = np.asfortranarray(a, dtype=np.complex128)
    b = np.asfortranarray(b, dtype=np.complex128)
    m = a.shape[1] if adjoint_a else a.shape[0]
    k = a.shape[0] if adjoint_a else a.shape[1]
    if b.shape[0] != k:
        raise ValueError("inner dimensions differ")
    n = b.shape[1]
    add = c is not None
    out = np.asfortranarray(c, dtype=np.complex128).copy(order="F") if add else np.zeros((m, n), np.complex128, order="F")
    C.check(lib.sdft_b200_complex_gemm_immutable_left(
        context.handle, identity, 1 if adjoint_a else 0, m, n, k, ctypes.c_void_p(a.ctypes.data), a.shape[0],
        ctypes.c_void_p(b.ctypes.data), b.shape[0], ctypes.c_void_p(out.ctypes.data), m, _precision(precision),
        int(add), C.HOST))
    return out


def complex_gemm_triple_right(context: Context, lefts, b, precision="fp64"):
    """[A_0 B, A_1 B, A_2 B] for three m x k left operands sharing B (the
    reference's complex_gemm_triple_right; host arrays)."""
    lib = C.library()
    lefts = [np.asfortranarray(x, dtype=np.complex128) for x in lefts]
    if len(lefts) != 3 or any(x.shape != lefts[0].shape for x in lefts):
        raise ValueError("three left operands of one shape")
    b = np.asfortranarray(b, dtype=np.complex128)
    m, k = lefts[0].shape
    if b.shape[0] != k:
        raise ValueError("inner dimensions differ")
    n = b.shape[1]
    outs = [np.zeros((m, n), np.complex128, order="F") for _ in range(3)]
    a_ptrs = (ctypes.c_void_p * 3)(*[x.ctypes.data for x in lefts])
    c_ptrs = (ctypes.c_void_p * 3)(*[x.ctypes.data for x in outs])
    C.check(lib.sdft_b200_complex_gemm_triple_right(context.handle, m, n, k, a_ptrs, m, ctypes.c_void_p(b.ctypes.data),
                                                    k, c_ptrs, m, _precision(precision), C.HOST))
    return outs


def rayleigh_ritz(context: Context, h, s, requested: int = 0):
    """Lowest `requested` (0 = all) solutions of H y = e S y for n x n Hermitian
    H and S (lower triangles referenced), the reference's rayleigh_ritz. Returns
    (values, vectors) with S-orthonormal vector columns (host arrays)."""
    lib = C.library()
    h = np.asfortranarray(h, dtype=np.complex128)
    s = np.asfortranarray(s, dtype=np.complex128)
    n = h.shape[0]
    if h.shape != (n, n) or s.shape != (n, n):
        raise ValueError("h and s must be square and of the same order")
    count = requested or n
    values = np.zeros(count)
    vectors = np.zeros((n, count), dtype=np.complex128, order="F")
    C.check(lib.sdft_b200_rayleigh_ritz(context.handle, n, requested, ctypes.c_void_p(h.ctypes.data),
                                        ctypes.c_void_p(s.ctypes.data), ctypes.c_void_p(values.ctypes.data),
                                        ctypes.c_void_p(vectors.ctypes.data), C.HOST))
    return values, vectors
