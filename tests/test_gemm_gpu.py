"""Complex GEMM boundary (the reference's complex_gemm): FP64 and tcgen05 mixed.

Oracle: numpy complex128 products. Bars: FP64 1e-13 relative (Frobenius);
mixed (BF16 split products, FP32 tensor-memory accumulation) 2e-5 relative,
the same bar as the mixed operator applications.
"""
import numpy as np
import pytest

from conftest import relative_error
from sdft_b200.operator import complex_gemm

pytestmark = pytest.mark.gpu

SHAPES = [(512, 160, 3001, False), (300, 17, 130, True), (64, 1, 64, False), (1, 9, 5000, True),
          (700, 40, 512, True), (129, 129, 257, False)]


def random(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("m,n,k,adjoint", SHAPES)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-5)])
def test_complex_gemm_matches_numpy(context, m, n, k, adjoint, precision, tol):
    rng = np.random.default_rng(m * 7919 + n * 31 + k)
    a = random(rng, (k, m) if adjoint else (m, k))
    b = random(rng, (k, n))
    ref = (a.conj().T if adjoint else a) @ b
    out = complex_gemm(context, a, b, adjoint_a=adjoint, precision=precision)
    assert relative_error(out, ref) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-5)])
def test_complex_gemm_accumulates(context, precision, tol):
    rng = np.random.default_rng(5)
    a, b, c = random(rng, (96, 400)), random(rng, (400, 33)), random(rng, (96, 33))
    out = complex_gemm(context, a, b, precision=precision, c=c)
    assert relative_error(out, a @ b + c) < tol


def test_mixed_gemm_is_deterministic(context):
    rng = np.random.default_rng(9)
    a, b = random(rng, (256, 6000)), random(rng, (6000, 48))
    first = complex_gemm(context, a, b, precision="mixed")
    second = complex_gemm(context, a, b, precision="mixed")
    assert np.array_equal(first, second)


@pytest.mark.parametrize("add", [0, 1])
def test_host_gemm_on_submatrix_leaves_other_rows(context, add):
    """C is a row block of a taller host matrix (ldc > m), as in the reference's
    per-atom products into a shared projection array: only the block changes."""
    import ctypes
    from sdft_b200 import _capi as C
    rng = np.random.Generator(np.random.PCG64(17))
    m, n, k, ldc, offset = 8, 13, 8, 40, 16
    a = np.asfortranarray(rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k)))
    b = np.asfortranarray(rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n)))
    full = np.asfortranarray(rng.standard_normal((ldc, n)) + 1j * rng.standard_normal((ldc, n)))
    expected = full.copy(order="F")
    expected[offset:offset + m] = a @ b + (expected[offset:offset + m] if add else 0)
    base = full.ctypes.data + 16 * offset
    C.check(C.library().sdft_b200_complex_gemm(context.handle, 0, 0, m, n, k, ctypes.c_void_p(a.ctypes.data), m,
                                               ctypes.c_void_p(b.ctypes.data), k, ctypes.c_void_p(base), ldc, C.FP64,
                                               add, C.HOST))
    assert np.array_equal(full[:offset], expected[:offset])
    assert np.array_equal(full[offset + m:], expected[offset + m:])
    assert relative_error(full[offset:offset + m], expected[offset:offset + m]) < 1e-14
